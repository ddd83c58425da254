// Instantiations of the pipelined axis-pass kernel for PCplx / StoreCplx, one per
// in-CTA DFT length 2^1 .. 2^13 (index 0 is unused).
#include "pipe_pass.cuh"

namespace mb {

const void* pipe_kernel_cplx(int log2L) {
  static const void* const table[] = {
      nullptr,                                           (const void*)axis_pipe_kernel<2, PCplx, StoreCplx>,
      (const void*)axis_pipe_kernel<4, PCplx, StoreCplx>,    (const void*)axis_pipe_kernel<8, PCplx, StoreCplx>,
      (const void*)axis_pipe_kernel<16, PCplx, StoreCplx>,   (const void*)axis_pipe_kernel<32, PCplx, StoreCplx>,
      (const void*)axis_pipe_kernel<64, PCplx, StoreCplx>,   (const void*)axis_pipe_kernel<128, PCplx, StoreCplx>,
      (const void*)axis_pipe_kernel<256, PCplx, StoreCplx>,  (const void*)axis_pipe_kernel<512, PCplx, StoreCplx>,
      (const void*)axis_pipe_kernel<1024, PCplx, StoreCplx>, (const void*)axis_pipe_kernel<2048, PCplx, StoreCplx>,
      (const void*)axis_pipe_kernel<4096, PCplx, StoreCplx>, (const void*)axis_pipe_kernel<8192, PCplx, StoreCplx>,
  };
  return (log2L >= 1 && log2L <= 13) ? table[log2L] : nullptr;
}

}  // namespace mb
