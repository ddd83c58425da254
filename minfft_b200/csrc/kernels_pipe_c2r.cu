// Instantiations of the pipelined axis-pass kernel for PC2R / StoreC2R, one per
// in-CTA DFT length 2^1 .. 2^13 (index 0 is unused).
#include "pipe_pass.cuh"

namespace mb {

const void* pipe_kernel_c2r(int log2L) {
  static const void* const table[] = {
      nullptr,                                           (const void*)axis_pipe_kernel<2, PC2R, StoreC2R>,
      (const void*)axis_pipe_kernel<4, PC2R, StoreC2R>,    (const void*)axis_pipe_kernel<8, PC2R, StoreC2R>,
      (const void*)axis_pipe_kernel<16, PC2R, StoreC2R>,   (const void*)axis_pipe_kernel<32, PC2R, StoreC2R>,
      (const void*)axis_pipe_kernel<64, PC2R, StoreC2R>,   (const void*)axis_pipe_kernel<128, PC2R, StoreC2R>,
      (const void*)axis_pipe_kernel<256, PC2R, StoreC2R>,  (const void*)axis_pipe_kernel<512, PC2R, StoreC2R>,
      (const void*)axis_pipe_kernel<1024, PC2R, StoreC2R>, (const void*)axis_pipe_kernel<2048, PC2R, StoreC2R>,
      (const void*)axis_pipe_kernel<4096, PC2R, StoreC2R>, (const void*)axis_pipe_kernel<8192, PC2R, StoreC2R>,
  };
  return (log2L >= 1 && log2L <= 13) ? table[log2L] : nullptr;
}

}  // namespace mb
