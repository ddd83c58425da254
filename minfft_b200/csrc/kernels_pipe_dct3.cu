// Instantiations of the pipelined axis-pass kernel for PDCT3 / StoreDCT3, one per
// in-CTA DFT length 2^1 .. 2^13 (index 0 is unused).
#include "pipe_pass.cuh"

namespace mb {

const void* pipe_kernel_dct3(int log2L) {
  static const void* const table[] = {
      nullptr,                                           (const void*)axis_pipe_kernel<2, PDCT3, StoreDCT3>,
      (const void*)axis_pipe_kernel<4, PDCT3, StoreDCT3>,    (const void*)axis_pipe_kernel<8, PDCT3, StoreDCT3>,
      (const void*)axis_pipe_kernel<16, PDCT3, StoreDCT3>,   (const void*)axis_pipe_kernel<32, PDCT3, StoreDCT3>,
      (const void*)axis_pipe_kernel<64, PDCT3, StoreDCT3>,   (const void*)axis_pipe_kernel<128, PDCT3, StoreDCT3>,
      (const void*)axis_pipe_kernel<256, PDCT3, StoreDCT3>,  (const void*)axis_pipe_kernel<512, PDCT3, StoreDCT3>,
      (const void*)axis_pipe_kernel<1024, PDCT3, StoreDCT3>, (const void*)axis_pipe_kernel<2048, PDCT3, StoreDCT3>,
      (const void*)axis_pipe_kernel<4096, PDCT3, StoreDCT3>, (const void*)axis_pipe_kernel<8192, PDCT3, StoreDCT3>,
  };
  return (log2L >= 1 && log2L <= 13) ? table[log2L] : nullptr;
}

}  // namespace mb
