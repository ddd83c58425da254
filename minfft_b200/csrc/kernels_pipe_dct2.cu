// Instantiations of the pipelined axis-pass kernel for PDCT2 / StoreDCT2, one per
// in-CTA DFT length 2^1 .. 2^13 (index 0 is unused).
#include "pipe_pass.cuh"

namespace mb {

const void* pipe_kernel_dct2(int log2L) {
  static const void* const table[] = {
      nullptr,                                           (const void*)axis_pipe_kernel<2, PDCT2, StoreDCT2>,
      (const void*)axis_pipe_kernel<4, PDCT2, StoreDCT2>,    (const void*)axis_pipe_kernel<8, PDCT2, StoreDCT2>,
      (const void*)axis_pipe_kernel<16, PDCT2, StoreDCT2>,   (const void*)axis_pipe_kernel<32, PDCT2, StoreDCT2>,
      (const void*)axis_pipe_kernel<64, PDCT2, StoreDCT2>,   (const void*)axis_pipe_kernel<128, PDCT2, StoreDCT2>,
      (const void*)axis_pipe_kernel<256, PDCT2, StoreDCT2>,  (const void*)axis_pipe_kernel<512, PDCT2, StoreDCT2>,
      (const void*)axis_pipe_kernel<1024, PDCT2, StoreDCT2>, (const void*)axis_pipe_kernel<2048, PDCT2, StoreDCT2>,
      (const void*)axis_pipe_kernel<4096, PDCT2, StoreDCT2>, (const void*)axis_pipe_kernel<8192, PDCT2, StoreDCT2>,
  };
  return (log2L >= 1 && log2L <= 13) ? table[log2L] : nullptr;
}

}  // namespace mb
