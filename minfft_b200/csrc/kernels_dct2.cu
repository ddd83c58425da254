// Instantiations of the axis-pass kernel for the LoadDCT2 / StoreDCT2 combination,
// one per in-CTA DFT length 2^0 .. 2^13.
#include "axis_pass.cuh"

namespace mb {

const void* axis_kernel_dct2(int log2L) {
  static const void* const table[] = {
      (const void*)axis_pass_kernel<1, LoadDCT2, StoreDCT2>,    (const void*)axis_pass_kernel<2, LoadDCT2, StoreDCT2>,
      (const void*)axis_pass_kernel<4, LoadDCT2, StoreDCT2>,    (const void*)axis_pass_kernel<8, LoadDCT2, StoreDCT2>,
      (const void*)axis_pass_kernel<16, LoadDCT2, StoreDCT2>,   (const void*)axis_pass_kernel<32, LoadDCT2, StoreDCT2>,
      (const void*)axis_pass_kernel<64, LoadDCT2, StoreDCT2>,   (const void*)axis_pass_kernel<128, LoadDCT2, StoreDCT2>,
      (const void*)axis_pass_kernel<256, LoadDCT2, StoreDCT2>,  (const void*)axis_pass_kernel<512, LoadDCT2, StoreDCT2>,
      (const void*)axis_pass_kernel<1024, LoadDCT2, StoreDCT2>, (const void*)axis_pass_kernel<2048, LoadDCT2, StoreDCT2>,
      (const void*)axis_pass_kernel<4096, LoadDCT2, StoreDCT2>, (const void*)axis_pass_kernel<8192, LoadDCT2, StoreDCT2>,
  };
  return (log2L >= 0 && log2L <= 13) ? table[log2L] : nullptr;
}

}  // namespace mb
