// Instantiations of the axis-pass kernel for the LoadDCT3 / StoreDCT3 combination,
// one per in-CTA DFT length 2^0 .. 2^13.
#include "axis_pass.cuh"

namespace mb {

const void* axis_kernel_dct3(int log2L) {
  static const void* const table[] = {
      (const void*)axis_pass_kernel<1, LoadDCT3, StoreDCT3>,    (const void*)axis_pass_kernel<2, LoadDCT3, StoreDCT3>,
      (const void*)axis_pass_kernel<4, LoadDCT3, StoreDCT3>,    (const void*)axis_pass_kernel<8, LoadDCT3, StoreDCT3>,
      (const void*)axis_pass_kernel<16, LoadDCT3, StoreDCT3>,   (const void*)axis_pass_kernel<32, LoadDCT3, StoreDCT3>,
      (const void*)axis_pass_kernel<64, LoadDCT3, StoreDCT3>,   (const void*)axis_pass_kernel<128, LoadDCT3, StoreDCT3>,
      (const void*)axis_pass_kernel<256, LoadDCT3, StoreDCT3>,  (const void*)axis_pass_kernel<512, LoadDCT3, StoreDCT3>,
      (const void*)axis_pass_kernel<1024, LoadDCT3, StoreDCT3>, (const void*)axis_pass_kernel<2048, LoadDCT3, StoreDCT3>,
      (const void*)axis_pass_kernel<4096, LoadDCT3, StoreDCT3>, (const void*)axis_pass_kernel<8192, LoadDCT3, StoreDCT3>,
  };
  return (log2L >= 0 && log2L <= 13) ? table[log2L] : nullptr;
}

}  // namespace mb
