// Instantiations of the axis-pass kernel for the LoadC2R / StoreC2R combination,
// one per in-CTA DFT length 2^0 .. 2^13.
#include "axis_pass.cuh"

namespace mb {

const void* axis_kernel_c2r(int log2L) {
  static const void* const table[] = {
      (const void*)axis_pass_kernel<1, LoadC2R, StoreC2R>,    (const void*)axis_pass_kernel<2, LoadC2R, StoreC2R>,
      (const void*)axis_pass_kernel<4, LoadC2R, StoreC2R>,    (const void*)axis_pass_kernel<8, LoadC2R, StoreC2R>,
      (const void*)axis_pass_kernel<16, LoadC2R, StoreC2R>,   (const void*)axis_pass_kernel<32, LoadC2R, StoreC2R>,
      (const void*)axis_pass_kernel<64, LoadC2R, StoreC2R>,   (const void*)axis_pass_kernel<128, LoadC2R, StoreC2R>,
      (const void*)axis_pass_kernel<256, LoadC2R, StoreC2R>,  (const void*)axis_pass_kernel<512, LoadC2R, StoreC2R>,
      (const void*)axis_pass_kernel<1024, LoadC2R, StoreC2R>, (const void*)axis_pass_kernel<2048, LoadC2R, StoreC2R>,
      (const void*)axis_pass_kernel<4096, LoadC2R, StoreC2R>, (const void*)axis_pass_kernel<8192, LoadC2R, StoreC2R>,
  };
  return (log2L >= 0 && log2L <= 13) ? table[log2L] : nullptr;
}

}  // namespace mb
