// Instantiations of the axis-pass kernel for the LoadR2C / StoreR2C combination,
// one per in-CTA DFT length 2^0 .. 2^13.
#include "axis_pass.cuh"

namespace mb {

const void* axis_kernel_r2c(int log2L) {
  static const void* const table[] = {
      (const void*)axis_pass_kernel<1, LoadR2C, StoreR2C>,    (const void*)axis_pass_kernel<2, LoadR2C, StoreR2C>,
      (const void*)axis_pass_kernel<4, LoadR2C, StoreR2C>,    (const void*)axis_pass_kernel<8, LoadR2C, StoreR2C>,
      (const void*)axis_pass_kernel<16, LoadR2C, StoreR2C>,   (const void*)axis_pass_kernel<32, LoadR2C, StoreR2C>,
      (const void*)axis_pass_kernel<64, LoadR2C, StoreR2C>,   (const void*)axis_pass_kernel<128, LoadR2C, StoreR2C>,
      (const void*)axis_pass_kernel<256, LoadR2C, StoreR2C>,  (const void*)axis_pass_kernel<512, LoadR2C, StoreR2C>,
      (const void*)axis_pass_kernel<1024, LoadR2C, StoreR2C>, (const void*)axis_pass_kernel<2048, LoadR2C, StoreR2C>,
      (const void*)axis_pass_kernel<4096, LoadR2C, StoreR2C>, (const void*)axis_pass_kernel<8192, LoadR2C, StoreR2C>,
  };
  return (log2L >= 0 && log2L <= 13) ? table[log2L] : nullptr;
}

}  // namespace mb
