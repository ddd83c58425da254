// Instantiations of the axis-pass kernel for the LoadT4 / StoreT4 combination,
// one per in-CTA DFT length 2^0 .. 2^13.
#include "axis_pass.cuh"

namespace mb {

const void* axis_kernel_t4(int log2L) {
  static const void* const table[] = {
      (const void*)axis_pass_kernel<1, LoadT4, StoreT4>,    (const void*)axis_pass_kernel<2, LoadT4, StoreT4>,
      (const void*)axis_pass_kernel<4, LoadT4, StoreT4>,    (const void*)axis_pass_kernel<8, LoadT4, StoreT4>,
      (const void*)axis_pass_kernel<16, LoadT4, StoreT4>,   (const void*)axis_pass_kernel<32, LoadT4, StoreT4>,
      (const void*)axis_pass_kernel<64, LoadT4, StoreT4>,   (const void*)axis_pass_kernel<128, LoadT4, StoreT4>,
      (const void*)axis_pass_kernel<256, LoadT4, StoreT4>,  (const void*)axis_pass_kernel<512, LoadT4, StoreT4>,
      (const void*)axis_pass_kernel<1024, LoadT4, StoreT4>, (const void*)axis_pass_kernel<2048, LoadT4, StoreT4>,
      (const void*)axis_pass_kernel<4096, LoadT4, StoreT4>, (const void*)axis_pass_kernel<8192, LoadT4, StoreT4>,
  };
  return (log2L >= 0 && log2L <= 13) ? table[log2L] : nullptr;
}

}  // namespace mb
