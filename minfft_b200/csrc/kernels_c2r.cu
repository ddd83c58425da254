// Instantiations of the one-tile-per-CTA axis-pass kernel for LoadC2R / StoreC2R:
// in-CTA DFT lengths 2^0 .. 2^13, radix 8 and 16 per thread (lengths below 16
// use their own length as the radix; configurations above 512 threads per
// transform do not exist).
#include "axis_pass.cuh"

namespace mb {

const void* axis_kernel_c2r(int log2L, int radix16) {
  static const void* const table[14][2] = {
      {(const void*)axis_pass_kernel<1, 1, LoadC2R, StoreC2R>, (const void*)axis_pass_kernel<1, 1, LoadC2R, StoreC2R>},
      {(const void*)axis_pass_kernel<2, 2, LoadC2R, StoreC2R>, (const void*)axis_pass_kernel<2, 2, LoadC2R, StoreC2R>},
      {(const void*)axis_pass_kernel<4, 4, LoadC2R, StoreC2R>, (const void*)axis_pass_kernel<4, 4, LoadC2R, StoreC2R>},
      {(const void*)axis_pass_kernel<8, 8, LoadC2R, StoreC2R>, (const void*)axis_pass_kernel<8, 8, LoadC2R, StoreC2R>},
      {(const void*)axis_pass_kernel<16, 8, LoadC2R, StoreC2R>, (const void*)axis_pass_kernel<16, 16, LoadC2R, StoreC2R>},
      {(const void*)axis_pass_kernel<32, 8, LoadC2R, StoreC2R>, (const void*)axis_pass_kernel<32, 16, LoadC2R, StoreC2R>},
      {(const void*)axis_pass_kernel<64, 8, LoadC2R, StoreC2R>, (const void*)axis_pass_kernel<64, 16, LoadC2R, StoreC2R>},
      {(const void*)axis_pass_kernel<128, 8, LoadC2R, StoreC2R>, (const void*)axis_pass_kernel<128, 16, LoadC2R, StoreC2R>},
      {(const void*)axis_pass_kernel<256, 8, LoadC2R, StoreC2R>, (const void*)axis_pass_kernel<256, 16, LoadC2R, StoreC2R>},
      {(const void*)axis_pass_kernel<512, 8, LoadC2R, StoreC2R>, (const void*)axis_pass_kernel<512, 16, LoadC2R, StoreC2R>},
      {(const void*)axis_pass_kernel<1024, 8, LoadC2R, StoreC2R>, (const void*)axis_pass_kernel<1024, 16, LoadC2R, StoreC2R>},
      {(const void*)axis_pass_kernel<2048, 8, LoadC2R, StoreC2R>, (const void*)axis_pass_kernel<2048, 16, LoadC2R, StoreC2R>},
      {(const void*)axis_pass_kernel<4096, 8, LoadC2R, StoreC2R>, (const void*)axis_pass_kernel<4096, 16, LoadC2R, StoreC2R>},
      {nullptr, (const void*)axis_pass_kernel<8192, 16, LoadC2R, StoreC2R>},
  };
  return (log2L >= 0 && log2L <= 13) ? table[log2L][radix16 ? 1 : 0] : nullptr;
}

}  // namespace mb
