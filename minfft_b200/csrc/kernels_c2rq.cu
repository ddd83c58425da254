// Instantiations of the one-tile-per-CTA axis-pass kernel for LoadC2RQ / StoreC2R (the
// split column DFT of the 2-D real DFT: four rows per CTA): in-CTA DFT lengths
// 2^4 .. 2^11, radix 8 and 16 per thread, at most 512 threads per CTA.
#include "axis_pass.cuh"

namespace mb {

const void* axis_kernel_c2rq(int log2L, int radix16) {
  static const void* const table[14][2] = {
      {nullptr, nullptr},
      {nullptr, nullptr},
      {nullptr, nullptr},
      {nullptr, nullptr},
      {(const void*)axis_pass_kernel<16, 8, LoadC2RQ, StoreC2R>, (const void*)axis_pass_kernel<16, 16, LoadC2RQ, StoreC2R>},
      {(const void*)axis_pass_kernel<32, 8, LoadC2RQ, StoreC2R>, (const void*)axis_pass_kernel<32, 16, LoadC2RQ, StoreC2R>},
      {(const void*)axis_pass_kernel<64, 8, LoadC2RQ, StoreC2R>, (const void*)axis_pass_kernel<64, 16, LoadC2RQ, StoreC2R>},
      {(const void*)axis_pass_kernel<128, 8, LoadC2RQ, StoreC2R>, (const void*)axis_pass_kernel<128, 16, LoadC2RQ, StoreC2R>},
      {(const void*)axis_pass_kernel<256, 8, LoadC2RQ, StoreC2R>, (const void*)axis_pass_kernel<256, 16, LoadC2RQ, StoreC2R>},
      {(const void*)axis_pass_kernel<512, 8, LoadC2RQ, StoreC2R>, (const void*)axis_pass_kernel<512, 16, LoadC2RQ, StoreC2R>},
      {(const void*)axis_pass_kernel<1024, 8, LoadC2RQ, StoreC2R>, (const void*)axis_pass_kernel<1024, 16, LoadC2RQ, StoreC2R>},
      {nullptr, (const void*)axis_pass_kernel<2048, 16, LoadC2RQ, StoreC2R>},
      {nullptr, nullptr},
      {nullptr, nullptr},
  };
  return (log2L >= 0 && log2L <= 13) ? table[log2L][radix16 ? 1 : 0] : nullptr;
}

}  // namespace mb
