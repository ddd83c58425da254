// Instantiations of the one-tile-per-CTA axis-pass kernel for the first and
// last passes of a 1-D type-4 chain over HBM (the pre-rotation fused into the
// first pass's load, the post-rotation into the last pass's store): pass
// lengths 2^1 .. 2^12, radix 16 (radix 8 from 16 points).
#include "axis_pass.cuh"

namespace mb {

namespace {
template <class Ld, class St>
const void* chain_kernel(int log2L, int radix16) {
  static const void* const table[13][2] = {
      {nullptr, nullptr},
      {(const void*)axis_pass_kernel<2, 2, Ld, St>, (const void*)axis_pass_kernel<2, 2, Ld, St>},
      {(const void*)axis_pass_kernel<4, 4, Ld, St>, (const void*)axis_pass_kernel<4, 4, Ld, St>},
      {(const void*)axis_pass_kernel<8, 8, Ld, St>, (const void*)axis_pass_kernel<8, 8, Ld, St>},
      {(const void*)axis_pass_kernel<16, 8, Ld, St>, (const void*)axis_pass_kernel<16, 16, Ld, St>},
      {(const void*)axis_pass_kernel<32, 8, Ld, St>, (const void*)axis_pass_kernel<32, 16, Ld, St>},
      {(const void*)axis_pass_kernel<64, 8, Ld, St>, (const void*)axis_pass_kernel<64, 16, Ld, St>},
      {(const void*)axis_pass_kernel<128, 8, Ld, St>, (const void*)axis_pass_kernel<128, 16, Ld, St>},
      {(const void*)axis_pass_kernel<256, 8, Ld, St>, (const void*)axis_pass_kernel<256, 16, Ld, St>},
      {(const void*)axis_pass_kernel<512, 8, Ld, St>, (const void*)axis_pass_kernel<512, 16, Ld, St>},
      {(const void*)axis_pass_kernel<1024, 8, Ld, St>, (const void*)axis_pass_kernel<1024, 16, Ld, St>},
      {(const void*)axis_pass_kernel<2048, 8, Ld, St>, (const void*)axis_pass_kernel<2048, 16, Ld, St>},
      {(const void*)axis_pass_kernel<4096, 8, Ld, St>, (const void*)axis_pass_kernel<4096, 16, Ld, St>},
  };
  return (log2L >= 1 && log2L <= 12) ? table[log2L][radix16 ? 1 : 0] : nullptr;
}
}  // namespace

const void* axis_kernel_t4in(int log2L, int radix16) { return chain_kernel<LoadT4Chain, StoreCplx>(log2L, radix16); }
const void* axis_kernel_t4out(int log2L, int radix16) { return chain_kernel<LoadCplx, StoreT4Chain>(log2L, radix16); }

}  // namespace mb
