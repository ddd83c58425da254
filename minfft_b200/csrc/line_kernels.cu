// Standalone pre- and post-processing kernels for real-data transforms whose
// half-length complex DFT is too long for one CTA (it then runs as several
// HBM passes, see plan.cu), plus the length-1 axis kernels.  The element-wise
// steps themselves are in line_ops.cuh.
#include <type_traits>

#include "line_ops.cuh"

namespace mb {

namespace {

template <class Op, class = void>
struct HasItem32 : std::false_type {};
template <class Op>
struct HasItem32<Op, std::void_t<decltype(&Op::item32)>> : std::true_type {};

// Grid-stride walk over the items; steps with a 32-bit form (Op::item32)
// take it when Op::fast(p) holds for the whole launch.
template <class Op>
__global__ void k_line(const LineParams p) {
  pdl_release();
  pdl_wait();
  if constexpr (HasItem32<Op>::value) {
    if (Op::fast(p)) {
      const uint32_t total = Op::count32(p), stride = gridDim.x * blockDim.x;
      for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) Op::item32(p, e);
      return;
    }
  }
  const int64_t total = Op::count(p);
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x)
    Op::item(p, e);
}

}  // namespace

const void* line_kernel(int which) {
  switch (which) {
    case LK_DCT2_PRE: return (const void*)k_line<Op_dct2_pre>;
    case LK_T4_PRE: return (const void*)k_line<Op_t4_pre>;
    case LK_C2R_PACK: return (const void*)k_line<Op_c2r_pack>;
    case LK_DCT3_PACK: return (const void*)k_line<Op_dct3_pack>;
    case LK_R2C_UNPACK: return (const void*)k_line<Op_r2c_unpack>;
    case LK_DCT2_POST: return (const void*)k_line<Op_dct2_post>;
    case LK_DCT3_POST: return (const void*)k_line<Op_dct3_post>;
    case LK_T4_POST: return (const void*)k_line<Op_t4_post>;
    case LK_UNIT: return (const void*)k_line<Op_unit>;
    default: return nullptr;
  }
}

}  // namespace mb
