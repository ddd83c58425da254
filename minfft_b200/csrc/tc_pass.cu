// Tensor-core split-precision axis pass (single-precision library).
//
// A batch of complex DFTs of length 256 = 16 x 16 along one axis, computed as
// two radix-16 stages, each a dense 16-point DFT-matrix contraction on the
// 5th-generation tensor cores:
//
//   stage 1: for every transform t and low digit n2, the 16 values
//            x[16*n1 + n2] (n1 = 0..15) are transformed over n1 and result
//            k1 is multiplied by w_256^(n2*k1);
//   stage 2: for every t and k1 the 16 values of stage 1 (n2 = 0..15) are
//            transformed over n2, giving output k1 + 16*k2.
//
// One thread per sub-DFT: a CTA of 16*TB threads holds TB transforms, i.e.
// 16*TB sub-DFTs per stage, in TB/8 groups of 128 rows (one UMMA of M = 128
// per group).  A 16-point complex DFT is the real 32 x 32 matrix
// [[C, S], [-S, C]] (C = cos, S = sin of 2*pi*k*n/16) acting on
// (Re x, Im x), so a stage is D[128 x 32] = A[128 x 32] * B^T with A the
// sub-DFT inputs (K-major, one row per sub-DFT) and B the fixed matrix.
// Tensor cores take FP16 or BF16 operands; to keep FP32 accuracy each
// transform is scaled by a power of two (bringing the largest component of
// its input to [256, 512); the scale is undone when the result is stored)
// and every row of A is split into 16-bit terms, as is B:
//   FP16: A = A0 + A1, B = B0 + B1 (11 + 11 significant bits), D = A0 B0 +
//         A0 B1 + A1 B0                                  (3 products)
//   BF16: A = A0 + A1 + A2 (8 + 8 + 8 bits), likewise B; the six products
//         Ai Bj with i + j <= 2 are kept.
// Products accumulate in FP32 in tensor memory and are read back with
// tcgen05.ld.  The leading product A0 B0 and the correction products go to
// two separate accumulators (32 columns each per group) that are added on the
// CUDA cores: the matrix units round each accumulation step, and keeping the
// long chain of small corrections away from the leading sum leaves only the
// two K steps of A0 B0 to round at full magnitude.  The unscaling and the
// twiddles between the stages also run on the CUDA cores.
//
// In a later pass of a Stockham FFT over HBM (st_ns > 1) every input element
// is first multiplied in FP32 by its pre-twiddle w_Lt^(n * gq), read as the
// product of a coarse and a fine table root, before the scale is chosen; the
// CUDA-core pass applies the same factors.
//
// Synchronisation: warp 0 allocates and frees the TMEM columns; thread 0
// issues the MMAs and commits them to an mbarrier; every thread waits on it
// with a bounded spin.  A wait that runs out records the failure in
// *status, the CTA skips its remaining work, waits once more (bounded) for
// the MMAs in flight, frees its TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>

#include "axis_pass.cuh"
#include "stream_pass.cuh"
#include "tc_pass.h"

namespace mb {

// ------------------------------------------------------------ host side
void tc_split_host(int fmt, float v, uint16_t* terms) {
  float r = v;
  for (int i = 0; i < tc_terms(fmt); ++i) {
    if (fmt == TC_F16) {
      const __half h = __float2half_rn(r);
      terms[i] = __half_as_ushort(h);
      r -= __half2float(h);
    } else {
      const __nv_bfloat16 h = __float2bfloat16_rn(r);
      terms[i] = __bfloat16_as_ushort(h);
      r -= __bfloat162float(h);
    }
  }
}

void tc_bmat_host(int fmt, std::vector<uint16_t>& out) {
  const int nt = tc_terms(fmt);
  out.assign(size_t(nt) * 32 * 32, 0);
  // cos and sin of 2*pi*m/16, zeros exact
  double c16[16], s16[16];
  for (int m = 0; m < 16; ++m) {
    const double a = 2.0 * 3.141592653589793238462643383279502884 * m / 16.0;
    c16[m] = (m % 8 == 4) ? 0.0 : std::cos(a);
    s16[m] = (m % 8 == 0) ? 0.0 : std::sin(a);
  }
  for (int n = 0; n < 32; ++n)
    for (int k = 0; k < 32; ++k) {
      const int m = ((n & 15) * (k & 15)) & 15;
      double v;
      if (n < 16)
        v = k < 16 ? c16[m] : s16[m];
      else
        v = k < 16 ? -s16[m] : c16[m];
      uint16_t t[3];
      tc_split_host(fmt, float(v), t);
      for (int s = 0; s < nt; ++s) out[size_t(s) * 1024 + tc_operand_offset(n, k) / 2] = t[s];
    }
}

#if MINFFT_SINGLE

namespace {

constexpr int kL = kTcLength;
constexpr int kLP = 273;  // tile pitch in complex values: odd, so adjacent columns fall in distinct banks
constexpr int kOpBytes = 128 * 32 * 2;  // A operand of one group: 128 rows x 32 columns x 16 bits
constexpr int kBBytes = 32 * 32 * 2;    // B operand: 32 rows x 32 columns
constexpr long long kSpinLimit = 1LL << 20;

template <int FMT, int TB>
struct TcLayout {
  static constexpr int G = TB / 8;
  static constexpr int NT = FMT == TC_F16 ? 2 : 3;
  // A operands (written after the tile has been read into registers) and
  // the data tile share one region
  static constexpr int a_bytes = NT * G * kOpBytes;
  static constexpr int d_bytes = (TB * kLP * int(sizeof(cpx)) + 15) / 16 * 16;
  static constexpr int region = a_bytes > d_bytes ? a_bytes : d_bytes;
  static constexpr int b_off = region;
  static constexpr int offs_off = b_off + NT * kBBytes;
  static constexpr int gq_off = offs_off + 4 * TB * 8;  // two sets of tile offsets
  static constexpr int mbar_off = gq_off + 2 * TB * 8;   // two sets of pre-twiddle steps
  static constexpr int inv_off = mbar_off + 16;  // per-transform unscale factors
  static constexpr int total = inv_off + (TB * 4 + 15) / 16 * 16;
  static constexpr int tmem_cols = 64 * G;  // per group: leading accumulator, correction accumulator
  static_assert(tmem_cols == 64 * (TB / 8), "tc_tmem_columns");
};

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  // start address >> 4; leading byte offset (between the two 8-column
  // blocks of one K step) 128 B; stride byte offset (between 8-row blocks)
  // 512 B; descriptor version 1; base offset 0; no swizzle
  return uint64_t((saddr >> 4) & 0x3FFF) | (uint64_t(128 >> 4) << 16) | (uint64_t(512 >> 4) << 32) | (1ull << 46);
}

template <int FMT>
__device__ __forceinline__ constexpr uint32_t instr_desc() {
  // D format F32 (bits 4-5), A and B formats (7-9, 10-12: 0 FP16, 1 BF16),
  // both K-major (15, 16 zero), N >> 3 (17-22), M >> 4 (24-28)
  return (1u << 4) | (uint32_t(FMT) << 7) | (uint32_t(FMT) << 10) | (uint32_t(32 >> 3) << 17) |
         (uint32_t(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
      "}\n" ::"r"(dtmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

// Splits the pair (a, b) into NT packed 16-bit pairs (a in the low half),
// each the correctly rounded value of the remainder: one packed conversion
// per term, the remainders formed exactly in FP32.
template <int FMT, int NT>
__device__ __forceinline__ void split_pair(float a, float b, uint32_t (&w)[3]) {
#pragma unroll
  for (int i = 0; i < NT; ++i) {
    if (FMT == TC_F16) {
      const __half2 h = __floats2half2_rn(a, b);
      w[i] = *reinterpret_cast<const uint32_t*>(&h);
      if (i + 1 < NT) {
        const float2 f = __half22float2(h);
        a -= f.x;
        b -= f.y;
      }
    } else {
      const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
      w[i] = *reinterpret_cast<const uint32_t*>(&h);
      if (i + 1 < NT) {
        a -= __uint_as_float(w[i] << 16);
        b -= __uint_as_float(w[i] & 0xFFFF0000u);
      }
    }
  }
}

// 16 consecutive FP32 columns of this warp's 32 TMEM lanes
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&d)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]), "=r"(d[8]),
        "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15])
      : "r"(taddr)
      : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase, long long limit = kSpinLimit) {
  for (long long i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t"
        "}"
        : "=r"(done)
        : "r"(mbar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 2^s for integer s in [-126, 127]
__device__ __forceinline__ float pow2i(int s) { return __int_as_float((127 + s) << 23); }

// The 16 input values this thread moves of tile `tile` (element e = tid +
// i * 16*TB of the tile's TB x 256 values; zero beyond the batch).
template <int TB>
__device__ __forceinline__ void load_tile(const AxisParams& p, const int64_t* offs, int nv, int tid, cpx (&v)[16]) {
  const cpx* in = static_cast<const cpx*>(p.in);
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int e = tid + i * 16 * TB;
    const int c = p.colmode ? (e % TB) : (e / kL);
    const int n = p.colmode ? (e / TB) : (e % kL);
    v[i] = c < nv ? in[offs[c] + int64_t(n) * p.in_n] : czero();
  }
}

// Offsets of the TB transforms of tile `tile` (threads 0..TB-1), and, in a
// later pass of a Stockham FFT over HBM, each transform's pre-twiddle step
// gq = q << st_shift (its element n is multiplied by w_Lt^(n * gq), q the
// span index).
template <int TB>
__device__ __forceinline__ void tile_offsets(const AxisParams& p, int64_t tile, int tid, int64_t* offs, int64_t* gq) {
  if (tid < TB) {
    const int64_t b = tile * TB + tid;
    int64_t b0, oi, oo;
    batch_offsets(p, b < p.nbatch ? b : 0, b0, oi, oo);
    offs[tid] = oi;
    offs[TB + tid] = oo;
    gq[tid] = p.st_ns > 1 ? (udiv(b0, p.st_div) & (p.st_ns - 1)) << p.st_shift : 0;
  }
}

// w_Lt^g as the product of a coarse and a fine table root
__device__ __forceinline__ cpx stockham_root(const AxisParams& p, int64_t g) {
  const int64_t lomask = (int64_t(1) << p.st_lobits) - 1;
  return cmul(ldg(p.st_hi + (g >> p.st_lobits)), ldg(p.st_lo + (g & lomask)));
}

// Persistent: CTA k handles tiles k, k + gridDim.x, ...; while the tensor
// cores work on one tile, the next tile's inputs are already on their way
// into registers.
template <int FMT, int TB>
__global__ void __launch_bounds__(16 * TB, TB == 8 ? 4 : 2) tc256_kernel(const AxisParams p, const TcParams q) {
  using Lay = TcLayout<FMT, TB>;
  constexpr int G = Lay::G, NT = Lay::NT, NTHR = 16 * TB;
  extern __shared__ __align__(128) unsigned char sm[];
  unsigned char* aop = sm;
  cpx* data = reinterpret_cast<cpx*>(sm);
  unsigned char* bop = sm + Lay::b_off;
  int64_t* offs = reinterpret_cast<int64_t*>(sm + Lay::offs_off);  // two sets of 2*TB (tile parity)
  int64_t* gqs = reinterpret_cast<int64_t*>(sm + Lay::gq_off);     // two sets of TB (tile parity)
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + Lay::mbar_off);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + Lay::mbar_off + 8);
  int* bad = reinterpret_cast<int*>(sm + Lay::mbar_off + 12);
  float* invs = reinterpret_cast<float*>(sm + Lay::inv_off);

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  pdl_release();
  pdl_wait();
  const uint32_t mbar_a = static_cast<uint32_t>(__cvta_generic_to_shared(mbar));
  const int64_t ntiles = (p.nbatch + TB - 1) / TB;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(tslot))),
                 "n"(Lay::tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *bad = 0;
  }
  {
    const uint4* src = reinterpret_cast<const uint4*>(q.bmat);
    uint4* dst = reinterpret_cast<uint4*>(bop);
    for (int i = tid; i < NT * kBBytes / 16; i += NTHR) dst[i] = src[i];
  }
  int64_t tile = blockIdx.x;
  tile_offsets<TB>(p, tile, tid, offs, gqs);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;

  const bool cj_in = (p.flags & F_CONJ_IN) != 0, cj_out = (p.flags & F_CONJ_OUT) != 0;
  const bool twid = p.st_ns > 1;
  constexpr uint32_t idesc = instr_desc<FMT>();
  const uint32_t aop_a = static_cast<uint32_t>(__cvta_generic_to_shared(aop));
  const uint32_t bop_a = static_cast<uint32_t>(__cvta_generic_to_shared(bop));
  const int grp = tid >> 7, row = tid & 127;  // UMMA group and row of this thread's sub-DFT
  const int t = tid >> 4, dgt = tid & 15;     // its transform and digit
  bool ok = true;
  bool pending = false;  // MMAs committed and not yet waited for
  bool first = true;     // the first stage of this CTA (test hook: withheld)
  uint32_t phase = 0;
  const long long first_limit = q.wait_polls > 0 ? q.wait_polls : kSpinLimit;

  cpx v[16];
  auto valid = [&](int64_t tl) {
    const int64_t left = p.nbatch - tl * TB;
    return int(left < TB ? left : TB);
  };
  if (tile < ntiles) load_tile<TB>(p, offs, valid(tile), tid, v);

#pragma unroll 1
  for (int par = 0; tile < ntiles && ok; tile += gridDim.x, par ^= 1) {
    const int64_t* cur = offs + par * 2 * TB;
    const int64_t* cur_gq = gqs + par * TB;
    // ---- the tile's inputs into shared memory (the previous tile's store
    // has finished reading it), pre-twiddled in FP32 in a later HBM pass
    if (twid && p.colmode) {
      // column mode: this thread's 16 values are elements n0 + 16*i of
      // transform tid % TB, so their roots are w^(n0*gq) * d^i with
      // d = w^(16*gq): three table roots (w^(n0*gq), d, d^4), the other
      // powers of d as at most two products
      const int64_t gq = cur_gq[tid % TB];
      const cpx base = stockham_root(p, int64_t(tid / TB) * gq);
      const cpx d1 = stockham_root(p, 16 * gq);
      const cpx d2 = cmul(d1, d1);
      const cpx d3 = cmul(d2, d1);
      const cpx d4 = stockham_root(p, 64 * gq);
      const cpx d8 = cmul(d4, d4);
      const cpx d12 = cmul(d8, d4);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int e = tid + i * NTHR;
        const int c = e % TB, n = e / TB;
        cpx w = base;
        if ((i >> 2) == 1) w = cmul(w, d4);
        if ((i >> 2) == 2) w = cmul(w, d8);
        if ((i >> 2) == 3) w = cmul(w, d12);
        if ((i & 3) == 1) w = cmul(w, d1);
        if ((i & 3) == 2) w = cmul(w, d2);
        if ((i & 3) == 3) w = cmul(w, d3);
        cpx x = v[i];
        if (cj_in) x.y = -x.y;
        data[c * kLP + pad16(n)] = cmul(x, w);
      }
    } else {
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int e = tid + i * NTHR;
        const int c = p.colmode ? (e % TB) : (e / kL);
        const int n = p.colmode ? (e / TB) : (e % kL);
        cpx x = v[i];
        if (cj_in) x.y = -x.y;
        if (twid) x = cmul(x, stockham_root(p, int64_t(n) * cur_gq[c]));
        data[c * kLP + pad16(n)] = x;
      }
    }
    const int64_t next = tile + gridDim.x;
    int64_t* nxt = offs + (par ^ 1) * 2 * TB;
    if (next < ntiles) tile_offsets<TB>(p, next, tid, nxt, gqs + (par ^ 1) * TB);
    __syncthreads();
    // ---- the next tile's loads are issued now and land during the stages
    if (next < ntiles) load_tile<TB>(p, nxt, valid(next), tid, v);

#pragma unroll
    for (int stage = 0; stage < 2; ++stage) {
      // ---- this row's inputs: stage 1 x[16*n1 + n2], stage 2 y[16*k1 + n2]
      float re[16], im[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int pos = stage == 0 ? 16 * i + dgt : 16 * dgt + i;
        const cpx u = data[t * kLP + pad16(pos)];
        re[i] = u.x;
        im[i] = u.y;
      }
      // one scale 2^s per transform, from its input: the largest input
      // component goes to [2^8, 2^9); the stage-1 outputs stay scaled (at most
      // 16*sqrt(2)*2^9 < 2^14 in magnitude, inside the FP16 range) and the
      // store unscales
      float sc = 1.f;
      if (stage == 0) {
        float mx = 0.f;
#pragma unroll
        for (int i = 0; i < 16; ++i) mx = fmaxf(mx, fmaxf(fabsf(re[i]), fabsf(im[i])));
#pragma unroll
        for (int o = 8; o >= 1; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));  // the 16 rows
        const int ex = (__float_as_int(mx) >> 23) & 0xFF;  // biased exponent (mx >= 0)
        const int s = min(max(135 - ex, -126), 126);
        sc = pow2i(s);
        if (dgt == 0) invs[t] = pow2i(-s);
      }
      __syncthreads();  // the tile is read: the A operands overwrite it
      // ---- split into NT terms and write the A operands (K: Re 0..15, Im 16..31)
#pragma unroll
      for (int kb = 0; kb < 4; ++kb) {
        uint32_t w[NT][4];
#pragma unroll
        for (int u = 0; u < 8; u += 2) {
          uint32_t o[3];
          const int k = kb * 8 + u;
          const float a = k < 16 ? re[k] : im[k - 16], b = k + 1 < 16 ? re[k + 1] : im[k + 1 - 16];
          if (stage == 0)
            split_pair<FMT, NT>(a * sc, b * sc, o);
          else
            split_pair<FMT, NT>(a, b, o);
#pragma unroll
          for (int z = 0; z < NT; ++z) w[z][u / 2] = o[z];
        }
#pragma unroll
        for (int z = 0; z < NT; ++z)
          *reinterpret_cast<uint4*>(aop + (z * G + grp) * kOpBytes + tc_operand_offset(row, kb * 8)) =
              make_uint4(w[z][0], w[z][1], w[z][2], w[z][3]);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      // ---- the MMAs, two K steps of 16 each: per group, the corrections
      // Ai Bj (0 < i + j < NT, smallest first) into columns 64g+32.., then
      // the leading A0 B0 into columns 64g..
      const bool withheld = first && q.withhold;
      if (tid == 0 && !withheld) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
        for (int g = 0; g < G; ++g) {
          uint32_t acc = 0;
#pragma unroll
          for (int sum = NT - 1; sum >= 1; --sum)
#pragma unroll
            for (int i = 0; i <= sum; ++i) {
              const int j = sum - i;
#pragma unroll
              for (int kh = 0; kh < 2; ++kh) {
                const uint64_t ad = smem_desc(aop_a + (i * G + g) * kOpBytes + kh * 256);
                const uint64_t bd = smem_desc(bop_a + j * kBBytes + kh * 256);
                mma_f16(tmem + uint32_t(64 * g + 32), ad, bd, idesc, acc);
                acc = 1;
              }
            }
#pragma unroll
          for (int kh = 0; kh < 2; ++kh) {
            const uint64_t ad = smem_desc(aop_a + g * kOpBytes + kh * 256);
            const uint64_t bd = smem_desc(bop_a + kh * 256);
            mma_f16(tmem + uint32_t(64 * g), ad, bd, idesc, kh);
          }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar_a)
                     : "memory");
      }
      pending = !withheld;
      if (!mbar_wait(mbar_a, phase, first ? first_limit : kSpinLimit)) atomicExch(bad, 1);
      first = false;
      __syncthreads();
      if (*bad) {
        ok = false;
        break;
      }
      pending = false;
      phase ^= 1;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // ---- this row of D: columns 0..15 Re y_k, 16..31 Im y_k of both
      // accumulators (TMEM lanes 32*(warp % 4) .. +31)
      const uint32_t taddr = tmem + (uint32_t((warp & 3) * 32) << 16) + uint32_t(64 * grp);
      {
        uint32_t d[16], e[16];
        tmem_ld16(taddr, d);
        tmem_ld16(taddr + 32, e);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int k = 0; k < 16; ++k) re[k] = __uint_as_float(d[k]) + __uint_as_float(e[k]);
        tmem_ld16(taddr + 16, d);
        tmem_ld16(taddr + 48, e);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int k = 0; k < 16; ++k) im[k] = __uint_as_float(d[k]) + __uint_as_float(e[k]);
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      // the MMAs have completed (mbarrier), so the A region is free again
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        cpx y = cmk(re[k], im[k]);
        if (stage == 0) {
          y = cmul(y, ldg(p.tw + dgt * k));  // w_256^(n2*k1): n2 = digit, k1 = k
          data[t * kLP + pad16(16 * k + dgt)] = y;
        } else {
          data[t * kLP + pad16(dgt + 16 * k)] = y;  // output k1 + 16*k2 with k1 = digit, k2 = k
        }
      }
      __syncthreads();
    }
    if (!ok) break;

    // ---- store the tile: transform by transform where each transform's
    // outputs are contiguous (rows, and the first pass of a Stockham chain),
    // else adjacent threads on adjacent transforms
    {
      cpx* out = static_cast<cpx*>(p.out);
      const int nv = valid(tile);
      const bool rows_out = !p.colmode || p.out_k == 1;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int e = tid + i * NTHR;
        const int c = rows_out ? (e / kL) : (e % TB);
        const int n = rows_out ? (e % kL) : (e / TB);
        if (c < nv) {
          cpx x = cscale(data[c * kLP + pad16(n)], invs[c]);
          if (cj_out) x.y = -x.y;
          out[cur[TB + c] + int64_t(n) * p.out_k] = x;
        }
      }
    }
    __syncthreads();  // the tile is stored: the next one may overwrite it
  }

  if (!ok) {
    if (tid == 0 && q.status) atomicExch(q.status, 1);
    // the MMAs of the abandoned stage may still be running: give them one
    // more bounded wait (the full limit) before the columns are released;
    // a stage that committed nothing has nothing to wait for
    if (pending) mbar_wait(mbar_a, phase);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(Lay::tmem_cols)
                 : "memory");
  }
}


// ===================================================== streamed TC pass
// The same two radix-16 contractions, on the tile pipeline of the streamed
// column pass (stream_pass.cuh): persistent CTAs of 128 threads (one UMMA
// group of 128 rows, four warps), tiles of 8 transforms of 256 points copied
// into S shared-memory stages by tensor copies (or cp.async where the
// strides do not allow them), an mbarrier per stage.  Small CTAs let four of
// them share an SM in FP16 (three in BF16), so that while one waits for its
// matrix operations or its barriers the others issue: with 256-thread CTAs
// of two groups, two per SM, the pass ran 10-20% slower.
//
// Thread t owns row t of the contraction: in stage 1 the sub-DFT (c, n2) --
// inputs x[16 n1 + n2], n1 = 0..15 -- and in stage 2 the sub-DFT (c, k1) --
// inputs y1[16 k1 + n2] after the twiddles, n2 = 0..15 -- with c the
// transform of the tile and the digit d = n2 (stage 1) or k1 (stage 2):
// column tiles c = t % 8, d = t / 8; row tiles d = t % 16, c = t / 16, so
// that a warp reads contiguous runs of the tile.  Each row is scaled by its
// own power of two (largest component into [2^8, 2^9)), split into NT
// 16-bit terms and written as row t of the K-major A operand; thread 0
// issues the MMAs (corrections into one accumulator, the leading product
// into another) and commits them to an mbarrier; every thread reads its row
// of both accumulators with one tcgen05.ld each, adds them and unscales.
//
// Between the stages the twiddled values go back into the stage, which then
// holds y1 in a layout chosen per tile kind so that the writes (lanes over
// n2) and the reads (lanes over k1) are both conflict-free: column tiles
// (16 k1 + (n2 ^ (k1 & 1))) * 8 + c (a warp's four k1 rows of 64 bytes then
// fall on both halves of the banks), row tiles c * 256 + 16 k1 + (n2 ^ k1).
constexpr int kTcsW = kTcStreamTile;     // transforms per tile
constexpr int kTcsNT = kTcStreamThreads; // threads
constexpr int kTcsG = kTcsNT / 128;      // UMMA groups of 128 rows
static_assert(kTcsW * 16 == kTcsNT, "one contraction row per thread");
constexpr int kTcsStages = 2;

template <int FMT>
struct TcsLayout {
  static constexpr int NT = FMT == TC_F16 ? 2 : 3;
  static constexpr int bar_bytes = 128;                  // mbarriers, TMEM slot, flag
  static constexpr int b_off = bar_bytes;                // B operands: NT x 2 KB
  static constexpr int tw_off = b_off + NT * kBBytes;    // w_256^(d k1) at 16 k1 + d (2 KB)
  static constexpr int a_off = tw_off + kL * 8;          // A operands: groups x NT x 8 KB
  static constexpr int st_off = a_off + kTcsG * NT * kOpBytes;
  static constexpr int tmem_cols = 64 * kTcsG;           // groups x (leading, correction) x 32
  static_assert(tmem_cols == kTcStreamTmemCols, "tensor-memory columns");
};

__host__ __device__ inline int tcs_stage_bytes() { return (kTcsW * (kL + 1) * 8 + 127) / 128 * 128; }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&d)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]), "=r"(d[8]),
        "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15]), "=r"(d[16]),
        "=r"(d[17]), "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]), "=r"(d[22]), "=r"(d[23]), "=r"(d[24]),
        "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]), "=r"(d[29]), "=r"(d[30]), "=r"(d[31])
      : "r"(taddr)
      : "memory");
}

// Power-of-two scale putting the largest component of 16 complex values
// into [2^8, 2^9): returns the scale; *inv receives its inverse.
__device__ __forceinline__ float tcs_scale(const float (&re)[16], const float (&im)[16], float* inv) {
  float mx = 0.f;
#pragma unroll
  for (int i = 0; i < 16; ++i) mx = fmaxf(mx, fmaxf(fabsf(re[i]), fabsf(im[i])));
  const int ex = (__float_as_int(mx) >> 23) & 0xFF;
  const int s = min(max(135 - ex, -126), 126);
  *inv = pow2i(-s);
  return pow2i(s);
}

// Split row (re, im) * sc into NT terms and write them as row `row` of the
// K-major A operands of group g (K: Re 0..15, Im 16..31).
template <int FMT>
__device__ __forceinline__ void tcs_write_a(unsigned char* aop, int g, int row, const float (&re)[16],
                                            const float (&im)[16], float sc) {
  constexpr int NT = TcsLayout<FMT>::NT;
#pragma unroll
  for (int kb = 0; kb < 4; ++kb) {
    uint32_t w[NT][4];
#pragma unroll
    for (int u = 0; u < 8; u += 2) {
      uint32_t o[3];
      const int k = kb * 8 + u;
      const float a = k < 16 ? re[k] : im[k - 16], b = k + 1 < 16 ? re[k + 1] : im[k + 1 - 16];
      split_pair<FMT, NT>(a * sc, b * sc, o);
#pragma unroll
      for (int z = 0; z < NT; ++z) w[z][u / 2] = o[z];
    }
#pragma unroll
    for (int z = 0; z < NT; ++z)
      *reinterpret_cast<uint4*>(aop + (z * kTcsG + g) * kOpBytes + tc_operand_offset(row, kb * 8)) =
          make_uint4(w[z][0], w[z][1], w[z][2], w[z][3]);
  }
}

// Thread 0: the MMAs of both groups for the A operands in place, committed
// to mbarrier `mb`.
template <int FMT>
__device__ __forceinline__ void tcs_issue_mma(uint32_t aop_a, uint32_t bop_a, uint32_t tmem, uint32_t mb) {
  constexpr int NT = TcsLayout<FMT>::NT;
  constexpr uint32_t idesc = instr_desc<FMT>();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
  for (int g = 0; g < kTcsG; ++g) {
    uint32_t acc = 0;
#pragma unroll
    for (int sum = NT - 1; sum >= 1; --sum)
#pragma unroll
      for (int i = 0; i <= sum; ++i) {
        const int j = sum - i;
#pragma unroll
        for (int kh = 0; kh < 2; ++kh) {
          const uint64_t ad = smem_desc(aop_a + (i * kTcsG + g) * kOpBytes + kh * 256);
          const uint64_t bd = smem_desc(bop_a + j * kBBytes + kh * 256);
          mma_f16(tmem + uint32_t(64 * g + 32), ad, bd, idesc, acc);
          acc = 1;
        }
      }
#pragma unroll
    for (int kh = 0; kh < 2; ++kh) {
      const uint64_t ad = smem_desc(aop_a + g * kOpBytes + kh * 256);  // term 0 of group g
      const uint64_t bd = smem_desc(bop_a + kh * 256);
      mma_f16(tmem + uint32_t(64 * g), ad, bd, idesc, kh);
    }
  }
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb) : "memory");
}

// This thread's row of both accumulators, summed: re[k], im[k], k = 0..15.
__device__ __forceinline__ void tcs_read_d(uint32_t tmem, int warp, float (&re)[16], float (&im)[16]) {
  const uint32_t taddr = tmem + (uint32_t((warp & 3) * 32) << 16) + uint32_t(64 * (warp >> 2));
  uint32_t d[32], e[32];
  tmem_ld32(taddr, d);
  tmem_ld32(taddr + 32, e);
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    re[k] = __uint_as_float(d[k]) + __uint_as_float(e[k]);
    im[k] = __uint_as_float(d[16 + k]) + __uint_as_float(e[16 + k]);
  }
}

template <int FMT, bool ROWS>
__global__ void __launch_bounds__(kTcsNT, FMT == TC_F16 ? 4 : 3) tc_stream_kernel(const AxisParams p, const TcParams q,
                                                              const __grid_constant__ CUtensorMap tmap) {
  using Lay = TcsLayout<FMT>;
  constexpr int NT = Lay::NT;
  constexpr int W = kTcsW;
  extern __shared__ __align__(1024) unsigned char sm[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm);  // [0, 8): stage barriers, [8]: MMA barrier
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + 80);
  int* bad = reinterpret_cast<int*>(sm + 84);
  unsigned char* bop = sm + Lay::b_off;
  cpx* tws = reinterpret_cast<cpx*>(sm + Lay::tw_off);
  unsigned char* aop = sm + Lay::a_off;
  unsigned char* stages = sm + Lay::st_off;
  const int S = p.cpb;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int c = ROWS ? tid / 16 : tid % kTcsW;  // transform of the tile
  const int d = ROWS ? tid % 16 : tid / kTcsW;  // digit: n2 in stage 1, k1 in stage 2
  const int g = tid >> 7, row = tid & 127;   // UMMA group and row
  const bool tma = (p.flags & F_STREAM_TMA) != 0;
  const uint32_t bar0 = static_cast<uint32_t>(__cvta_generic_to_shared(bars));
  const uint32_t mma_bar = bar0 + 64;
  const uint32_t st0 = static_cast<uint32_t>(__cvta_generic_to_shared(stages));
  const uint32_t aop_a = static_cast<uint32_t>(__cvta_generic_to_shared(aop));
  const uint32_t bop_a = static_cast<uint32_t>(__cvta_generic_to_shared(bop));
  const int sb = p.stage_bytes;
  const int64_t gpd = (p.d0 + W - 1) / W;
  const int64_t ntiles = p.ntiles;

  pdl_release();
  pdl_wait();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(tslot))),
                 "n"(Lay::tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < S; ++s) smbar_init(bar0 + 8 * s, tma ? 1 : kTcsNT);
    smbar_init(mma_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *bad = 0;
  }
  {
    const uint4* src = reinterpret_cast<const uint4*>(q.bmat);
    uint4* dst = reinterpret_cast<uint4*>(bop);
    for (int i = tid; i < NT * kBBytes / 16; i += kTcsNT) dst[i] = src[i];
    // the twiddles between the stages, w_256^(d k1) at k1 * 16 + d: the 16
    // values of d a warp reads for one k1 sit in 16 consecutive slots (no
    // bank conflicts, where reading w_256^m at m = d k1 put up to 8 in one bank)
    for (int i = tid; i < kL; i += kTcsNT) tws[i] = ldg(p.tw + (i >> 4) * (i & 15));
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;

  auto tile_pos = [&](int64_t t, int64_t& c0, int64_t& b1, int64_t& b2) {
    const int64_t rest = udiv(t, gpd);
    c0 = (t - rest * gpd) * W;
    b2 = udiv(rest, p.d1);
    b1 = rest - b2 * p.d1;
  };
  // tile element (transform cc, point n) -> complex index in the stage
  auto pos_in = [&](int cc, int n) { return ROWS ? (n >> 7) * (W * 128) + cc * 128 + (n & 127) : n * W + cc; };

  auto issue = [&](int64_t t, int s) {
    if (t >= ntiles) return;
    int64_t c0, b1, b2;
    tile_pos(t, c0, b1, b2);
    const uint32_t mb = bar0 + 8 * s;
    const uint32_t dst = st0 + uint32_t(s) * uint32_t(sb);
    if (tma) {
      if (tid == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(W * kL * 8) : "memory");
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          // column tiles: box (2W reals = W transforms, 128 points); row
          // tiles: box (256 reals = 128 points, W transforms)
          const int x0 = ROWS ? 256 * h : int(2 * c0);
          const int x1 = ROWS ? int(c0) : 128 * h;
          asm volatile(
              "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
              "[%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst + uint32_t(h * W * 128 * 8)),
              "l"(&tmap), "r"(x0), "r"(x1), "r"(int(b1)), "r"(int(b2)), "r"(mb)
              : "memory");
        }
      }
    } else {
      const int nv = int(p.d0 - c0 < W ? p.d0 - c0 : W);
      const char* src = static_cast<const char*>(p.in) + (b1 * p.is1 + b2 * p.is2 + c0 * p.is0) * 8;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int e = tid + i * kTcsNT;
        const int cc = ROWS ? e / kL : e % W, n = ROWS ? e % kL : e / W;
        if (cc < nv) {
          const char* gp = src + (int64_t(n) * p.in_n + cc * p.is0) * 8;
          const uint32_t dd = dst + uint32_t(pos_in(cc, n) * 8);
          asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dd), "l"(gp) : "memory");
        }
      }
      asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(mb) : "memory");
    }
  };

  for (int s = 0; s < S; ++s) issue(blockIdx.x + int64_t(s) * gridDim.x, s);

  const bool cj_in = (p.flags & F_CONJ_IN) != 0, cj_out = (p.flags & F_CONJ_OUT) != 0;
  const bool rows_out = (p.flags & F_STAGE_ROWS) != 0;
  const bool twid = p.st_ns > 1;
  const long long first_limit = q.wait_polls > 0 ? q.wait_polls : kSpinLimit;
  bool ok = true, pending = false, first = true;
  uint32_t mph = 0;
  int it = 0;
  int64_t t = blockIdx.x;
  for (; t < ntiles; t += gridDim.x, ++it) {
    const int s = it % S;
    if (!smbar_wait(bar0 + 8 * s, uint32_t(it / S) & 1u, kStreamSpinLimit)) atomicExch(bad, 1);
    __syncthreads();
    if (*bad) {
      ok = false;
      break;
    }
    cpx* tile = reinterpret_cast<cpx*>(stages + size_t(s) * sb);
    int64_t c0, b1, b2;
    tile_pos(t, c0, b1, b2);
    const int64_t col = c0 + c;  // this thread's transform (b0 index)
    const bool active = col < p.d0;
    float re[16], im[16], inv;

    // ---- stage 1: row (c, n2 = d), inputs x[16 n1 + d]
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1) {
      const cpx u = tile[pos_in(c, 16 * n1 + d)];
      re[n1] = u.x;
      im[n1] = cj_in ? -u.y : u.y;
    }
    if (twid) {
      // pre-twiddle of a later pass of a Stockham chain: element n = 16 n1 + d
      // times w_Lt^(n * gq) = w^(d*gq) * (w^(16*gq))^n1
      const int64_t gq = (udiv(col, p.st_div) & (p.st_ns - 1)) << p.st_shift;
      const cpx base = stockham_root(p, int64_t(d) * gq);
      const cpx d1 = stockham_root(p, 16 * gq);
      const cpx d2 = cmul(d1, d1);
      const cpx d3 = cmul(d2, d1);
      const cpx d4 = stockham_root(p, 64 * gq);
      const cpx d8 = cmul(d4, d4);
      const cpx d12 = cmul(d8, d4);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        cpx w = base;
        if ((i >> 2) == 1) w = cmul(w, d4);
        if ((i >> 2) == 2) w = cmul(w, d8);
        if ((i >> 2) == 3) w = cmul(w, d12);
        if ((i & 3) == 1) w = cmul(w, d1);
        if ((i & 3) == 2) w = cmul(w, d2);
        if ((i & 3) == 3) w = cmul(w, d3);
        const cpx x = cmul(cmk(re[i], im[i]), w);
        re[i] = x.x;
        im[i] = x.y;
      }
    }
    float sc = tcs_scale(re, im, &inv);
    tcs_write_a<FMT>(aop, g, row, re, im, sc);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    const bool withheld = first && q.withhold;
    if (tid == 0 && !withheld) tcs_issue_mma<FMT>(aop_a, bop_a, tmem, mma_bar);
    pending = !withheld;
    if (!smbar_wait(mma_bar, mph, first ? first_limit : kSpinLimit)) atomicExch(bad, 1);
    first = false;
    __syncthreads();
    if (*bad) {
      ok = false;
      break;
    }
    pending = false;
    mph ^= 1;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    tcs_read_d(tmem, warp, re, im);
    // unscale and twiddle: y1[k1][n2] * w_256^(n2 k1), n2 = d; into the stage
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) {
      const cpx w = tws[16 * k1 + d];
      const cpx y = cmul(cmk(re[k1] * inv, im[k1] * inv), w);
      const int idx = ROWS ? c * kL + 16 * k1 + (d ^ k1) : (16 * k1 + (d ^ (k1 & 1))) * W + c;
      tile[idx] = y;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();

    // ---- stage 2: row (c, k1 = d), inputs y1[16 d + n2], n2 = 0..15
#pragma unroll
    for (int n2 = 0; n2 < 16; ++n2) {
      const int idx = ROWS ? c * kL + 16 * d + (n2 ^ d) : (16 * d + (n2 ^ (d & 1))) * W + c;
      const cpx u = tile[idx];
      re[n2] = u.x;
      im[n2] = u.y;
    }
    sc = tcs_scale(re, im, &inv);
    tcs_write_a<FMT>(aop, g, row, re, im, sc);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (tid == 0) tcs_issue_mma<FMT>(aop_a, bop_a, tmem, mma_bar);
    pending = true;
    if (!smbar_wait(mma_bar, mph, kSpinLimit)) atomicExch(bad, 1);
    __syncthreads();
    if (*bad) {
      ok = false;
      break;
    }
    pending = false;
    mph ^= 1;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    tcs_read_d(tmem, warp, re, im);
    const float so = cj_out ? -inv : inv;
    // outputs y[k1 + 16 k2], k1 = d
    cpx* out = static_cast<cpx*>(p.out);
    const int64_t ob = b1 * p.os1 + b2 * p.os2;
    if (!rows_out) {
      if (active) {
        cpx* o = out + ob + col * p.os0 + int64_t(d) * p.out_k;
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) o[int64_t(16 * k2) * p.out_k] = cmk(re[k2] * inv, im[k2] * so);
      }
    } else {
      // contiguous outputs per transform: transpose through the stage
      // (transform c at c*(256+1)), then store with k running fastest
#pragma unroll
      for (int k2 = 0; k2 < 16; ++k2) tile[c * (kL + 1) + d + 16 * k2] = cmk(re[k2] * inv, im[k2] * so);
      __syncthreads();
      const int nv = int(p.d0 - c0 < W ? p.d0 - c0 : W);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int e = tid + i * kTcsNT;
        const int cc = e / kL, k = e % kL;
        if (cc < nv) out[ob + (c0 + cc) * p.os0 + int64_t(k) * p.out_k] = tile[cc * (kL + 1) + k];
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();  // the stage and the accumulators are free
    if (tma && tid == 0) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    issue(t + int64_t(S) * gridDim.x, s);
  }

  if (!ok) {
    if (tid == 0 && q.status) atomicExch(q.status, 1);
    if (pending) mbar_wait(mma_bar, mph);
    for (int k = 0; k < S; ++k, ++it, t += gridDim.x) {
      if (t >= ntiles) break;
      smbar_wait(bar0 + 8 * (it % S), uint32_t(it / S) & 1u, kStreamSpinLimit);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(Lay::tmem_cols)
                 : "memory");
  }
}

}  // namespace

const void* tc_kernel(int fmt, int tb) {
  if (fmt == TC_F16) {
    if (tb == 8) return (const void*)tc256_kernel<TC_F16, 8>;
    if (tb == 16) return (const void*)tc256_kernel<TC_F16, 16>;
  } else if (fmt == TC_BF16) {
    if (tb == 8) return (const void*)tc256_kernel<TC_BF16, 8>;
    if (tb == 16) return (const void*)tc256_kernel<TC_BF16, 16>;
  }
  return nullptr;
}

size_t tc_smem(int fmt, int tb) {
  if (fmt == TC_F16) return tb == 8 ? TcLayout<TC_F16, 8>::total : TcLayout<TC_F16, 16>::total;
  return tb == 8 ? TcLayout<TC_BF16, 8>::total : TcLayout<TC_BF16, 16>::total;
}

const void* tc_stream_kernel_fn(int fmt, bool rows) {
  if (fmt == TC_F16) return rows ? (const void*)tc_stream_kernel<TC_F16, true> : (const void*)tc_stream_kernel<TC_F16, false>;
  if (fmt == TC_BF16)
    return rows ? (const void*)tc_stream_kernel<TC_BF16, true> : (const void*)tc_stream_kernel<TC_BF16, false>;
  return nullptr;
}

size_t tc_stream_smem(int fmt, int stages) {
  const size_t st = fmt == TC_F16 ? TcsLayout<TC_F16>::st_off : TcsLayout<TC_BF16>::st_off;
  return st + size_t(stages) * tcs_stage_bytes();
}

int tc_stream_stage_bytes() { return tcs_stage_bytes(); }

#else

const void* tc_kernel(int, int) { return nullptr; }
size_t tc_smem(int, int) { return 0; }
const void* tc_stream_kernel_fn(int, bool) { return nullptr; }
size_t tc_stream_smem(int, int) { return 0; }
int tc_stream_stage_bytes() { return 0; }

#endif

}  // namespace mb
