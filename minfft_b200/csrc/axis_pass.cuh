// One "axis pass": a batch of power-of-two complex DFTs of length L, each
// computed by one group of L/R threads of a CTA, with the pre- and
// post-processing of the transform kind fused into the load and the store.
//
// Addressing.  Transform b of the batch is split as b0 = b % d0,
// b1 = (b / d0) % d1, b2 = b / (d0*d1); its input starts at
// b0*is0 + b1*is1 + b2*is2 and element n sits at +n*in_n (likewise for the
// output with os*, out_k).  This one form covers rows (in_n = 1), columns of
// a C-order array (in_n = product of trailing dims) and the large-length
// passes of a Stockham FFT over HBM (see plan.cu).
//
// Thread layout.  Row mode: the L/R threads of one transform are adjacent,
// so a warp reads consecutive elements of one row.  Column mode: the cpb
// transforms of the CTA are adjacent in memory (consecutive columns), so the
// thread index runs fastest over the transform.  Either way every global
// access of a warp is a contiguous run.
//
// Within the CTA the DFT is a Stockham autosort FFT: thread j of a transform
// holds elements j + r*(L/R), r < R, in registers; each pass multiplies by
// table twiddles, runs an R-point (or smaller) DFT in registers and exchanges
// through padded shared memory.  The last pass leaves output element
// k = j + r*(L/R) in register r, so the first load and the last store need
// no shared memory at all for the plain complex transform.
//
// Kind roots.  The load and store stages multiply by roots w_M^k of the kind
// tables at k = j + i*(L/R).  Thread j reads only table entry j (one load per
// table) and forms the others as w_M^j * w_M^(i*L/R); for the tables used
// here M is 2L, 4L or 8L, so the second factor is the 128th root of unity
// w_128^(i*128L/(M*R)), a constant-memory operand (w128).  When L/R = 1 the
// only thread is j = 0 and w_M^0 = 1 is not read at all.
#pragma once

#include "common.cuh"
#include "roots128.h"

namespace mb {

// w_128^m, m < 32 (m is a compile-time constant once the caller's loop is unrolled)
__device__ __forceinline__ cpx w128(int m) {
#if MINFFT_SINGLE
  return cmk(roots128::kReF[m], roots128::kImF[m]);
#else
  return cmk(roots128::kReD[m], roots128::kImD[m]);
#endif
}

// Entry j of a kind table: the base of this thread's roots (see above).
template <int TPT>
__device__ __forceinline__ cpx kind_base(const cpx* table, int j) {
  if constexpr (TPT == 1) {
    return cmk(real(1), real(0));
  } else {
    return ldg(table + j);
  }
}

struct AxisParams {
  const void* in;
  void* out;
  int64_t nbatch;
  int64_t d0, d1;
  int64_t is0, is1, is2;
  int64_t os0, os1, os2;
  int64_t in_n, out_k;
  const cpx* tw;     // w_L^m, m < L (forward roots for the in-CTA passes)
  const cpx* t1;     // kind table 1 (see the load/store stages)
  const cpx* t2;     // kind table 2
  const cpx* st_hi;  // large-length pass roots: w_Lt^(a << st_lobits)
  const cpx* st_lo;  // large-length pass roots: w_Lt^c, c < 2^st_lobits
  int64_t st_ns;     // span of the preceding HBM passes (1: no pre-twiddle)
  int64_t st_div;    // elements per span index (product of trailing dims)
  int st_shift;      // log2(Lt / (st_ns * L))
  int st_lobits;
  int cpb;      // transforms per CTA (per tile in the pipelined kernel)
  int colmode;  // 1: thread index runs fastest over the transform
  int flags;
  int chunk;    // pipelined kernel: bytes per asynchronous copy (16, 8 or 4)
  int64_t ntiles;       // pipelined kernel: number of tiles
  int64_t gpb;          // pipelined kernel, column mode: tiles per d0 block
  int stage_bytes;      // pipelined kernel: bytes of one shared-memory stage
  int lp;               // shared-memory pitch between transforms (tile_pitch)
  int* status;          // set to 1 by a kernel whose bounded device-side wait ran out
  // type-4 steps fused into the first / last pass of a 1-D chain over HBM:
  // real length N of the line, reals between lines of the real input /
  // output, and the fine-table bits of the post-rotation roots (t1, t2)
  int64_t kn, k_in_line, k_out_line;
  int kbits;
  // streamed row pass: stages in flight, bytes copied per row, bytes
  // between rows of a stage
  int nstages, row_bytes, row_pitch;
};

enum : int {
  F_SRC_SMEM = 1 << 9,  // the input pointer is a shared-memory stage (generic loads, no ld.global)
  F_CONJ_IN = 1,      // conjugate the input (inverse DFT = conj . DFT . conj)
  F_CONJ_OUT = 2,     // conjugate the output
  F_DST = 4,          // sine variant of a real symmetric transform
  F_STAGE_ROWS = 8,   // store through shared memory with k running fastest
  F_VEC = 16,         // real rows are aligned for paired (complex) vector access
};

// Shared-memory tile: cpb transforms of L complex values, transform c at
// c*lp, element p at pad16(p) (one spare slot every 16 elements, so strided
// Stockham scatters spread over all banks).  The pitch lp is skewed by the
// host (tile_pitch) so that the threads of one 128-byte wavefront -- several
// short transforms in row mode, several adjacent columns in column mode --
// land in distinct banks.
struct Tile {
  cpx* s;
  int lp;
  __device__ __forceinline__ int idx(int c, int p) const { return c * lp + pad16(p); }
};

// Pitch (in complex elements) between the transforms of a tile.
__host__ __device__ inline int tile_pitch(int L, int R, int cpb, int colmode) {
  const int W = int(128 / sizeof(cpx));  // complex values per wavefront
  const int tpt = L / (L < R ? L : R);
  int target = 0;
  if (colmode)
    target = cpb >= W ? 1 : W / cpb;
  else if (tpt < W)
    target = tpt;
  int lp = padded_len(L);
  if (target > 0)
    while (lp % W != target % W) ++lp;
  return lp;
}

// Per-thread context: which transform, which thread within it, offsets.
struct Ctx {
  int64_t b;
  int64_t b0;
  int64_t oin, oout;
  int c, j;
  bool active;
};

__device__ __forceinline__ void batch_offsets(const AxisParams& p, int64_t b, int64_t& b0, int64_t& oi, int64_t& oo) {
  const int64_t r = udiv(b, p.d0);
  b0 = b - r * p.d0;
  const int64_t b2 = udiv(r, p.d1);
  const int64_t b1 = r - b2 * p.d1;
  oi = b0 * p.is0 + b1 * p.is1 + b2 * p.is2;
  oo = b0 * p.os0 + b1 * p.os1 + b2 * p.os2;
}

// ------------------------------------------------------------ Stockham core
// u[r] *= w^r for r = 1..RP-1 with w = tw[i1]: two table roots (w, w^4) per
// sub-DFT, the other powers formed just before use as products of at most
// four roundings, so only a handful of roots are live at a time.
template <int RP>
__device__ __forceinline__ void apply_root_powers(cpx* u, const cpx* __restrict__ tw, int i1) {
  static_assert(RP <= 16, "radix up to 16");
  const cpx w1 = ldg(tw + i1);
  u[1] = cmul(u[1], w1);
  if constexpr (RP > 2) {
    const cpx w2 = cmul(w1, w1);
    u[2] = cmul(u[2], w2);
    const cpx w3 = cmul(w2, w1);
    u[3] = cmul(u[3], w3);
    if constexpr (RP > 4) {
      const cpx w4 = ldg(tw + 4 * i1);
      u[4] = cmul(u[4], w4);
      u[5] = cmul(u[5], cmul(w4, w1));
      u[6] = cmul(u[6], cmul(w4, w2));
      u[7] = cmul(u[7], cmul(w4, w3));
      if constexpr (RP > 8) {
        const cpx w8 = cmul(w4, w4);
        u[8] = cmul(u[8], w8);
        u[9] = cmul(u[9], cmul(w8, w1));
        u[10] = cmul(u[10], cmul(w8, w2));
        u[11] = cmul(u[11], cmul(w8, w3));
        const cpx w12 = cmul(w8, w4);
        u[12] = cmul(u[12], w12);
        u[13] = cmul(u[13], cmul(w12, w1));
        u[14] = cmul(u[14], cmul(w12, w2));
        u[15] = cmul(u[15], cmul(w12, w3));
      }
    }
  }
}

template <int L, int R, int RP, int NS>
__device__ __forceinline__ void pass_compute(cpx (&v)[R], int j, const cpx* __restrict__ tw) {
  constexpr int S = R / RP;  // sub-DFTs per thread in this pass
#pragma unroll
  for (int s = 0; s < S; ++s) {
    cpx u[RP];
#pragma unroll
    for (int r = 0; r < RP; ++r) u[r] = v[s + r * S];
    if constexpr (NS > 1) {
      const int jp = j + s * (L / R);
      const int q = jp & (NS - 1);
      constexpr int step = L / (NS * RP);
      apply_root_powers<RP>(u, tw, q * step);
    }
    fft_reg<RP>(u);
#pragma unroll
    for (int r = 0; r < RP; ++r) v[s + r * S] = u[r];
  }
}

// Stockham scatter of a pass with span NS: element r of sub-DFT jp goes to
// B + r*NS with B = (jp/NS)*NS*RP + jp%NS.  Either NS = 1 (B is a multiple of
// RP and r < RP) or NS*RP >= 16 (the part of B above jp%NS is a multiple of
// 16 and jp%NS < NS); in both cases pad16(B + r*NS) = pad16(B) + r*NS +
// ((r*NS) >> 4), so each sub-DFT computes one padded base and the offsets of
// its RP elements are compile-time constants.
template <int L, int R, int RP, int NS>
__device__ __forceinline__ void pass_scatter(const cpx (&v)[R], int j, int c, const Tile& t) {
  constexpr int S = R / RP;
  static_assert(NS == 1 || NS * RP >= 16, "padded offsets are linear in r");
  cpx* tb = t.s + c * t.lp;
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int jp = j + s * (L / R);
    cpx* q = tb + pad16((jp / NS) * (NS * RP) + (jp & (NS - 1)));
#pragma unroll
    for (int r = 0; r < RP; ++r) q[r * NS + ((r * NS) >> 4)] = v[s + r * S];
  }
}

// Padded position of element j + r*(L/R) relative to that of element j
// (TPT = L/R either divides 16 with j < TPT, or is a multiple of 16).
template <int TPT>
__host__ __device__ constexpr int nat_off(int r) {
  return TPT >= 16 ? r * (TPT + TPT / 16) : r * TPT + ((r * TPT) >> 4);
}

template <int L, int R>
__device__ __forceinline__ void gather_natural(cpx (&v)[R], int j, int c, const Tile& t) {
  constexpr int TPT = L / R;
  const cpx* q = t.s + c * t.lp + (TPT >= 16 ? pad16(j) : j);
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = q[nat_off<TPT>(r)];
}

template <int L, int R>
__device__ __forceinline__ void scatter_natural(const cpx (&v)[R], int j, int c, const Tile& t) {
  constexpr int TPT = L / R;
  cpx* q = t.s + c * t.lp + (TPT >= 16 ? pad16(j) : j);
#pragma unroll
  for (int r = 0; r < R; ++r) q[nat_off<TPT>(r)] = v[r];
}

template <int L, int R, int NS>
__device__ __forceinline__ void run_passes(cpx (&v)[R], int j, int c, const Tile& t, const cpx* __restrict__ tw) {
  constexpr int RP = (L / NS >= R) ? R : (L / NS);
  pass_compute<L, R, RP, NS>(v, j, tw);
  if constexpr (NS * RP < L) {
    __syncthreads();
    pass_scatter<L, R, RP, NS>(v, j, c, t);
    __syncthreads();
    gather_natural<L, R>(v, j, c, t);
    run_passes<L, R, NS * RP>(v, j, c, t, tw);
  }
}

// A streaming (evict-first) load from global memory, or a plain load where
// the kernel reads its input from a shared-memory stage (F_SRC_SMEM): the
// streaming form is a global-only instruction.
template <typename T>
__device__ __forceinline__ T src_ld(const T* q, bool smem) {
  return smem ? *q : __ldcs(q);
}

// ------------------------------------------------------------- row staging
// In row mode a transform's real row (N = 2L contiguous reals) is moved
// between global memory and the transform's tile slot in shared memory by its
// TPT threads as 16-byte vectors (single elements when either side is not
// 16-byte aligned), so that strided gathers and scatters (stride 4 elements,
// mirrored halves) happen in shared memory while global memory sees whole
// coalesced 16-byte accesses.  Every thread loads all of its share before
// storing any of it.  The type-3 kinds use it for both their load and their
// store (measured: 18% faster in f64, 11% in f32 on 2048-real rows); the
// type-2 and type-4 kinds were measured slower with it and keep direct
// global accesses.
__device__ __forceinline__ real* tile_row(const Tile& t, int c) { return reinterpret_cast<real*>(t.s + c * t.lp); }

template <int L, int R>
__device__ __forceinline__ void row_g2s(real* sr, const real* g, int j, bool smem = false) {
  constexpr int TPT = L / R;
  constexpr int NV = 2 * L * int(sizeof(real)) / 16;  // 16-byte vectors in the row
  static_assert(NV % TPT == 0, "whole vectors per thread");
  if (((reinterpret_cast<uintptr_t>(g) | reinterpret_cast<uintptr_t>(sr)) & 15) == 0) {
    const uint4* gv = reinterpret_cast<const uint4*>(g) + j;
    uint4* sv = reinterpret_cast<uint4*>(sr) + j;
    uint4 r[NV / TPT];
#pragma unroll
    for (int i = 0; i < NV / TPT; ++i) r[i] = src_ld(gv + i * TPT, smem);
#pragma unroll
    for (int i = 0; i < NV / TPT; ++i) sv[i * TPT] = r[i];
  } else {
    real r[2 * R];
#pragma unroll
    for (int i = 0; i < 2 * R; ++i) r[i] = src_ld(g + j + i * TPT, smem);
#pragma unroll
    for (int i = 0; i < 2 * R; ++i) sr[j + i * TPT] = r[i];
  }
}

template <int L, int R>
__device__ __forceinline__ void row_s2g(real* g, const real* sr, int j) {
  constexpr int TPT = L / R;
  constexpr int NV = 2 * L * int(sizeof(real)) / 16;
  static_assert(NV % TPT == 0, "whole vectors per thread");
  if (((reinterpret_cast<uintptr_t>(g) | reinterpret_cast<uintptr_t>(sr)) & 15) == 0) {
    uint4* gv = reinterpret_cast<uint4*>(g) + j;
    const uint4* sv = reinterpret_cast<const uint4*>(sr) + j;
    uint4 r[NV / TPT];
#pragma unroll
    for (int i = 0; i < NV / TPT; ++i) r[i] = sv[i * TPT];
#pragma unroll
    for (int i = 0; i < NV / TPT; ++i) __stcs(gv + i * TPT, r[i]);
  } else {
    real r[2 * R];
#pragma unroll
    for (int i = 0; i < 2 * R; ++i) r[i] = sr[j + i * TPT];
#pragma unroll
    for (int i = 0; i < 2 * R; ++i) __stcs(g + j + i * TPT, r[i]);
  }
}

// Column mode: thread j of the transform moves reals n = j + m*TPT (m < 2R)
// of its column (element stride s) into the column's tile slot, all loads
// issued before any store; a warp's load covers cpb adjacent columns of a
// few rows.
template <int L, int R>
__device__ __forceinline__ void col_g2s(real* sr, const real* g, int64_t s, int j, bool smem = false) {
  constexpr int TPT = L / R;
  real r[2 * R];
#pragma unroll
  for (int m = 0; m < 2 * R; ++m) r[m] = src_ld(g + int64_t(j + m * TPT) * s, smem);
#pragma unroll
  for (int m = 0; m < 2 * R; ++m) sr[j + m * TPT] = r[m];
}

// row mode with unit element strides
__device__ __forceinline__ bool rows_staged_in(const AxisParams& p) { return !p.colmode && p.in_n == 1; }
__device__ __forceinline__ bool rows_staged_out(const AxisParams& p) { return !p.colmode && p.out_k == 1; }

// ------------------------------------------------- root progressions
// W^(g0 + r*D), r < R, for the root table pair (hi, lo) of W: each table
// root is hi[e >> lobits] * lo[e & (2^lobits - 1)].  Three table roots per
// thread (W^g0, W^D, W^4D); at(r) forms the rest as at most two products, as
// the Stockham passes form theirs (apply_root_powers), just before use so
// that only the seven factors stay live.  Every exponent g0 + r*D must lie
// inside the tables; exponents are 32-bit (the planner keeps the tables
// below 2^32 roots).
template <int R>
struct RootProgression {
  cpx base, d1, d2, d3, d4, d8, d12;
  __device__ __forceinline__ RootProgression(const cpx* __restrict__ hi, const cpx* __restrict__ lo, int lobits,
                                             uint32_t g0, uint32_t D) {
    const uint32_t lomask = (1u << lobits) - 1u;
    auto root = [&](uint32_t e) { return cmul(ldg(hi + (e >> lobits)), ldg(lo + (e & lomask))); };
    base = root(g0);
    d1 = R > 1 ? root(D) : czero();
    d2 = cmul(d1, d1);
    d3 = cmul(d2, d1);
    d4 = R > 4 ? root(4 * D) : czero();
    d8 = cmul(d4, d4);
    d12 = cmul(d8, d4);
  }
  __device__ __forceinline__ cpx at(int r) const {
    const int lo2 = r & 3, hi2 = r >> 2;
    cpx t = base;
    if (hi2 == 1) t = cmul(t, d4);
    if (hi2 == 2) t = cmul(t, d8);
    if (hi2 == 3) t = cmul(t, d12);
    if (lo2 == 1) t = cmul(t, d1);
    if (lo2 == 2) t = cmul(t, d2);
    if (lo2 == 3) t = cmul(t, d3);
    return t;
  }
};

// ------------------------------------------------------- HBM pre-twiddle
// In a pass of a Stockham FFT over HBM, element n of a sub-DFT with span
// index q is multiplied by w_Lt^g, g = q*n*Lt/(st_ns*L), each root read as
// the product of a coarse and a fine table entry.  Thread j holds
// n = j + r*TPT, so its roots are w^g0 * d^r with w^g0 = w_Lt^(q*j*s) and
// d = w_Lt^(q*TPT*s) (s = 2^st_shift): three table roots per thread (w^g0,
// d, d^4), the other powers of d formed as at most two products, as the
// in-CTA passes form theirs (apply_root_powers).
template <int L, int R>
__device__ __forceinline__ void hbm_pretwiddle(cpx (&v)[R], const AxisParams& p, int64_t b0, int j) {
  constexpr int TPT = L / R;
  const int64_t q = udiv(b0, p.st_div) & (p.st_ns - 1);
  const int64_t lomask = (int64_t(1) << p.st_lobits) - 1;
  auto root = [&](int64_t g) { return cmul(ldg(p.st_hi + (g >> p.st_lobits)), ldg(p.st_lo + (g & lomask))); };
  if constexpr (R < 4) {
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = cmul(v[r], root((q * (j + r * TPT)) << p.st_shift));
  } else {
    const int64_t gd = (q * TPT) << p.st_shift;
    const cpx base = root((q * j) << p.st_shift);
    const cpx d1 = root(gd);
    const cpx d2 = cmul(d1, d1);
    const cpx d3 = cmul(d2, d1);
    const cpx d4 = R > 4 ? root(4 * gd) : czero();
    const cpx d8 = cmul(d4, d4);
    const cpx d12 = cmul(d8, d4);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int lo = r & 3, hi = r >> 2;
      cpx w = base;
      if (hi == 1) w = cmul(w, d4);
      if (hi == 2) w = cmul(w, d8);
      if (hi == 3) w = cmul(w, d12);
      if (lo == 1) w = cmul(w, d1);
      if (lo == 2) w = cmul(w, d2);
      if (lo == 3) w = cmul(w, d3);
      v[r] = cmul(v[r], w);
    }
  }
}

// ---------------------------------------------------------------- load ops
// Each load op fills v[r] with complex input element n = j + r*(L/R) of the
// length-L DFT of transform x.b.

// Plain complex input; optional conjugation and large-length pre-twiddle.
struct LoadCplx {
  static constexpr bool kComplexIn = true;  // whether the raw input elements are complex
  static constexpr bool kStaged = false;
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile&, cpx (&v)[R]) {
    constexpr int TPT = L / R;
    const cpx* in = static_cast<const cpx*>(p.in) + x.oin;
    if (!x.active) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = czero();
    } else if (p.in_n == 1) {  // contiguous: compile-time offsets
      const cpx* q = in + x.j;
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = src_ld(q + r * TPT, (p.flags & F_SRC_SMEM) != 0);
    } else {
      const cpx* q = in + x.j * p.in_n;
      const int64_t st = int64_t(TPT) * p.in_n;
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = src_ld(q + r * st, (p.flags & F_SRC_SMEM) != 0);
    }
    if (p.flags & F_CONJ_IN) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r].y = -v[r].y;
    }
    if (p.st_ns > 1) hbm_pretwiddle<L, R>(v, p, x.b0, x.j);
  }
};

// Real row read as L complex pairs (x[2n], x[2n+1]): the half-length complex
// DFT of the real DFT (reference minfft.c:541-543).
struct LoadR2C {
  static constexpr bool kComplexIn = false;  // whether the raw input elements are complex
  static constexpr bool kStaged = false;
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile&, cpx (&v)[R]) {
    constexpr int TPT = L / R;
    const real* in = static_cast<const real*>(p.in) + x.oin;
    if (!x.active) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = czero();
    } else if (p.flags & F_VEC) {
      const cpx* q = reinterpret_cast<const cpx*>(in) + x.j;
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = src_ld(q + r * TPT, (p.flags & F_SRC_SMEM) != 0);
    } else {
      const real* q = in + 2 * x.j;
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = cmk(q[2 * r * TPT], q[2 * r * TPT + 1]);
    }
  }
};

// Type-2 input permutation (reference minfft.c:707-710, 756-759): the
// length-N sequence u_i = x[2i] (i < N/2), u_i = +-x[2N-1-2i] (i >= N/2)
// read as complex pairs (u_2m, u_2m+1); N = 2L.
struct LoadDCT2 {
  static constexpr bool kComplexIn = false;  // whether the raw input elements are complex
  static constexpr bool kStaged = false;
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile&, cpx (&v)[R]) {
    const real* in = static_cast<const real*>(p.in) + x.oin;
    const real sg = (p.flags & F_DST) ? real(-1) : real(1);
    constexpr int N = 2 * L;
    constexpr int TPT = L / R;
    if (!x.active) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = czero();
      return;
    }
    if constexpr (L >= 2) {
      // element m = j + r*TPT lies in the first half (m < L/2) exactly when r < R/2:
      // pair (x[4m], x[4m+2]) there, (x[2N-1-4m], x[2N-3-4m]) (times sg) after
      const int64_t s = p.in_n;
      const real* lo = in + int64_t(4 * x.j) * s;
      const real* hi = in + int64_t(2 * N - 1 - 4 * x.j) * s;
      const int64_t st = int64_t(4 * TPT) * s;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (r < R / 2)
          v[r] = cmk(lo[r * st], lo[r * st + 2 * s]);
        else
          v[r] = cmk(sg * hi[-r * st], sg * hi[-r * st - 2 * s]);
      }
    } else {
      v[0] = cmk(in[0], sg * in[p.in_n]);  // L = 1: u = (x0, +-x1)
    }
  }
};

// Type-4 pre-rotation (reference minfft.c:906-910, 953-957):
// t_n = e_n (x[2n] + i x[N-1-2n]) for DCT-4, -e_n (x[2n] - i x[N-1-2n]) for
// DST-4, with e_n = w_2N^n from table t1.
struct LoadT4 {
  static constexpr bool kComplexIn = false;  // whether the raw input elements are complex
  static constexpr bool kStaged = false;
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile&, cpx (&v)[R]) {
    const real* in = static_cast<const real*>(p.in) + x.oin;
    const bool dst = (p.flags & F_DST) != 0;
    constexpr int N = 2 * L;
    constexpr int TPT = L / R;
    if (!x.active) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = czero();
      return;
    }
    const int64_t s = p.in_n;
    const real* lo = in + int64_t(2 * x.j) * s;
    const real* hi = in + int64_t(N - 1 - 2 * x.j) * s;
    const int64_t st = int64_t(2 * TPT) * s;
    const cpx e = kind_base<TPT>(p.t1, x.j);  // w_2N^j; w_2N^(j + r*TPT) = e * w_4R^r
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const real a = lo[r * st];
      const real b = hi[-r * st];
      const cpx w = cmul(e, w128(r * (32 / R)));
      if (!dst) {
        v[r] = cmul(w, cmk(a, b));
      } else {
        const cpx q = cmul(w, cmk(a, -b));
        v[r] = cmk(-q.x, -q.y);
      }
    }
  }
};

// Packing step of the inverse real DFT (reference minfft.c:628-656) for the
// spectrum pair (z_k, z_{L-k}); returns t_k and t_{L-k}.  f = w_N^k.
__device__ __forceinline__ void pack_pair(cpx za, cpx zb, cpx f, cpx& ta, cpx& tb) {
  const cpx m = cconj(zb);
  const cpx u = cadd(za, m);
  const cpx d = csub(za, m);
  const cpx vv = cmul(d, cmk(f.y, f.x));  // times i*conj(f)
  ta = cadd(u, vv);
  tb = cconj(csub(u, vv));
}

// Unpacking step of the real DFT (reference minfft.c:556-575) for the pair
// (Z_k, Z_{L-k}) of the half-length DFT; returns X_k and X_{L-k}.
__device__ __forceinline__ void unpack_pair(cpx za, cpx zb, cpx f, cpx& xa, cpx& xb) {
  const cpx m = cconj(zb);
  const real h = real(0.5);
  const cpx u = cscale(cadd(za, m), h);
  const cpx d = csub(za, m);
  const cpx vv = cscale(cmul(d, cmk(f.y, -f.x)), h);  // times f/(2i)
  xa = cadd(u, vv);
  xb = cconj(csub(u, vv));
}

// The same without the factor 1/2: returns 2 X_k and 2 X_{L-k} (for the
// type-2 output, which doubles them; scaling by 1/2 and 2 is exact, so the
// results are the same to the bit with two multiplies fewer per value).
__device__ __forceinline__ void unpack_pair2(cpx za, cpx zb, cpx f, cpx& xa, cpx& xb) {
  const cpx m = cconj(zb);
  const cpx u = cadd(za, m);
  const cpx d = csub(za, m);
  const cpx vv = cmul(d, cmk(f.y, -f.x));  // times f/i
  xa = cadd(u, vv);
  xb = cconj(csub(u, vv));
}

// Visits the spectrum pairs (k, L-k), k = 0 .. L/2, owned by thread j of a
// transform: k = j + i*TPT for i = 0 .. R/2 (only j = 0 reaches k = L/2).
// zf(k) reads a spectrum value -- for k = 0 also zf(L), which readers of an
// L-element tile must fold back into range; body(i, k, z_k, z_{L-k})
// consumes the pair.
template <int L, int R, class Zf, class Body>
__device__ __forceinline__ void pair_loop(const Ctx& x, const Zf& zf, const Body& body) {
  constexpr int TPT = L / R;
#pragma unroll
  for (int i = 0; i <= R / 2; ++i) {
    const int k = x.j + i * TPT;
    if (i == R / 2 && x.j != 0) break;
    body(i, k, zf(k), zf(L - k));
  }
}

// w_N^k (N = 2L) at k = j + i*(L/R) from base = w_N^j (kind roots, above);
// used for 0 < k < L/2, i.e. i < R/2 (other i map to w_128^0 and stay
// inside the constant table).
template <int R>
__device__ __forceinline__ cpx rft_root(cpx base, int i) {
  return cmul(base, w128((i < R / 2 ? i : 0) * (64 / R)));
}
// w_4N^k (N = 2L) at k = j + i*(L/R) from base = w_4N^j.
template <int R>
__device__ __forceinline__ cpx t23_root(cpx base, int i) {
  return cmul(base, w128(i * (16 / R)));
}
// w_4N^(L-k) from w_4N^k: w_4N^L = w_8 times the conjugate.
__device__ __forceinline__ cpx t23_mirror(cpx rk) { return cmulc(w128(16), rk); }

// Packs the pair (z_k, z_{L-k}) into the conjugated inverse-DFT inputs t_k,
// t_{L-k} of the tile (k = 0 and k = L/2 are the self-paired ends); f = w_N^k.
__device__ __forceinline__ void pack_into(const Tile& t, int c, int k, int L, cpx z0, cpx z1, cpx f) {
  if (k == 0) {
    t.s[t.idx(c, 0)] = cmk(z0.x + z1.x, -(z0.x - z1.x));
  } else if (2 * k == L) {
    t.s[t.idx(c, k)] = cmk(2 * z0.x, 2 * z0.y);
  } else {
    cpx ta, tb;
    pack_pair(z0, z1, f, ta, tb);
    t.s[t.idx(c, k)] = cconj(ta);
    t.s[t.idx(c, L - k)] = cconj(tb);
  }
}

// Inverse real DFT input: spectrum X_k, k = 0..L, packed into L complex
// values, staged in shared memory.  Stored conjugated: the inverse DFT is
// computed as conj(DFT(conj(t))).  t2 = w_N^k, k < L/2.
struct LoadC2R {
  static constexpr bool kComplexIn = true;  // whether the raw input elements are complex
  static constexpr bool kStaged = true;
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile& t, cpx (&v)[R]) {
    const cpx* in = static_cast<const cpx*>(p.in) + x.oin;
    const cpx b2 = kind_base<L / R>(p.t2, x.j);
    pair_loop<L, R>(x, [&](int k) { return x.active ? in[int64_t(k) * p.in_n] : czero(); },
                    [&](int i, int k, cpx z0, cpx z1) { pack_into(t, x.c, k, L, z0, z1, rft_root<R>(b2, i)); });
    __syncthreads();
    gather_natural<L, R>(v, x.j, x.c, t);
  }
};

// Split column DFT of a 2-D real DFT with Nr = 4Q rows, inverse half.  The
// CTA's four rows j + Q*m (layout as for StoreR2CQ; input block stride is0,
// element stride in_n) receive the last radix-4 stage of the inverse column
// DFTs from row j of the four blocks V_q left by the length-Q inverse DFTs,
//   X_m = sum_q w_4^(-m*q) (w_Nr^(-j*q) V_q),
// and are packed for their inverse real DFTs as LoadC2R does.  One pass over
// the spectrum pairs (k, L-k) covers all four rows: each thread forms both
// columns of the pair for every row and packs them (one root w_N^k for all
// four).  t1 = w_Nr^n, t2 = w_N^k.
struct LoadC2RQ {
  static constexpr bool kComplexIn = true;  // whether the raw input elements are complex
  static constexpr bool kStaged = true;
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile& t, cpx (&v)[R]) {
    constexpr int NT = 4 * (L / R);  // threads of the CTA (four transforms)
    const cpx* in = static_cast<const cpx*>(p.in) + (x.oin - int64_t(x.c) * p.is0);  // row j of block 0
    const int64_t jr = umod(udiv(x.b, p.d0), p.d1);  // the CTA's row index j
    const cpx w1 = cconj(ldg(p.t1 + jr)), w2 = cconj(ldg(p.t1 + 2 * jr)), w3 = cconj(ldg(p.t1 + 3 * jr));
    const int64_t bs = p.is0;
    // column col of the four blocks -> the four rows' spectra at col
    auto gather4 = [&](int col, cpx (&X)[4]) {
      const cpx* q = in + int64_t(col) * p.in_n;
      const cpx u0 = q[0], u1 = cmul(q[bs], w1), u2 = cmul(q[2 * bs], w2), u3 = cmul(q[3 * bs], w3);
      const cpx a0 = cadd(u0, u2), a1 = csub(u0, u2), c0 = cadd(u1, u3), c1 = csub(u1, u3);
      const cpx ic1 = cmk(-c1.y, c1.x);  // i * c1
      X[0] = cadd(a0, c0);
      X[1] = cadd(a1, ic1);
      X[2] = csub(a0, c0);
      X[3] = csub(a1, ic1);
    };
#pragma unroll
    for (int it = 0; it < (L / 2 + NT) / NT; ++it) {
      const int k = threadIdx.x + it * NT;  // pair (k, L-k), k = 0 .. L/2
      if (k <= L / 2) {
        cpx Xa[4], Xb[4];
        gather4(k, Xa);
        if (2 * k != L) gather4(k == 0 ? L : L - k, Xb);  // X_L pairs with X_0
        const cpx f = (k > 0 && 2 * k < L) ? ldg(p.t2 + k) : cmk(real(1), real(0));
#pragma unroll
        for (int m = 0; m < 4; ++m) pack_into(t, m, k, L, Xa[m], Xb[m], f);
      }
    }
    __syncthreads();
    gather_natural<L, R>(v, x.j, x.c, t);
  }
};

// Type-3 input (reference minfft.c:807-817, 857-867) followed by the
// inverse-real-DFT packing, staged in shared memory (conjugated as above).
// t1 = w_4N^n (n < N/2), t2 = w_N^k (k < L/2); N = 2L.
struct LoadDCT3 {
  static constexpr bool kComplexIn = false;  // whether the raw input elements are complex
  static constexpr bool kStaged = true;
  // z_n of the type-3 pre-rotation; rd(i) returns input real x_i
  template <class Rd>
  static __device__ __forceinline__ cpx zval_r(const Rd& rd, int n, int L, bool dst, const cpx* e) {
    return zval_w(rd, n, L, dst, [&](int m) { return ldg(e + m); });
  }
  // z_n with the root w_4N^n from a function
  template <class Rd, class Rt>
  static __device__ __forceinline__ cpx zval_w(const Rd& rd, int n, int L, bool dst, const Rt& root) {
    const int N = 2 * L;
    if (n == 0) return cmk(dst ? rd(N - 1) : rd(0), real(0));
    if (n == L) {
      const real r2 = real(1.414213562373095048801688724209698079);
      return cmk(r2 * (dst ? rd(L - 1) : rd(L)), real(0));
    }
    const real a = dst ? rd(N - n - 1) : rd(n);
    const real b = dst ? rd(n - 1) : rd(N - n);
    return cconj(cmul(cmk(a, b), root(n)));
  }
  static __device__ __forceinline__ cpx zval(const real* in, int64_t s, int n, int L, bool dst, const cpx* e) {
    return zval_r([&](int i) { return in[int64_t(i) * s]; }, n, L, dst, e);
  }
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile& t, cpx (&v)[R]) {
    const real* in = static_cast<const real*>(p.in) + x.oin;
    const bool dst = (p.flags & F_DST) != 0;
    if constexpr (L >= 2) {
      if (rows_staged_in(p) || p.colmode) {
        // the row (or column) through shared memory, its loads all issued
        // up front; every thread reads its pairs before any packed value
        // overwrites the row
        constexpr int TPT = L / R;
        const cpx b1 = kind_base<TPT>(p.t1, x.j), b2 = kind_base<TPT>(p.t2, x.j);
        real* sr = tile_row(t, x.c);
        if (x.active) {
          if (p.colmode)
            col_g2s<L, R>(sr, in, p.in_n, x.j, (p.flags & F_SRC_SMEM) != 0);
          else
            row_g2s<L, R>(sr, in, x.j, (p.flags & F_SRC_SMEM) != 0);
        }
        __syncthreads();
        constexpr int NP = R / 2 + 1;
        cpx za[NP], zb[NP];
        auto rd = [&](int m) { return sr[m]; };
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          const int k = x.j + i * TPT;
          const bool own = x.active && (i < R / 2 || x.j == 0);
          const cpx rk = t23_root<R>(b1, i);  // w_4N^k
          za[i] = own ? zval_w(rd, k, L, dst, [&](int) { return rk; }) : czero();
          zb[i] = own ? zval_w(rd, L - k, L, dst, [&](int) { return t23_mirror(rk); }) : czero();
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < NP; ++i)
          if (i < R / 2 || x.j == 0) pack_into(t, x.c, x.j + i * TPT, L, za[i], zb[i], rft_root<R>(b2, i));
        __syncthreads();
        gather_natural<L, R>(v, x.j, x.c, t);
        return;
      }
    }
    // the pairs (k, L-k) of pair_loop, read straight from global memory
    constexpr int TPT = L / R;
    const cpx b1 = kind_base<TPT>(p.t1, x.j), b2 = kind_base<TPT>(p.t2, x.j);
    auto rd = [&](int m) { return in[int64_t(m) * p.in_n]; };
#pragma unroll
    for (int i = 0; i <= R / 2; ++i) {
      const int k = x.j + i * TPT;
      if (i == R / 2 && x.j != 0) break;
      const cpx rk = t23_root<R>(b1, i);  // w_4N^k
      const cpx z0 = x.active ? zval_w(rd, k, L, dst, [&](int) { return rk; }) : czero();
      const cpx z1 = x.active ? zval_w(rd, L - k, L, dst, [&](int) { return t23_mirror(rk); }) : czero();
      pack_into(t, x.c, k, L, z0, z1, rft_root<R>(b2, i));
    }
    __syncthreads();
    gather_natural<L, R>(v, x.j, x.c, t);
  }
};

// Type-4 pre-rotation fused into the first pass of a Stockham chain over
// HBM along a 1-D line (reference minfft.c:906-910, 953-957).  Element n of
// sub-DFT b (b1 = its index in the line, b2 = the line) is the line's
// complex point g = b1 + n*in_n: t_g = w_2N^g (x[2g] + i x[N-1-2g]) for
// DCT-4, -w_2N^g (x[2g] - i x[N-1-2g]) for DST-4, x the line's N = kn reals
// at b2 * k_in_line.  w_2N^g is the product of the coarse and fine roots
// (st_hi, st_lo, st_lobits) of 2N: the first pass has no pre-twiddle of its
// own.  The CTA holds mirror pairs of sub-DFTs (MirrorPairs below): point
// g's mirror Lt-1-g (Lt = N/2) is element L-1-n of the partner sub-DFT, and
// x[2g+1] = x[N-1-2(Lt-1-g)].  So each element reads the real pair
// (x[2g], x[2g+1]) as one vector, keeps x[2g] and hands x[2g+1] to its
// mirror element's thread through the tile: every real is read once, in
// whole sectors.
struct LoadT4Chain {
  static constexpr bool kComplexIn = false;  // whether the raw input elements are complex
  static constexpr bool kStaged = false;
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile& t, cpx (&v)[R]) {
    constexpr int TPT = L / R;
    const int64_t rest = udiv(x.b, p.d0);
    const int64_t b2 = udiv(rest, p.d1), b1 = rest - b2 * p.d1;
    const real* in = static_cast<const real*>(p.in) + b2 * p.k_in_line;
    const bool dst = (p.flags & F_DST) != 0;
    const int h = p.cpb / 2;
    const int pc = x.c < h ? x.c + h : x.c - h;  // the mirror sub-DFT's slot
    real* sb = reinterpret_cast<real*>(t.s);
    const bool vec = (reinterpret_cast<uintptr_t>(in) % sizeof(cpx)) == 0;
    real a[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int n = x.j + r * TPT;
      const int64_t g = b1 * p.is1 + int64_t(n) * p.in_n;
      real lo, hi;
      if (vec) {
        const cpx q = __ldcs(reinterpret_cast<const cpx*>(in + 2 * g));
        lo = q.x;
        hi = q.y;
      } else {
        lo = __ldcs(in + 2 * g);
        hi = __ldcs(in + 2 * g + 1);
      }
      a[r] = lo;
      sb[pc * 2 * t.lp + (L - 1 - n)] = hi;
    }
    __syncthreads();
    // w_2N^g for g = g0 + r*TPT*in_n
    const RootProgression<R> ew(p.st_hi, p.st_lo, p.st_lobits, uint32_t(b1 * p.is1 + int64_t(x.j) * p.in_n),
                                uint32_t(int64_t(TPT) * p.in_n));
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int n = x.j + r * TPT;
      const real b = sb[x.c * 2 * t.lp + n];
      const cpx e = ew.at(r);
      if (!dst) {
        v[r] = cmul(e, cmk(a[r], b));
      } else {
        const cpx q = cmul(e, cmk(a[r], -b));
        v[r] = cmk(-q.x, -q.y);
      }
    }
  }
};

// --------------------------------------------------------------- store ops
// Each store op receives output element k = j + r*(L/R) of the length-L DFT
// in v[r].

// Offsets of the CTA's transforms, kept in shared memory so staged stores
// can address any transform of the tile.
struct TileOffsets {
  int64_t* in_off;
  int64_t* out_off;
  int nvalid;  // transforms of the tile that exist (the rest are padding)
};

struct StoreCplx {
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile& t, const TileOffsets& to,
                                             cpx (&v)[R]) {
    cpx* out = static_cast<cpx*>(p.out);
    const bool cj = (p.flags & F_CONJ_OUT) != 0;
    if (!(p.flags & F_STAGE_ROWS)) {
      if (!x.active) return;
      constexpr int TPT = L / R;
      if (cj) {
#pragma unroll
        for (int r = 0; r < R; ++r) v[r].y = -v[r].y;
      }
      if (p.out_k == 1) {
        cpx* q = out + x.oout + x.j;
#pragma unroll
        for (int r = 0; r < R; ++r) q[r * TPT] = v[r];
      } else {
        cpx* q = out + x.oout + x.j * p.out_k;
        const int64_t st = int64_t(TPT) * p.out_k;
#pragma unroll
        for (int r = 0; r < R; ++r) q[r * st] = v[r];
      }
      return;
    }
    // staged: each transform's L outputs written with k running fastest
    __syncthreads();
    scatter_natural<L, R>(v, x.j, x.c, t);
    __syncthreads();
    const int total = to.nvalid * L;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int c = e / L, k = e - c * L;
      cpx o = t.s[t.idx(c, k)];
      if (cj) o.y = -o.y;
      out[to.out_off[c] + int64_t(k) * p.out_k] = o;
    }
  }
};

// Real DFT output (reference minfft.c:547-578): L+1 complex values from the
// half-length DFT, via the pair unpacking; t1 = w_N^k, k < L/2.
struct StoreR2C {
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile& t, const TileOffsets&,
                                             cpx (&v)[R]) {
    __syncthreads();
    scatter_natural<L, R>(v, x.j, x.c, t);
    __syncthreads();
    if (!x.active) return;
    cpx* out = static_cast<cpx*>(p.out) + x.oout;
    const cpx b1 = kind_base<L / R>(p.t1, x.j);
    pair_loop<L, R>(x, [&](int k) { return t.s[t.idx(x.c, k & (L - 1))]; }, [&](int i, int k, cpx za, cpx zb) {
      if (k == 0) {
        out[0] = cmk(za.x + za.y, real(0));
        out[int64_t(L) * p.out_k] = cmk(za.x - za.y, real(0));
      } else if (2 * k == L) {
        out[int64_t(k) * p.out_k] = cconj(za);
      } else {
        cpx xa, xb;
        unpack_pair(za, zb, rft_root<R>(b1, i), xa, xb);
        out[int64_t(k) * p.out_k] = xa;
        out[int64_t(L - k) * p.out_k] = xb;
      }
    });
  }
};

// Type-2 output (reference minfft.c:714-725, 763-774): real-DFT unpacking,
// then y_n = 2 Re(V_n e_n), y_{N-n} = -2 Im(V_n e_n) (DCT-2; DST-2 maps the
// same values to reversed positions).  t1 = w_4N^n (n < N/2), t2 = w_N^k.
struct StoreDCT2 {
  static __device__ __forceinline__ void emit(real* out, int64_t s, int n, int N, bool dst, cpx V, cpx e) {
    const cpx q = cmul(V, e);
    if (!dst) {
      out[int64_t(n) * s] = 2 * q.x;
      out[int64_t(N - n) * s] = -2 * q.y;
    } else {
      out[int64_t(n - 1) * s] = -2 * q.y;
      out[int64_t(N - n - 1) * s] = 2 * q.x;
    }
  }
  // emit() for V2 = 2V (from unpack_pair2)
  static __device__ __forceinline__ void emit2(real* out, int64_t s, int n, int N, bool dst, cpx V2, cpx e) {
    const cpx q = cmul(V2, e);
    if (!dst) {
      out[int64_t(n) * s] = q.x;
      out[int64_t(N - n) * s] = -q.y;
    } else {
      out[int64_t(n - 1) * s] = -q.y;
      out[int64_t(N - n - 1) * s] = q.x;
    }
  }
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile& t, const TileOffsets&,
                                             cpx (&v)[R]) {
    __syncthreads();
    scatter_natural<L, R>(v, x.j, x.c, t);
    __syncthreads();
    if (!x.active) return;
    real* out = static_cast<real*>(p.out) + x.oout;
    const bool dst = (p.flags & F_DST) != 0;
    constexpr int N = 2 * L;
    const real r2 = real(1.414213562373095048801688724209698079);
    const cpx b1 = kind_base<L / R>(p.t1, x.j), b2 = kind_base<L / R>(p.t2, x.j);
    pair_loop<L, R>(x, [&](int k) { return t.s[t.idx(x.c, k & (L - 1))]; }, [&](int i, int k, cpx za, cpx zb) {
      if (k == 0) {
        const real v0 = za.x + za.y, vl = za.x - za.y;
        out[int64_t(dst ? N - 1 : 0) * p.out_k] = 2 * v0;
        out[int64_t(dst ? L - 1 : L) * p.out_k] = r2 * vl;
      } else if (2 * k == L) {
        emit(out, p.out_k, k, N, dst, cconj(za), w128(8));  // w_4N^(L/2) = w_16
      } else {
        cpx xa2, xb2;
        unpack_pair2(za, zb, rft_root<R>(b2, i), xa2, xb2);
        const cpx e = t23_root<R>(b1, i);  // w_4N^k
        emit2(out, p.out_k, k, N, dst, xa2, e);
        emit2(out, p.out_k, L - k, N, dst, xb2, t23_mirror(e));
      }
    });
  }
};

// Inverse real DFT output: the inverse half-length DFT (conjugate of the
// forward result) read as interleaved reals (reference minfft.c:605,658).
// Split column DFT of a 2-D real DFT with Nr = 4Q rows, forward half.  The
// CTA holds the four rows j + Q*m (transform c = m: batch layout d0 = 4 with
// is0 = Q rows, d1 = Q with is1 = one row, cpb = 4).  After their half-length
// DFTs it applies, column by column, the first radix-4 stage of the length-Nr
// column DFTs across the four rows' spectra X_m,
//   Z_q[j] = w_Nr^(j*q) * sum_m X_m w_4^(m*q),
// and writes Z_q to row j of block q of the output (block stride os0, element
// stride out_k); length-Q DFTs of each block then finish the column DFTs
// (their output p is row q + 4p).  One pass over the spectrum pairs (k, L-k)
// covers all four rows: each thread unpacks the pair for every row (one root
// w_N^k for all four) and stores both columns.  t1 = w_N^k (real-DFT table),
// t2 = w_Nr^n.
struct StoreR2CQ {
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile& t, const TileOffsets& to,
                                             cpx (&v)[R]) {
    constexpr int NT = 4 * (L / R);  // threads of the CTA (four transforms)
    __syncthreads();
    scatter_natural<L, R>(v, x.j, x.c, t);
    __syncthreads();
    const int64_t jr = umod(udiv(x.b, p.d0), p.d1);  // the CTA's row index j
    const cpx w1 = ldg(p.t2 + jr), w2 = ldg(p.t2 + 2 * jr), w3 = ldg(p.t2 + 3 * jr);
    cpx* out = static_cast<cpx*>(p.out) + to.out_off[0];  // row j of block 0
    const int64_t bs = p.os0;
    // column col of the four rows -> blocks 0..3
    auto emit = [&](int col, const cpx (&X)[4]) {
      const cpx a0 = cadd(X[0], X[2]), a1 = csub(X[0], X[2]), c0 = cadd(X[1], X[3]), c1 = csub(X[1], X[3]);
      const cpx mic1 = cmk(c1.y, -c1.x);  // -i * c1
      cpx* q = out + int64_t(col) * p.out_k;
      q[0] = cadd(a0, c0);
      q[bs] = cmul(cadd(a1, mic1), w1);
      q[2 * bs] = cmul(csub(a0, c0), w2);
      q[3 * bs] = cmul(csub(a1, mic1), w3);
    };
#pragma unroll
    for (int it = 0; it < (L / 2 + NT) / NT; ++it) {
      const int k = threadIdx.x + it * NT;  // pair (k, L-k), k = 0 .. L/2
      if (k <= L / 2) {
        cpx Xa[4], Xb[4];
        if (k == 0) {
#pragma unroll
          for (int m = 0; m < 4; ++m) {
            const cpx z = t.s[t.idx(m, 0)];
            Xa[m] = cmk(z.x + z.y, real(0));
            Xb[m] = cmk(z.x - z.y, real(0));  // X_L
          }
          emit(0, Xa);
          emit(L, Xb);
        } else if (2 * k == L) {
#pragma unroll
          for (int m = 0; m < 4; ++m) Xa[m] = cconj(t.s[t.idx(m, k)]);
          emit(k, Xa);
        } else {
          const cpx f = ldg(p.t1 + k);
#pragma unroll
          for (int m = 0; m < 4; ++m) unpack_pair(t.s[t.idx(m, k)], t.s[t.idx(m, L - k)], f, Xa[m], Xb[m]);
          emit(k, Xa);
          emit(L - k, Xb);
        }
      }
    }
  }
};

struct StoreC2R {
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile&, const TileOffsets&,
                                             cpx (&v)[R]) {
    if (!x.active) return;
    constexpr int TPT = L / R;
    real* out = static_cast<real*>(p.out) + x.oout;
    if (p.flags & F_VEC) {
      cpx* q = reinterpret_cast<cpx*>(out) + x.j;
#pragma unroll
      for (int r = 0; r < R; ++r) q[r * TPT] = cconj(v[r]);
    } else {
      real* q = out + 2 * x.j;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        q[2 * r * TPT] = v[r].x;
        q[2 * r * TPT + 1] = -v[r].y;
      }
    }
  }
};

// Type-3 output (reference minfft.c:821-824, 871-874): the inverse real
// DFT's reals t_i go to y[2i] (i < N/2) and y[2N-1-2i] (i >= N/2, negated
// for DST-3).
struct StoreDCT3 {
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile& t, const TileOffsets&,
                                             cpx (&v)[R]) {
    real* out = static_cast<real*>(p.out) + x.oout;
    real* gout = out;
    int64_t s = p.out_k;
    bool staged = false;
    if constexpr (L >= 2) {
      if (rows_staged_out(p)) {  // the outputs into the row's shared-memory slot, then the row out whole
        __syncthreads();
        out = tile_row(t, x.c);
        s = 1;
        staged = true;
      }
    }
    const bool dst = (p.flags & F_DST) != 0;
    constexpr int N = 2 * L;
    constexpr int TPT = L / R;
    if constexpr (L >= 2) {
      // reals t_2m, t_2m+1 (m = j + r*TPT) go to y[4m], y[4m+2] while r < R/2,
      // else to y[2N-1-4m], y[2N-3-4m] (negated for DST-3)
      const real sg = dst ? real(-1) : real(1);
      if (x.active) {
        real* lo = out + int64_t(4 * x.j) * s;
        real* hi = out + int64_t(2 * N - 1 - 4 * x.j) * s;
        const int64_t st = int64_t(4 * TPT) * s;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const cpx w = cconj(v[r]);
          if (r < R / 2) {
            lo[r * st] = w.x;
            lo[r * st + 2 * s] = w.y;
          } else {
            hi[-r * st] = sg * w.x;
            hi[-r * st - 2 * s] = sg * w.y;
          }
        }
      }
      if (staged) {
        __syncthreads();
        if (x.active) row_s2g<L, R>(gout, out, x.j);
      }
    } else {  // L = 1: y0 = t0, y1 = +-t1
      if (!x.active) return;
      const cpx w = cconj(v[0]);
      out[0] = w.x;
      out[p.out_k] = dst ? -w.y : w.y;
    }
  }
};

// Type-4 post-rotation (reference minfft.c:916-921, 963-968): T_m feeds
// y[2m] = 2 Re(g_2m T_m) and y[N-1-2m] = 2 Re(g_{N-1-2m} conj(T_m)) (Im for
// DST-4), g_q = w_8N^(2q+1) from table t2.
struct StoreT4 {
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile&, const TileOffsets&,
                                             cpx (&v)[R]) {
    if (!x.active) return;
    real* out = static_cast<real*>(p.out) + x.oout;
    const bool dst = (p.flags & F_DST) != 0;
    constexpr int N = 2 * L;
    constexpr int TPT = L / R;
    const int64_t s = p.out_k;
    real* lo = out + int64_t(2 * x.j) * s;
    real* hi = out + int64_t(N - 1 - 2 * x.j) * s;
    const int64_t st = int64_t(2 * TPT) * s;
    // t2[q] = w_8N^(2q+1): t2[2m] = t2[2j] * w_4R^r and t2[N-1-2m] =
    // t2[N-1-2j] * conj(w_4R^r) for m = j + r*TPT
    const cpx glo = ldg(p.t2 + 2 * x.j);
    const cpx ghi = ldg(p.t2 + (N - 1 - 2 * x.j));
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const cpx T = v[r];
      const cpx a = cmul(cmul(glo, w128(r * (32 / R))), T);
      const cpx b = cmul(cmulc(ghi, w128(r * (32 / R))), cconj(T));
      lo[r * st] = 2 * (dst ? a.y : a.x);
      hi[-r * st] = 2 * (dst ? b.y : b.x);
    }
  }
};

// Type-4 post-rotation fused into the last pass of a Stockham chain over
// HBM along a 1-D line (reference minfft.c:916-921, 963-968): output k of
// sub-DFT b is the line's point m = (its normal offset) + k*out_k, and
// T_m gives y[2m] = 2 Re(g_2m T_m), y[N-1-2m] = 2 Re(g_{N-1-2m} conj(T_m))
// (Im for DST-4), g_q = w_8N^(2q+1) as the product of the coarse and fine
// roots t1, t2 of 8N (kbits fine bits), and g_{N-1-2m} = -i conj(g_2m); y is
// the line's N reals at b2 * k_out_line (the pass's os2 is 0).  As in
// LoadT4Chain the CTA holds mirror pairs of sub-DFTs: y[2m+1] is
// y[N-1-2m'] of the mirror point m' = Lt-1-m (output L-1-k of the partner
// sub-DFT), so each element hands that value to its mirror's thread through
// the tile and writes the pair (y[2m], y[2m+1]) as one vector.
struct StoreT4Chain {
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile& t, const TileOffsets&,
                                             cpx (&v)[R]) {
    constexpr int TPT = L / R;
    const int64_t b2 = udiv(x.b, p.d0 * p.d1);
    real* out = static_cast<real*>(p.out) + b2 * p.k_out_line;
    const bool dst = (p.flags & F_DST) != 0;
    const int h = p.cpb / 2;
    const int pc = x.c < h ? x.c + h : x.c - h;  // the mirror sub-DFT's slot
    real* sb = reinterpret_cast<real*>(t.s);
    const bool vec = (reinterpret_cast<uintptr_t>(out) % sizeof(cpx)) == 0;
    // g_2m = w_8N^(4m+1) for m = m0 + r*TPT*out_k
    const RootProgression<R> gw(p.t1, p.t2, p.kbits, uint32_t(4 * (x.oout + int64_t(x.j) * p.out_k) + 1),
                                uint32_t(4 * int64_t(TPT) * p.out_k));
    __syncthreads();  // the last Stockham exchange has finished with the tile
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int k = x.j + r * TPT;
      const cpx ga = gw.at(r);
      const cpx gb = cmk(-ga.y, -ga.x);  // -i conj(ga) = w_8N^(2N-1-4m)
      const cpx T = v[r];
      const cpx A = cmul(ga, T);
      const cpx B = cmul(gb, cconj(T));
      // a slot holds 2*lp >= 2L reals: the mirror's values below L, its own above
      sb[x.c * 2 * t.lp + L + k] = 2 * (dst ? A.y : A.x);
      sb[pc * 2 * t.lp + (L - 1 - k)] = 2 * (dst ? B.y : B.x);
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int k = x.j + r * TPT;
      const int64_t m = x.oout + int64_t(k) * p.out_k;
      const real own = sb[x.c * 2 * t.lp + L + k];
      const real part = sb[x.c * 2 * t.lp + k];
      if (vec) {
        __stcs(reinterpret_cast<cpx*>(out + 2 * m), cmk(own, part));
      } else {
        __stcs(out + 2 * m, own);
        __stcs(out + 2 * m + 1, part);
      }
    }
  }
};

// Element-wise steps of a long real transform fused into the first or last
// pass of a Stockham chain whose sub-DFTs hold single points of the
// half-length sequence (one line, no mirror pairing; the mixed batch's long
// items).  Point g of sub-DFT b is b1 + n*in_n (first pass, b1 = b % d1),
// point m of the output is the sub-DFT's normal offset + k*out_k (last
// pass); N = kn reals in the line.

// Type-2 permutation (Op_dct2_pre): t_g = (u_2g, u_2g+1), u_i = x[2i] for
// i < N/2, else sg * x[2N-1-2i].
struct LoadDCT2Chain {
  static constexpr bool kComplexIn = false;  // whether the raw input elements are complex
  static constexpr bool kStaged = false;
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile&, cpx (&v)[R]) {
    constexpr int TPT = L / R;
    const real* in = static_cast<const real*>(p.in);
    const int64_t N = p.kn, H = N / 2;
    const real sg = (p.flags & F_DST) ? real(-1) : real(1);
    const int64_t b1 = umod(x.b, p.d1);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t g = b1 + int64_t(x.j + r * TPT) * p.in_n;
      const int64_t i0 = 2 * g, i1 = 2 * g + 1;
      v[r] = cmk(i0 < H ? in[2 * i0] : sg * in[2 * N - 1 - 2 * i0], i1 < H ? in[2 * i1] : sg * in[2 * N - 1 - 2 * i1]);
    }
  }
};

// Type-4 pre-rotation (Op_t4_pre) with a direct root table t1 = w_2N^g.
struct LoadT4Direct {
  static constexpr bool kComplexIn = false;  // whether the raw input elements are complex
  static constexpr bool kStaged = false;
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile&, cpx (&v)[R]) {
    constexpr int TPT = L / R;
    const real* in = static_cast<const real*>(p.in);
    const int64_t N = p.kn;
    const bool dst = (p.flags & F_DST) != 0;
    const int64_t b1 = umod(x.b, p.d1);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t g = b1 + int64_t(x.j + r * TPT) * p.in_n;
      const real a = in[2 * g], b = in[N - 1 - 2 * g];
      const cpx w = ldg(p.t1 + g);
      if (!dst) {
        v[r] = cmul(w, cmk(a, b));
      } else {
        const cpx q = cmul(w, cmk(a, -b));
        v[r] = cmk(-q.x, -q.y);
      }
    }
  }
};

// Type-3 de-interleave (Op_dct3_post) of point m of the forward result.
struct StoreDCT3Chain {
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile&, const TileOffsets&,
                                             cpx (&v)[R]) {
    if (!x.active) return;
    constexpr int TPT = L / R;
    real* out = static_cast<real*>(p.out);
    const int64_t N = p.kn, H = N / 2;
    const bool dst = (p.flags & F_DST) != 0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t m = x.oout + int64_t(x.j + r * TPT) * p.out_k;
      const cpx w = cconj(v[r]);
      const int64_t i0 = 2 * m, i1 = 2 * m + 1;
      out[i0 < H ? 2 * i0 : 2 * N - 1 - 2 * i0] = (dst && i0 >= H) ? -w.x : w.x;
      out[i1 < H ? 2 * i1 : 2 * N - 1 - 2 * i1] = (dst && i1 >= H) ? -w.y : w.y;
    }
  }
};

// Type-4 post-rotation (Op_t4_post) with a direct root table t2 = w_8N^(2q+1).
struct StoreT4Direct {
  template <int L, int R>
  static __device__ __forceinline__ void run(const AxisParams& p, const Ctx& x, const Tile&, const TileOffsets&,
                                             cpx (&v)[R]) {
    if (!x.active) return;
    constexpr int TPT = L / R;
    real* out = static_cast<real*>(p.out);
    const int64_t N = p.kn;
    const bool dst = (p.flags & F_DST) != 0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t m = x.oout + int64_t(x.j + r * TPT) * p.out_k;
      const cpx T = v[r];
      const cpx a = cmul(ldg(p.t2 + 2 * m), T);
      const cpx b = cmul(ldg(p.t2 + (N - 1 - 2 * m)), cconj(T));
      out[2 * m] = 2 * (dst ? a.y : a.x);
      out[N - 1 - 2 * m] = 2 * (dst ? b.y : b.x);
    }
  }
};

// The fused type-4 passes take mirror pairs of sub-DFTs into one CTA: with
// M = d0*d1 sub-DFTs per line, slots c < cpb/2 hold sub-DFTs i of the line
// and slots c + cpb/2 their mirrors M-1-i (the planner makes cpb even and a
// divisor of M).
template <class Op>
struct MirrorPairs {
  static constexpr bool value = false;
};
template <>
struct MirrorPairs<LoadT4Chain> {
  static constexpr bool value = true;
};
template <>
struct MirrorPairs<StoreT4Chain> {
  static constexpr bool value = true;
};

// Batch index of the CTA's transform in slot c.
template <bool kMirror>
__device__ __forceinline__ int64_t tile_batch(const AxisParams& p, int c) {
  if constexpr (kMirror) {
    const int64_t M = p.d0 * p.d1;
    const int64_t per_line = udiv(M, p.cpb);  // CTAs per line
    const int64_t line = udiv(int64_t(blockIdx.x), per_line), q = int64_t(blockIdx.x) - line * per_line;
    const int h = p.cpb / 2;
    const int64_t i = q * h + (c < h ? c : c - h);
    return line * M + (c < h ? i : M - 1 - i);
  } else {
    return int64_t(blockIdx.x) * p.cpb + c;
  }
}

// ------------------------------------------------------------------ kernel
// Register budget per thread: a radix-R thread holds R complex values; with
// 512-thread CTAs, 16 doubles-complex get 128 registers (1 CTA per SM), and
// every halving of the state doubles the CTAs the budget allows.
template <int R>
struct MinBlocks {
  // double: 128 registers at radix 16, 64 at radix 8 (and below);
  // single: 64 at radix 16, 40 at radix 8, 64 below
  static constexpr int value = sizeof(real) == 8 ? (R >= 16 ? 1 : 2) : (R >= 16 ? 2 : R == 8 ? 3 : 2);
};

template <int L, int R, class LoadOp, class StoreOp>
__global__ void __launch_bounds__(512, MinBlocks<R>::value) axis_pass_kernel(const AxisParams p) {
  static_assert(R <= L || L < 2, "radix at most the length");
  constexpr int TPT = L / R;
  pdl_release();
  pdl_wait();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int64_t* offs = reinterpret_cast<int64_t*>(smem_raw);
  const int64_t left = p.nbatch - int64_t(blockIdx.x) * p.cpb;
  TileOffsets to{offs, offs + p.cpb, int(left < p.cpb ? left : p.cpb)};
  Tile t{reinterpret_cast<cpx*>(smem_raw + 16 * ((2 * p.cpb * sizeof(int64_t) + 15) / 16)), p.lp};

  constexpr bool kMirror = MirrorPairs<LoadOp>::value || MirrorPairs<StoreOp>::value;
  // offsets of the CTA's transforms, computed once per transform
  for (int c = threadIdx.x; c < p.cpb; c += blockDim.x) {
    const int64_t b = tile_batch<kMirror>(p, c);
    int64_t b0, oi, oo;
    batch_offsets(p, b < p.nbatch ? b : 0, b0, oi, oo);
    to.in_off[c] = oi;
    to.out_off[c] = oo;
  }
  __syncthreads();

  Ctx x;
  if (p.colmode) {
    x.c = threadIdx.x % p.cpb;
    x.j = threadIdx.x / p.cpb;
  } else {
    x.j = threadIdx.x % TPT;
    x.c = threadIdx.x / TPT;
  }
  x.b = tile_batch<kMirror>(p, x.c);
  x.active = x.b < p.nbatch;
  x.oin = to.in_off[x.c];
  x.oout = to.out_off[x.c];
  x.b0 = umod(x.b, p.d0);

  cpx v[R];
  LoadOp::template run<L, R>(p, x, t, v);
  run_passes<L, R, 1>(v, x.j, x.c, t, p.tw);
  StoreOp::template run<L, R>(p, x, t, to, v);
}

// Number of bytes of dynamic shared memory the kernel needs for cpb transforms.
inline size_t axis_pass_smem(int L, int R, int cpb, int colmode) {
  return 16 * ((2 * cpb * sizeof(int64_t) + 15) / 16) + size_t(cpb) * tile_pitch(L, R, cpb, colmode) * sizeof(cpx);
}

}  // namespace mb
