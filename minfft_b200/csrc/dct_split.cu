// Split column DFT of the 2-D DCT-2 / DST-2 and DCT-3 / DST-3 (Nr rows of N
// reals, Nr = 8Q).  Along a column, the type-2/3 transform reduces to a
// complex DFT of length Lc = Nr/2 = 4Q (reference minfft.c:692-887: the
// half-length real DFT inside DCT-2 / DST-2, its inverse inside DCT-3 /
// DST-3).  That DFT is split as 4 x Q, and its radix-4 stage is fused into
// a pass over the rows, so the column pass only holds Q-point columns:
//
// Forward (type 2).  With u the permuted column (u_i = y[2i], i < Nr/2;
// u_i = +-y[2Nr-1-2i], i >= Nr/2), t_m = u_2m + i u_2m+1 and
//   T[q + 4p] = DFT_Q over j of  Z_q[j],  Z_q[j] = w_Lc^(jq) sum_m' t[j + Q m'] w_4^(m'q).
// The 8 rows that make up t[j + Q m'] (m' = 0..3) are
//   4j + 2a + 4Qm' (m' < 2),  2Nr - 1 - 4j - 4Qm' - 2a (m' >= 2),  a = 0, 1.
// The row pass (dctq_row_fwd) gives one CTA those 8 rows: their row DCT-2s,
// then, column by column, the radix-4 stage, written as the four complex
// blocks Z_q (Q rows of N values each).  The column pass (dctq_col_fwd) runs
// the Q-point DFTs of blocks {0, 2} or {1, 3} for W adjacent columns -- the
// block pairs that hold T_k beside T_(Lc-k) -- and the type-2 unpacking and
// post-rotation of those pairs, writing rows k, Nr-k, Lc-k, Lc+k.
//
// Inverse (type 3).  The column pass (dctq_col_inv) applies the type-3
// pre-rotation and the packing of the inverse real DFT to the pairs
// (k, Lc-k) of its block pair, runs the Q-point DFTs over p of s[q + 4p] and
// writes V_q[j]; the row pass (dctq_row_inv) forms, column by column,
//   S[j + Q m'] = sum_q w_4^(qm') w_Lc^(qj) V_q[j]
// whose conjugates are the column outputs of the same 8 rows, then runs the
// row DCT-3s of those rows.
#include "axis_pass.cuh"
#include "dct_split.h"

namespace mb {

namespace {

// Row of slot c (0..7) of the CTA for column index j: slot c = 2m' + a.
__device__ __forceinline__ int64_t dctq_row(const DctqParams& q, int64_t j, int c) {
  const int m = c >> 1, a = c & 1;
  return m < 2 ? 4 * j + 2 * a + 4 * q.Q * m : 2 * q.Nr - 1 - 4 * j - 4 * q.Q * m - 2 * a;
}

// Axis parameters of a row transform (row mode, contiguous) for the kind's
// load and store stages.
__device__ __forceinline__ AxisParams dctq_row_params(const DctqParams& q, int lp) {
  AxisParams p;
  memset(&p, 0, sizeof(p));
  p.in = q.in;
  p.out = q.out;
  p.nbatch = 1;
  p.d0 = p.d1 = 1;
  p.in_n = 1;
  p.out_k = 1;
  p.tw = q.tw_row;
  p.st_ns = 1;
  p.st_div = 1;
  p.cpb = 8;
  p.lp = lp;
  p.flags = q.flags;
  return p;
}

}  // namespace

// ------------------------------------------------------------------ forward
// Row pass: CTA (h, j) = blockIdx.x (j fastest); 8 rows x L/R threads.
template <int L, int R>
__global__ void __launch_bounds__(8 * (L / R), 1) dctq_row_fwd(const DctqParams q) {
  constexpr int TPT = L / R;
  constexpr int NT = 8 * TPT;
  constexpr int N = 2 * L;
  pdl_release();
  pdl_wait();
  extern __shared__ __align__(16) unsigned char smem[];
  const int tid = threadIdx.x;
  const int c = tid / TPT, jt = tid % TPT;
  const int64_t j = blockIdx.x % q.Q, h = blockIdx.x / q.Q;
  Tile t{reinterpret_cast<cpx*>(smem), q.lp};
  AxisParams p = dctq_row_params(q, q.lp);
  p.t1 = q.t23_row;
  p.t2 = q.rft_row;
  p.in = static_cast<const real*>(q.in) + h * q.Nr * N;
  Ctx x;
  x.c = c;
  x.j = jt;
  x.b = 0;
  x.b0 = 0;
  x.active = true;
  x.oin = dctq_row(q, j, c) * N;
  x.oout = 0;
  cpx v[R];
  LoadDCT2::run<L, R>(p, x, t, v);
  run_passes<L, R, 1>(v, jt, c, t, q.tw_row);
  __syncthreads();
  scatter_natural<L, R>(v, jt, c, t);
  __syncthreads();
  // the pairs (k, L-k) of this thread's row into registers ...
  constexpr int NP = R / 2 + 1;
  cpx za[NP], zb[NP];
#pragma unroll
  for (int i = 0; i < NP; ++i) {
    const int k = jt + i * TPT;
    const bool own = i < R / 2 || jt == 0;
    za[i] = own ? t.s[t.idx(c, k & (L - 1))] : czero();
    zb[i] = own ? t.s[t.idx(c, (L - k) & (L - 1))] : czero();
  }
  __syncthreads();
  // ... then the row's DCT-2 outputs into the staging rows (reals, row c at c*N)
  real* st = reinterpret_cast<real*>(smem) + c * N;
  const bool dst = (q.flags & F_DST) != 0;
  {
    const cpx b1 = kind_base<TPT>(q.t23_row, jt), b2 = kind_base<TPT>(q.rft_row, jt);
    const real r2 = real(1.414213562373095048801688724209698079);
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      const int k = jt + i * TPT;
      if (i == R / 2 && jt != 0) break;
      if (k == 0) {
        const real v0 = za[i].x + za[i].y, vl = za[i].x - za[i].y;
        st[dst ? N - 1 : 0] = 2 * v0;
        st[dst ? L - 1 : L] = r2 * vl;
      } else if (2 * k == L) {
        StoreDCT2::emit(st, 1, k, N, dst, cconj(za[i]), w128(8));
      } else {
        cpx xa, xb;
        unpack_pair2(za[i], zb[i], rft_root<R>(b2, i), xa, xb);
        const cpx e = t23_root<R>(b1, i);
        StoreDCT2::emit2(st, 1, k, N, dst, xa, e);
        StoreDCT2::emit2(st, 1, L - k, N, dst, xb, t23_mirror(e));
      }
    }
  }
  __syncthreads();
  // the column radix-4 stage across the 8 rows, column by column
  const real* s0 = reinterpret_cast<const real*>(smem);
  const real sg = dst ? real(-1) : real(1);
  const cpx w1 = ldg(q.tw_c + j), w2 = ldg(q.tw_c + 2 * j), w3 = ldg(q.tw_c + 3 * j);
  cpx* mid = q.mid + (h * 4 * q.Q + j) * N;
  const int64_t bs = q.Q * N;  // block stride
  for (int n = tid; n < N; n += NT) {
    const cpx t0 = cmk(s0[0 * N + n], s0[1 * N + n]);
    const cpx t1 = cmk(s0[2 * N + n], s0[3 * N + n]);
    const cpx t2 = cmk(sg * s0[4 * N + n], sg * s0[5 * N + n]);
    const cpx t3 = cmk(sg * s0[6 * N + n], sg * s0[7 * N + n]);
    const cpx a0 = cadd(t0, t2), a1 = csub(t0, t2), c0 = cadd(t1, t3), c1 = csub(t1, t3);
    const cpx mic1 = cmk(c1.y, -c1.x);  // -i * c1
    mid[n] = cadd(a0, c0);
    mid[bs + n] = cmul(cadd(a1, mic1), w1);
    mid[2 * bs + n] = cmul(csub(a0, c0), w2);
    mid[3 * bs + n] = cmul(csub(a1, mic1), w3);
  }
}

// Column pass: CTA = (h, block pair P, W adjacent columns); transforms
// c = slot*W + col (slot 0: block P, slot 1: block P + 2), Q points each.
template <int QL, int R>
__global__ void __launch_bounds__(512, 1) dctq_col_fwd(const DctqParams q) {
  constexpr int TPT = QL / R;
  pdl_release();
  pdl_wait();
  extern __shared__ __align__(16) unsigned char smem[];
  const int W = q.W, cpb = 2 * W;
  const int tid = threadIdx.x;
  const int c = tid % cpb, jt = tid / cpb;
  const int slot = c / W, col = c % W;
  const int64_t N = q.N, Nr = q.Nr, Lc = 4 * int64_t(QL);
  const int64_t gpr = N / W;  // column groups per row
  const int64_t g = blockIdx.x % gpr, rest = blockIdx.x / gpr;
  const int P = int(rest % 2);
  const int64_t h = rest / 2;
  const int64_t n0 = g * W;
  const int blk = P + 2 * slot;
  Tile t{reinterpret_cast<cpx*>(smem), q.lp};
  // the Q-point DFT over j of Z_blk[j] at column n0 + col
  const cpx* src = q.mid + ((h * 4 + blk) * QL) * N + n0 + col;
  cpx v[R];
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = src[int64_t(jt + r * TPT) * N];
  run_passes<QL, R, 1>(v, jt, c, t, q.tw_q);
  __syncthreads();
  scatter_natural<QL, R>(v, jt, c, t);  // T[blk + 4p] at (c, p)
  __syncthreads();
  // type-2 unpacking and post-rotation of the pairs (k, Lc-k) the pair
  // holds: P = 1: k = 1 + 4p (partner 3 + 4(Q-1-p)); P = 0: k = 4p for
  // p <= Q/2 (partner 4(Q-p)) and k = 2 + 4p for p < Q/2 (partner 2 + 4(Q-1-p))
  real* out = static_cast<real*>(q.out) + h * Nr * N + n0;
  const bool dst = (q.flags & F_DST) != 0;
  const real r2 = real(1.414213562373095048801688724209698079);
  const int npairs = P == 1 ? QL : QL + 1;
  for (int e = tid; e < npairs * W; e += blockDim.x) {
    const int cc = e % W, pi = e / W;
    int64_t k;
    cpx za, zb;
    if (P == 1) {
      // the pair (k, Lc-k) with k = 1 + 4p in block 1 and Lc-k in block 3,
      // taken from its smaller member (the root table holds w_Nr^k for k < Lc/2)
      k = 1 + 4 * int64_t(pi);
      za = t.s[t.idx(cc, pi)];
      zb = t.s[t.idx(W + cc, QL - 1 - pi)];
      if (2 * k > Lc) {
        const cpx tmp = za;
        za = zb;
        zb = tmp;
        k = Lc - k;
      }
    } else if (pi <= QL / 2) {
      k = 4 * int64_t(pi);
      za = t.s[t.idx(cc, pi)];
      zb = t.s[t.idx(cc, (QL - pi) & (QL - 1))];
    } else {
      const int p2 = pi - QL / 2 - 1;  // 0 .. Q/2-1
      k = 2 + 4 * int64_t(p2);
      za = t.s[t.idx(W + cc, p2)];
      zb = t.s[t.idx(W + cc, QL - 1 - p2)];
    }
    real* o = out + cc;
    if (k == 0) {
      o[(dst ? Nr - 1 : 0) * N] = 2 * (za.x + za.y);
      o[(dst ? Lc - 1 : Lc) * N] = r2 * (za.x - za.y);
    } else if (2 * k == Lc) {
      StoreDCT2::emit(o, N, int(k), int(Nr), dst, cconj(za), ldg(q.t23_c + k));
    } else {
      cpx xa, xb;
      unpack_pair2(za, zb, ldg(q.rft_c + k), xa, xb);
      StoreDCT2::emit2(o, N, int(k), int(Nr), dst, xa, ldg(q.t23_c + k));
      StoreDCT2::emit2(o, N, int(Lc - k), int(Nr), dst, xb, ldg(q.t23_c + (Lc - k)));
    }
  }
}

// ------------------------------------------------------------------ inverse
// Column pass: the type-3 pre-rotation and packing of the pairs of block
// pair P into the tile (s[blk + 4p] at (slot*W + col, p)), then the Q-point
// DFTs over p, written as V_blk[j].
template <int QL, int R>
__global__ void __launch_bounds__(512, 1) dctq_col_inv(const DctqParams q) {
  constexpr int TPT = QL / R;
  pdl_release();
  pdl_wait();
  extern __shared__ __align__(16) unsigned char smem[];
  const int W = q.W, cpb = 2 * W;
  const int tid = threadIdx.x;
  const int64_t N = q.N, Nr = q.Nr, Lc = 4 * int64_t(QL);
  const int64_t gpr = N / W;
  const int64_t g = blockIdx.x % gpr, rest = blockIdx.x / gpr;
  const int P = int(rest % 2);
  const int64_t h = rest / 2;
  const int64_t n0 = g * W;
  Tile t{reinterpret_cast<cpx*>(smem), q.lp};
  const real* in = static_cast<const real*>(q.in) + h * Nr * N + n0;
  const bool dst = (q.flags & F_DST) != 0;
  const int npairs = P == 1 ? QL : QL + 1;
  for (int e = tid; e < npairs * W; e += blockDim.x) {
    const int cc = e % W, pi = e / W;
    auto rd = [&](int i) { return in[int64_t(i) * N + cc]; };
    auto z = [&](int64_t k) { return LoadDCT3::zval_r(rd, int(k), int(Lc), dst, q.t23_c); };
    if (P == 1) {  // k = 1 + 4p, partner 3 + 4(Q-1-p); packed from the smaller member
      const int64_t k = 1 + 4 * int64_t(pi);
      cpx ta, tb;
      if (2 * k < Lc) {
        pack_pair(z(k), z(Lc - k), ldg(q.rft_c + k), ta, tb);
        t.s[t.idx(cc, pi)] = cconj(ta);
        t.s[t.idx(W + cc, QL - 1 - pi)] = cconj(tb);
      } else {
        pack_pair(z(Lc - k), z(k), ldg(q.rft_c + (Lc - k)), ta, tb);
        t.s[t.idx(W + cc, QL - 1 - pi)] = cconj(ta);
        t.s[t.idx(cc, pi)] = cconj(tb);
      }
    } else if (pi <= QL / 2) {  // k = 4p, partner 4(Q-p) (k = 0 pairs with Lc)
      const int64_t k = 4 * int64_t(pi);
      const cpx z0 = z(k);
      if (k == 0) {
        const cpx z1 = z(Lc);
        t.s[t.idx(cc, 0)] = cmk(z0.x + z1.x, -(z0.x - z1.x));
      } else if (2 * k == Lc) {
        t.s[t.idx(cc, pi)] = cmk(2 * z0.x, 2 * z0.y);
      } else {
        cpx ta, tb;
        pack_pair(z0, z(Lc - k), ldg(q.rft_c + k), ta, tb);
        t.s[t.idx(cc, pi)] = cconj(ta);
        t.s[t.idx(cc, QL - pi)] = cconj(tb);
      }
    } else {  // k = 2 + 4p, partner 2 + 4(Q-1-p)
      const int p2 = pi - QL / 2 - 1;
      const int64_t k = 2 + 4 * int64_t(p2);
      cpx ta, tb;
      pack_pair(z(k), z(Lc - k), ldg(q.rft_c + k), ta, tb);
      t.s[t.idx(W + cc, p2)] = cconj(ta);
      t.s[t.idx(W + cc, QL - 1 - p2)] = cconj(tb);
    }
  }
  __syncthreads();
  const int c = tid % cpb, jt = tid / cpb;
  const int slot = c / W, col = c % W;
  const int blk = P + 2 * slot;
  cpx v[R];
  gather_natural<QL, R>(v, jt, c, t);
  run_passes<QL, R, 1>(v, jt, c, t, q.tw_q);
  cpx* dstp = q.mid + ((h * 4 + blk) * QL) * N + n0 + col;
#pragma unroll
  for (int r = 0; r < R; ++r) dstp[int64_t(jt + r * TPT) * N] = v[r];
}

// Row pass: the radix-4 stage S[j + Q m'] = sum_q w_4^(qm') w_Lc^(qj) V_q[j]
// for every column, its conjugate written as the reals of the 8 rows into
// their tile slots, then the rows' DCT-3s (the staged form of LoadDCT3).
template <int L, int R>
__global__ void __launch_bounds__(8 * (L / R), 1) dctq_row_inv(const DctqParams q) {
  constexpr int TPT = L / R;
  constexpr int NT = 8 * TPT;
  constexpr int N = 2 * L;
  pdl_release();
  pdl_wait();
  extern __shared__ __align__(16) unsigned char smem[];
  const int tid = threadIdx.x;
  const int64_t j = blockIdx.x % q.Q, h = blockIdx.x / q.Q;
  Tile t{reinterpret_cast<cpx*>(smem), q.lp};
  const bool dst = (q.flags & F_DST) != 0;
  const real sg = dst ? real(-1) : real(1);
  {
    const cpx w1 = ldg(q.tw_c + j), w2 = ldg(q.tw_c + 2 * j), w3 = ldg(q.tw_c + 3 * j);
    const cpx* src = q.mid + (h * 4 * q.Q + j) * N;
    const int64_t bs = q.Q * N;
    for (int n = tid; n < N; n += NT) {
      // V_q[j] times w_Lc^(qj), then the radix-4 DFT over q: S_m' = sum_q w_4^(qm') u_q
      const cpx u0 = src[n], u1 = cmul(src[bs + n], w1), u2 = cmul(src[2 * bs + n], w2),
                u3 = cmul(src[3 * bs + n], w3);
      const cpx a0 = cadd(u0, u2), a1 = csub(u0, u2), c0 = cadd(u1, u3), c1 = csub(u1, u3);
      const cpx mic1 = cmk(c1.y, -c1.x);  // -i * c1
      const cpx S[4] = {cadd(a0, c0), cadd(a1, mic1), csub(a0, c0), csub(a1, mic1)};
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const cpx w = cconj(S[m]);
        const real s = m < 2 ? real(1) : sg;
        tile_row(t, 2 * m)[n] = s * w.x;
        tile_row(t, 2 * m + 1)[n] = s * w.y;
      }
    }
  }
  __syncthreads();
  // the rows' DCT-3s: pre-rotation and packing from the staged rows
  const int c = tid / TPT, jt = tid % TPT;
  AxisParams p = dctq_row_params(q, q.lp);
  p.t1 = q.t23_row;
  p.t2 = q.rft_row;
  p.out = static_cast<real*>(q.out) + h * q.Nr * N;
  Ctx x;
  x.c = c;
  x.j = jt;
  x.b = 0;
  x.b0 = 0;
  x.active = true;
  x.oin = 0;
  x.oout = dctq_row(q, j, c) * N;
  cpx v[R];
  {
    const cpx b1 = kind_base<TPT>(q.t23_row, jt), b2 = kind_base<TPT>(q.rft_row, jt);
    real* sr = tile_row(t, c);
    constexpr int NPP = R / 2 + 1;
    cpx za[NPP], zb[NPP];
    auto rd = [&](int m) { return sr[m]; };
#pragma unroll
    for (int i = 0; i < NPP; ++i) {
      const int k = jt + i * TPT;
      const bool own = i < R / 2 || jt == 0;
      const cpx rk = t23_root<R>(b1, i);
      za[i] = own ? LoadDCT3::zval_w(rd, k, L, dst, [&](int) { return rk; }) : czero();
      zb[i] = own ? LoadDCT3::zval_w(rd, L - k, L, dst, [&](int) { return t23_mirror(rk); }) : czero();
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < NPP; ++i)
      if (i < R / 2 || jt == 0) pack_into(t, c, jt + i * TPT, L, za[i], zb[i], rft_root<R>(b2, i));
    __syncthreads();
    gather_natural<L, R>(v, jt, c, t);
  }
  run_passes<L, R, 1>(v, jt, c, t, q.tw_row);
  StoreDCT3::run<L, R>(p, x, t, TileOffsets{nullptr, nullptr, 8}, v);
}

// ------------------------------------------------------------------ registry
size_t dctq_row_smem(int L) {
  const int R = 16;
  return size_t(8) * tile_pitch(L, R, 8, 0) * sizeof(cpx);
}
size_t dctq_col_smem(int QL, int W) {
  const int R = 16;
  return size_t(2 * W) * tile_pitch(QL, R, 2 * W, 1) * sizeof(cpx);
}

const void* dctq_kernel(int which, int log2len) {
  // which: 0 row forward, 1 column forward, 2 column inverse, 3 row inverse;
  // rows L = 2^6 .. 2^10, columns Q = 2^6 .. 2^9
  switch (which) {
    case 0:
    case 3: {
      static const void* const f[5] = {(const void*)dctq_row_fwd<64, 16>, (const void*)dctq_row_fwd<128, 16>,
                                       (const void*)dctq_row_fwd<256, 16>, (const void*)dctq_row_fwd<512, 16>,
                                       (const void*)dctq_row_fwd<1024, 16>};
      static const void* const i[5] = {(const void*)dctq_row_inv<64, 16>, (const void*)dctq_row_inv<128, 16>,
                                       (const void*)dctq_row_inv<256, 16>, (const void*)dctq_row_inv<512, 16>,
                                       (const void*)dctq_row_inv<1024, 16>};
      if (log2len < 6 || log2len > 10) return nullptr;
      return which == 0 ? f[log2len - 6] : i[log2len - 6];
    }
    default: {
      static const void* const f[4] = {(const void*)dctq_col_fwd<64, 16>, (const void*)dctq_col_fwd<128, 16>,
                                       (const void*)dctq_col_fwd<256, 16>, (const void*)dctq_col_fwd<512, 16>};
      static const void* const i[4] = {(const void*)dctq_col_inv<64, 16>, (const void*)dctq_col_inv<128, 16>,
                                       (const void*)dctq_col_inv<256, 16>, (const void*)dctq_col_inv<512, 16>};
      if (log2len < 6 || log2len > 9) return nullptr;
      return which == 1 ? f[log2len - 6] : i[log2len - 6];
    }
  }
}

}  // namespace mb
