// Element-wise pre- and post-processing steps of real-data transforms whose
// half-length complex DFT runs as several HBM passes, and the length-1 axis
// steps, as device functions: Op::count(p) work items, Op::item(p, e) does
// item e.  The steps the mixed-batch kernel runs as sweeps also come as
// Op::load_at(p, it), which reads everything item it needs (data and roots)
// into an Op::In, and Op::finish_at(p, it, in), which computes and stores:
// a CTA that walks a line alone then issues the loads of several items
// before any of their stores.  Used by the line kernels (line_kernels.cu)
// and by the mixed-batch kernel (mixed.cu).
//
// Data layout: a batch of outer x inner lines along one axis; element n of
// line (o, i) of the input sits at o*in_so + n*in_sn + i, of the output at
// o*out_so + n*out_sn + i.  The item index runs fastest over i (adjacent
// columns) and then over n, so a warp touches contiguous memory for both
// column and row layouts.
#pragma once

#include "axis_pass.cuh"
#include "line_kernels.h"

namespace mb {

// Entry i of the kind tables t1 / t2 (coarse/fine product when given).
__device__ __forceinline__ cpx cf_root(const cpx* hi, const cpx* lo, int bits, int64_t e) {
  return cmul(ldg(hi + (e >> bits)), ldg(lo + (e & ((int64_t(1) << bits) - 1))));
}
__device__ __forceinline__ cpx root1(const LineParams& p, int64_t i) {
  return p.hi1 ? cf_root(p.hi1, p.lo1, p.bits1, i * p.mul1 + p.add1) : ldg(p.t1 + i);
}
__device__ __forceinline__ cpx root2(const LineParams& p, int64_t i) {
  return p.hi2 ? cf_root(p.hi2, p.lo2, p.bits2, i * p.mul2 + p.add2) : ldg(p.t2 + i);
}

struct ItemIdx {
  int64_t o, n, i;
};

// Item e = (o * K + n) * inner + i.  Power-of-two extents (inner always, K
// unless it counts L/2+1 spectrum points) split by masks and shifts: the
// 64-bit quotient sequences otherwise keep the conversion pipe busy for most
// of a line kernel's time.
__device__ __forceinline__ ItemIdx split_item(int64_t e, int64_t inner, int64_t K) {
  ItemIdx r;
  int64_t q;
  if ((inner & (inner - 1)) == 0) {
    r.i = e & (inner - 1);
    q = e >> (__ffsll(inner) - 1);
  } else {
    r.i = e % inner;
    q = e / inner;
  }
  if ((K & (K - 1)) == 0) {
    r.n = q & (K - 1);
    r.o = q >> (__ffsll(K) - 1);
  } else {
    r.n = q % K;
    r.o = q / K;
  }
  return r;
}

// complex t_m = (u_2m, u_2m+1) of the type-2 permutation (see LoadDCT2)
struct Op_dct2_pre {
  static __device__ __forceinline__ int64_t count(const LineParams& p) {
    const int64_t L = p.L;
    return p.outer * p.inner * L;
  }
  struct In {
    real a, b;
  };
  static __device__ __forceinline__ In load_at(const LineParams& p, const ItemIdx& it) {
    const int64_t L = p.L, N = 2 * L;
    const real* in = static_cast<const real*>(p.in) + it.o * p.in_so + it.i;
    const int64_t i0 = 2 * it.n, i1 = 2 * it.n + 1;
    return In{i0 < L ? in[(2 * i0) * p.in_sn] : in[(2 * N - 1 - 2 * i0) * p.in_sn],
              i1 < L ? in[(2 * i1) * p.in_sn] : in[(2 * N - 1 - 2 * i1) * p.in_sn]};
  }
  static __device__ __forceinline__ void finish_at(const LineParams& p, const ItemIdx& it, const In& v) {
    const int64_t L = p.L;
    const real sg = (p.flags & F_DST) ? real(-1) : real(1);
    const int64_t i0 = 2 * it.n, i1 = 2 * it.n + 1;
    static_cast<cpx*>(p.out)[it.o * p.out_so + it.n * p.out_sn + it.i] =
        cmk(i0 < L ? v.a : sg * v.a, i1 < L ? v.b : sg * v.b);
  }
  static __device__ __forceinline__ ItemIdx index(const LineParams& p, int64_t e) {
    return split_item(e, p.inner, p.L);
  }
  static __device__ __forceinline__ In load(const LineParams& p, int64_t e) { return load_at(p, index(p, e)); }
  static __device__ __forceinline__ void finish(const LineParams& p, int64_t e, const In& v) {
    finish_at(p, index(p, e), v);
  }
  static __device__ __forceinline__ void item(const LineParams& p, int64_t e) {
    const ItemIdx it = index(p, e);
    finish_at(p, it, load_at(p, it));
  }
};

// The type-4 steps take each point n < L/2 with its mirror n' = L-1-n:
// x[2n+1] = x[N-1-2n'] and x[N-2-2n] = x[2n'], so the pair reads the reals
// (x[2n], x[2n+1]) and (x[N-2-2n], x[N-1-2n]), and the post-rotation writes
// (y[2m], y[2m+1]) and (y[N-2-2m], y[N-1-2m]), as vectors where a line is
// contiguous and aligned (whole sectors instead of single reals at a
// stride of two).
template <class T>
__device__ __forceinline__ bool pair_vec(const T* base, const LineParams& p, int64_t sn) {
  return sn == 1 && p.inner == 1 && (reinterpret_cast<uintptr_t>(base) % sizeof(cpx)) == 0;
}

// type-4 pre-rotation (see LoadT4), points n and L-1-n per item
struct Op_t4_pre {
  static __device__ __forceinline__ int64_t count(const LineParams& p) { return p.outer * p.inner * (p.L / 2); }
  static __device__ __forceinline__ cpx rot(bool dst, cpx w, real a, real b) {
    if (!dst) return cmul(w, cmk(a, b));
    const cpx q = cmul(w, cmk(a, -b));
    return cmk(-q.x, -q.y);
  }
  static __device__ __forceinline__ void item(const LineParams& p, int64_t e) {
    const int64_t L = p.L, N = 2 * L;
    const bool dst = (p.flags & F_DST) != 0;
    const ItemIdx it = split_item(e, p.inner, L / 2);
    const int64_t n = it.n, m = L - 1 - n, sn = p.in_sn;
    const real* in = static_cast<const real*>(p.in) + it.o * p.in_so + it.i;
    real x0, x1, y0, y1;  // x[2n], x[2n+1], x[N-2-2n], x[N-1-2n]
    if (pair_vec(in, p, sn)) {
      const cpx u = *reinterpret_cast<const cpx*>(in + 2 * n), w = *reinterpret_cast<const cpx*>(in + N - 2 - 2 * n);
      x0 = u.x;
      x1 = u.y;
      y0 = w.x;
      y1 = w.y;
    } else {
      x0 = in[(2 * n) * sn];
      x1 = in[(2 * n + 1) * sn];
      y0 = in[(N - 2 - 2 * n) * sn];
      y1 = in[(N - 1 - 2 * n) * sn];
    }
    cpx* out = static_cast<cpx*>(p.out) + it.o * p.out_so + it.i;
    out[n * p.out_sn] = rot(dst, root1(p, n), x0, y1);
    out[m * p.out_sn] = rot(dst, root1(p, m), y0, x1);
  }
  // One contiguous line (unit strides, an input aligned for the vector
  // reads) shorter than 2^30 points, with roots w_2N^n: the same item in
  // 32-bit index arithmetic (the 64-bit products and shifts of the general
  // form are most of its instructions).
  static __device__ __forceinline__ bool fast(const LineParams& p) {
    return p.outer == 1 && p.inner == 1 && p.in_sn == 1 && p.out_sn == 1 && p.hi1 && p.mul1 == 1 &&
           p.add1 == 0 && p.L < (int64_t(1) << 30) && (reinterpret_cast<uintptr_t>(p.in) % sizeof(cpx)) == 0;
  }
  static __device__ __forceinline__ uint32_t count32(const LineParams& p) { return uint32_t(p.L / 2); }
  static __device__ __forceinline__ void item32(const LineParams& p, uint32_t n) {
    const uint32_t L = uint32_t(p.L), N = 2 * L, m = L - 1 - n;
    const real* in = static_cast<const real*>(p.in);
    const cpx u = *reinterpret_cast<const cpx*>(in + 2 * n);            // x[2n], x[2n+1]
    const cpx w = *reinterpret_cast<const cpx*>(in + (N - 2 - 2 * n));  // x[N-2-2n], x[N-1-2n]
    const uint32_t mask = (1u << p.bits1) - 1;
    const cpx r0 = cmul(ldg(p.hi1 + (n >> p.bits1)), ldg(p.lo1 + (n & mask)));
    const cpx r1 = cmul(ldg(p.hi1 + (m >> p.bits1)), ldg(p.lo1 + (m & mask)));
    const bool dst = (p.flags & F_DST) != 0;
    cpx* out = static_cast<cpx*>(p.out);
    out[n] = rot(dst, r0, u.x, w.y);
    out[m] = rot(dst, r1, w.x, u.y);
  }
};

// inverse-real-DFT packing, conjugated (see LoadC2R); in: L+1 spectrum values
struct Op_c2r_pack {
  static __device__ __forceinline__ int64_t count(const LineParams& p) {
    const int64_t L = p.L, K = L / 2 + 1;
    return p.outer * p.inner * K;
  }
  struct In {
    cpx z0, z1, f;
  };
  static __device__ __forceinline__ In load_at(const LineParams& p, const ItemIdx& it) {
    const int64_t L = p.L, K = L / 2 + 1;
    const cpx* in = static_cast<const cpx*>(p.in) + it.o * p.in_so + it.i;
    const int64_t k = it.n;
    return In{in[k * p.in_sn], in[(L - k) * p.in_sn], (k != 0 && 2 * k != L) ? root2(p, k) : czero()};
  }
  static __device__ __forceinline__ void finish_at(const LineParams& p, const ItemIdx& it, const In& v) {
    const int64_t L = p.L, K = L / 2 + 1;
    cpx* out = static_cast<cpx*>(p.out) + it.o * p.out_so + it.i;
    const int64_t k = it.n;
    if (k == 0) {
      out[0] = cmk(v.z0.x + v.z1.x, -(v.z0.x - v.z1.x));
    } else if (2 * k == L) {
      out[k * p.out_sn] = cmk(2 * v.z0.x, 2 * v.z0.y);
    } else {
      cpx ta, tb;
      pack_pair(v.z0, v.z1, v.f, ta, tb);
      out[k * p.out_sn] = cconj(ta);
      out[(L - k) * p.out_sn] = cconj(tb);
    }
  }
  static __device__ __forceinline__ ItemIdx index(const LineParams& p, int64_t e) {
    return split_item(e, p.inner, p.L / 2 + 1);
  }
  static __device__ __forceinline__ In load(const LineParams& p, int64_t e) { return load_at(p, index(p, e)); }
  static __device__ __forceinline__ void finish(const LineParams& p, int64_t e, const In& v) {
    finish_at(p, index(p, e), v);
  }
  static __device__ __forceinline__ void item(const LineParams& p, int64_t e) {
    const ItemIdx it = index(p, e);
    finish_at(p, it, load_at(p, it));
  }
};

// type-3 pre-rotation + packing, conjugated (see LoadDCT3)
struct Op_dct3_pack {
  static __device__ __forceinline__ int64_t count(const LineParams& p) {
    const int64_t L = p.L, K = L / 2 + 1;
    return p.outer * p.inner * K;
  }
  struct In {
    cpx z0, z1, f;
  };
  // the reads and the pre-rotation of both values of the pair
  static __device__ __forceinline__ In load_at(const LineParams& p, const ItemIdx& it) {
    const int64_t L = p.L, K = L / 2 + 1;
    const bool dst = (p.flags & F_DST) != 0;
    const real* in = static_cast<const real*>(p.in) + it.o * p.in_so + it.i;
    const int k = int(it.n);
    auto rd = [&](int i) { return in[int64_t(i) * p.in_sn]; };
    return In{LoadDCT3::zval_w(rd, k, int(L), dst, [&](int n) { return root1(p, n); }),
              LoadDCT3::zval_w(rd, int(L) - k, int(L), dst, [&](int n) { return root1(p, n); }),
              (k != 0 && 2 * k != L) ? root2(p, k) : czero()};
  }
  static __device__ __forceinline__ void finish_at(const LineParams& p, const ItemIdx& it, const In& v) {
    const int64_t L = p.L, K = L / 2 + 1;
    cpx* out = static_cast<cpx*>(p.out) + it.o * p.out_so + it.i;
    const int k = int(it.n);
    const cpx z0 = v.z0, z1 = v.z1;
    if (k == 0) {
      out[0] = cmk(z0.x + z1.x, -(z0.x - z1.x));
    } else if (2 * k == L) {
      out[k * p.out_sn] = cmk(2 * z0.x, 2 * z0.y);
    } else {
      cpx ta, tb;
      pack_pair(z0, z1, v.f, ta, tb);
      out[k * p.out_sn] = cconj(ta);
      out[(L - k) * p.out_sn] = cconj(tb);
    }
  }
  static __device__ __forceinline__ ItemIdx index(const LineParams& p, int64_t e) {
    return split_item(e, p.inner, p.L / 2 + 1);
  }
  static __device__ __forceinline__ In load(const LineParams& p, int64_t e) { return load_at(p, index(p, e)); }
  static __device__ __forceinline__ void finish(const LineParams& p, int64_t e, const In& v) {
    finish_at(p, index(p, e), v);
  }
  static __device__ __forceinline__ void item(const LineParams& p, int64_t e) {
    const ItemIdx it = index(p, e);
    finish_at(p, it, load_at(p, it));
  }
};

// real-DFT unpacking (see StoreR2C); out: L+1 spectrum values
struct Op_r2c_unpack {
  static __device__ __forceinline__ int64_t count(const LineParams& p) {
    const int64_t L = p.L, K = L / 2 + 1;
    return p.outer * p.inner * K;
  }
  struct In {
    cpx za, zb, f;
  };
  static __device__ __forceinline__ In load_at(const LineParams& p, const ItemIdx& it) {
    const int64_t L = p.L, K = L / 2 + 1;
    const cpx* in = static_cast<const cpx*>(p.in) + it.o * p.in_so + it.i;
    const int64_t k = it.n;
    const bool pair = k != 0 && 2 * k != L;
    return In{in[k * p.in_sn], pair ? in[(L - k) * p.in_sn] : czero(), pair ? root1(p, k) : czero()};
  }
  static __device__ __forceinline__ void finish_at(const LineParams& p, const ItemIdx& it, const In& v) {
    const int64_t L = p.L, K = L / 2 + 1;
    cpx* out = static_cast<cpx*>(p.out) + it.o * p.out_so + it.i;
    const int64_t k = it.n;
    const cpx za = v.za;
    if (k == 0) {
      out[0] = cmk(za.x + za.y, real(0));
      out[L * p.out_sn] = cmk(za.x - za.y, real(0));
    } else if (2 * k == L) {
      out[k * p.out_sn] = cconj(za);
    } else {
      cpx xa, xb;
      unpack_pair(za, v.zb, v.f, xa, xb);
      out[k * p.out_sn] = xa;
      out[(L - k) * p.out_sn] = xb;
    }
  }
  static __device__ __forceinline__ ItemIdx index(const LineParams& p, int64_t e) {
    return split_item(e, p.inner, p.L / 2 + 1);
  }
  static __device__ __forceinline__ In load(const LineParams& p, int64_t e) { return load_at(p, index(p, e)); }
  static __device__ __forceinline__ void finish(const LineParams& p, int64_t e, const In& v) {
    finish_at(p, index(p, e), v);
  }
  static __device__ __forceinline__ void item(const LineParams& p, int64_t e) {
    const ItemIdx it = index(p, e);
    finish_at(p, it, load_at(p, it));
  }
};

// type-2 unpacking + post-rotation (see StoreDCT2)
struct Op_dct2_post {
  static __device__ __forceinline__ int64_t count(const LineParams& p) {
    const int64_t L = p.L, K = L / 2 + 1;
    return p.outer * p.inner * K;
  }
  struct In {
    cpx za, zb, f, ea, eb;
  };
  static __device__ __forceinline__ In load_at(const LineParams& p, const ItemIdx& it) {
    const int64_t L = p.L, K = L / 2 + 1;
    const cpx* in = static_cast<const cpx*>(p.in) + it.o * p.in_so + it.i;
    const int64_t k = it.n;
    const bool pair = k != 0 && 2 * k != L;
    return In{in[k * p.in_sn], pair ? in[(L - k) * p.in_sn] : czero(), pair ? root2(p, k) : czero(),
              k != 0 ? root1(p, k) : czero(), pair ? root1(p, L - k) : czero()};
  }
  static __device__ __forceinline__ void finish_at(const LineParams& p, const ItemIdx& it, const In& v) {
    const int64_t L = p.L, K = L / 2 + 1;
    const int N = int(2 * L);
    const bool dst = (p.flags & F_DST) != 0;
    const real r2 = real(1.414213562373095048801688724209698079);
    real* out = static_cast<real*>(p.out) + it.o * p.out_so + it.i;
    const int k = int(it.n);
    const cpx za = v.za;
    if (k == 0) {
      const real v0 = za.x + za.y, vl = za.x - za.y;
      out[int64_t(dst ? N - 1 : 0) * p.out_sn] = 2 * v0;
      out[int64_t(dst ? L - 1 : L) * p.out_sn] = r2 * vl;
    } else if (2 * k == L) {
      StoreDCT2::emit(out, p.out_sn, k, N, dst, cconj(za), v.ea);
    } else {
      cpx xa, xb;
      unpack_pair2(za, v.zb, v.f, xa, xb);
      StoreDCT2::emit2(out, p.out_sn, k, N, dst, xa, v.ea);
      StoreDCT2::emit2(out, p.out_sn, int(L) - k, N, dst, xb, v.eb);
    }
  }
  static __device__ __forceinline__ ItemIdx index(const LineParams& p, int64_t e) {
    return split_item(e, p.inner, p.L / 2 + 1);
  }
  static __device__ __forceinline__ In load(const LineParams& p, int64_t e) { return load_at(p, index(p, e)); }
  static __device__ __forceinline__ void finish(const LineParams& p, int64_t e, const In& v) {
    finish_at(p, index(p, e), v);
  }
  static __device__ __forceinline__ void item(const LineParams& p, int64_t e) {
    const ItemIdx it = index(p, e);
    finish_at(p, it, load_at(p, it));
  }
};

// type-3 de-interleave of the conjugated forward result (see StoreDCT3)
struct Op_dct3_post {
  static __device__ __forceinline__ int64_t count(const LineParams& p) {
    const int64_t L = p.L;
    return p.outer * p.inner * L;
  }
  struct In {
    cpx w;
  };
  static __device__ __forceinline__ In load_at(const LineParams& p, const ItemIdx& it) {
    return In{static_cast<const cpx*>(p.in)[it.o * p.in_so + it.n * p.in_sn + it.i]};
  }
  static __device__ __forceinline__ ItemIdx index(const LineParams& p, int64_t e) {
    return split_item(e, p.inner, p.L);
  }
  static __device__ __forceinline__ In load(const LineParams& p, int64_t e) { return load_at(p, index(p, e)); }
  static __device__ __forceinline__ void finish(const LineParams& p, int64_t e, const In& v) {
    finish_at(p, index(p, e), v);
  }
  static __device__ __forceinline__ void item(const LineParams& p, int64_t e) {
    const ItemIdx it = index(p, e);
    finish_at(p, it, load_at(p, it));
  }
  static __device__ __forceinline__ void finish_at(const LineParams& p, const ItemIdx& it, const In& v) {
    const int64_t L = p.L, N = 2 * L;
    const bool dst = (p.flags & F_DST) != 0;
    const cpx w = cconj(v.w);
    real* out = static_cast<real*>(p.out) + it.o * p.out_so + it.i;
    const int64_t i0 = 2 * it.n, i1 = 2 * it.n + 1;
    const real a = (dst && i0 >= L) ? -w.x : w.x;
    const real b = (dst && i1 >= L) ? -w.y : w.y;
    out[(i0 < L ? 2 * i0 : 2 * N - 1 - 2 * i0) * p.out_sn] = a;
    out[(i1 < L ? 2 * i1 : 2 * N - 1 - 2 * i1) * p.out_sn] = b;
  }
};

// type-4 post-rotation (see StoreT4), points m and L-1-m per item
struct Op_t4_post {
  static __device__ __forceinline__ int64_t count(const LineParams& p) { return p.outer * p.inner * (p.L / 2); }
  static __device__ __forceinline__ void item(const LineParams& p, int64_t e) {
    const int64_t L = p.L, N = 2 * L;
    const bool dst = (p.flags & F_DST) != 0;
    const ItemIdx it = split_item(e, p.inner, L / 2);
    const int64_t m = it.n, mm = L - 1 - m;
    const cpx* in = static_cast<const cpx*>(p.in) + it.o * p.in_so + it.i;
    const cpx T = in[m * p.in_sn], U = in[mm * p.in_sn];
    // y[2m] = 2 Re(g_2m T_m), y[N-1-2m] = 2 Re(g_(N-1-2m) conj(T_m)); the
    // mirror's y[2mm] = y[N-2-2m] and y[N-1-2mm] = y[2m+1] (Im for DST-4)
    auto part = [&](cpx v) { return 2 * (dst ? v.y : v.x); };
    const real a0 = part(cmul(root2(p, 2 * m), T));            // y[2m]
    const real b0 = part(cmul(root2(p, N - 1 - 2 * m), cconj(T)));  // y[N-1-2m]
    const real a1 = part(cmul(root2(p, N - 2 - 2 * m), U));    // y[N-2-2m]
    const real b1 = part(cmul(root2(p, 2 * m + 1), cconj(U)));  // y[2m+1]
    real* out = static_cast<real*>(p.out) + it.o * p.out_so + it.i;
    const int64_t sn = p.out_sn;
    if (pair_vec(out, p, sn)) {
      *reinterpret_cast<cpx*>(out + 2 * m) = cmk(a0, b1);
      *reinterpret_cast<cpx*>(out + N - 2 - 2 * m) = cmk(a1, b0);
    } else {
      out[(2 * m) * sn] = a0;
      out[(2 * m + 1) * sn] = b1;
      out[(N - 2 - 2 * m) * sn] = a1;
      out[(N - 1 - 2 * m) * sn] = b0;
    }
  }
};

// p.L = number of elements, p.flags selects the mode, p.scale the factor.
struct Op_unit {
  static __device__ __forceinline__ int64_t count(const LineParams& p) {
    return p.L;
  }
  static __device__ __forceinline__ void item(const LineParams& p, int64_t e) {
    switch (p.mode) {
      case UNIT_SCALE_REAL:
        static_cast<real*>(p.out)[e] = p.scale * static_cast<const real*>(p.in)[e];
        break;
      case UNIT_REAL_TO_CPLX:
        static_cast<cpx*>(p.out)[e] = cmk(static_cast<const real*>(p.in)[e], real(0));
        break;
      case UNIT_CPLX_TO_REAL:
        static_cast<real*>(p.out)[e] = static_cast<const cpx*>(p.in)[e].x;
        break;
      default:
        static_cast<cpx*>(p.out)[e] = static_cast<const cpx*>(p.in)[e];
        break;
    }
  }
};

}  // namespace mb
