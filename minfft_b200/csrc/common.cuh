// Device-side building blocks shared by every transform kernel: the complex
// type of the working precision, complex arithmetic, compile-time twiddle
// constants and the in-register power-of-two DFT used as the butterfly of
// every Stockham pass.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

#ifndef MINFFT_SINGLE
#define MINFFT_SINGLE 0
#endif

namespace mb {

#if MINFFT_SINGLE
typedef float real;
typedef float2 cpx;
#else
typedef double real;
typedef double2 cpx;
#endif

// ---------------------------------------------------------------- complex ops
__device__ __forceinline__ cpx cmk(real re, real im) {
  cpx c;
  c.x = re;
  c.y = im;
  return c;
}
__device__ __forceinline__ cpx cadd(cpx a, cpx b) { return cmk(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ cpx csub(cpx a, cpx b) { return cmk(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ cpx cmul(cpx a, cpx b) { return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
// a * conj(b)
__device__ __forceinline__ cpx cmulc(cpx a, cpx b) { return cmk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); }
__device__ __forceinline__ cpx cconj(cpx a) { return cmk(a.x, -a.y); }
__device__ __forceinline__ cpx cscale(cpx a, real s) { return cmk(a.x * s, a.y * s); }
// a * (-i)
__device__ __forceinline__ cpx cmul_negi(cpx a) { return cmk(a.y, -a.x); }
__device__ __forceinline__ cpx czero() { return cmk(real(0), real(0)); }

// ------------------------------------------------- compile-time unit roots
// cos(pi*q/16) for q = 0..8 (exact decimal expansions of the constants).
__host__ __device__ constexpr double kCos32(int q) {
  return q == 0   ? 1.0
         : q == 1 ? 0.980785280403230449126182236134239037
         : q == 2 ? 0.923879532511286756128183189396788933
         : q == 3 ? 0.831469612302545237078788377617905756
         : q == 4 ? 0.707106781186547524400844362104849039
         : q == 5 ? 0.555570233019602224742830813948532874
         : q == 6 ? 0.382683432365089771728459984030398867
         : q == 7 ? 0.195090322016128267848284868477022240
                  : 0.0;
}

// Multiply a by w_M^K = exp(-2*pi*i*K/M) for M <= 32, all at compile time.
// Trivial angles (0, -pi/2, -pi/4, -3pi/4) cost no multiplies.
template <int M, int K>
__device__ __forceinline__ cpx twc(cpx a) {
  static_assert(M <= 32 && (32 % M) == 0, "compile-time roots cover M | 32");
  constexpr int q = (K * 32 / M) % 32;  // angle in units of 2*pi/32
  if constexpr (q == 0) {
    return a;
  } else if constexpr (q == 8) {
    return cmul_negi(a);
  } else if constexpr (q == 16) {
    return cmk(-a.x, -a.y);
  } else if constexpr (q == 24) {
    return cmk(-a.y, a.x);
  } else if constexpr (q == 4) {
    constexpr real h = real(kCos32(4));
    return cmk(h * (a.x + a.y), h * (a.y - a.x));
  } else if constexpr (q == 12) {
    constexpr real h = real(kCos32(4));
    return cmk(h * (a.y - a.x), -h * (a.x + a.y));
  } else {
    // w = c - i s with c = cos(2*pi*q/32), s = sin(2*pi*q/32)
    constexpr int qq = q % 16;  // angle mod pi
    constexpr double c0 = qq <= 8 ? kCos32(qq) : -kCos32(16 - qq);
    constexpr double s0 = qq <= 8 ? kCos32(8 - qq) : kCos32(qq - 8);
    constexpr real c = real(q < 16 ? c0 : -c0);
    constexpr real s = real(q < 16 ? s0 : -s0);
    return cmk(a.x * c + a.y * s, a.y * c - a.x * s);
  }
}

// ------------------------------------------------ in-register DFT (forward)
// Radix-2 decimation in frequency over N registers, fully resolved at
// compile time (index sequences, no loops over runtime indices), followed by
// a compile-time bit-reversal so the result is in natural order.
__host__ __device__ constexpr int bitrev_c(int k, int n) {
  int r = 0;
  for (int b = 1; b < n; b <<= 1) {
    r = (r << 1) | (k & 1);
    k >>= 1;
  }
  return r;
}

template <int H, int P, int K>
__device__ __forceinline__ void bfly2(cpx* v) {
  cpx a = v[P], b = v[P + H];
  v[P] = cadd(a, b);
  v[P + H] = twc<2 * H, K>(csub(a, b));
}

template <int H, int... I>
__device__ __forceinline__ void dif_stage(cpx* v, std::integer_sequence<int, I...>) {
  (bfly2<H, (I / H) * 2 * H + (I % H), I % H>(v), ...);
}

template <int N, int H>
__device__ __forceinline__ void dif_stages(cpx* v) {
  dif_stage<H>(v, std::make_integer_sequence<int, N / 2>{});
  if constexpr (H > 1) dif_stages<N, H / 2>(v);
}

template <int N, int... I>
__device__ __forceinline__ void bitrev_perm(cpx* v, std::integer_sequence<int, I...>) {
  cpx t[N] = {v[bitrev_c(I, N)]...};
  ((v[I] = t[I]), ...);
}

template <int N>
__device__ __forceinline__ void fft_reg(cpx* v) {
  if constexpr (N >= 2) {
    dif_stages<N, N / 2>(v);
    bitrev_perm<N>(v, std::make_integer_sequence<int, N>{});
  }
}

// ------------------------------------------------ programmatic dependent launch
// A kernel enqueued with the programmatic stream-serialization attribute may
// be scheduled while the kernel before it drains.  pdl_wait() blocks until
// that predecessor grid has completed and its writes are visible (a no-op
// for an ordinary launch); pdl_release() allows the next kernel to be
// scheduled once every CTA of this grid has called it or exited.  Every
// kernel the planner launches calls both before touching global memory.
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// --------------------------------------------------------------- misc utils
// Quotient and remainder of non-negative 64-bit values, in 32-bit
// arithmetic when both fit in 31 bits (every batch index and extent of the
// plans in practice; the 64-bit sequences are several times longer).
__device__ __forceinline__ int64_t udiv(int64_t a, int64_t b) {
  return ((a | b) >> 31) == 0 ? int64_t(uint32_t(a) / uint32_t(b)) : a / b;
}
__device__ __forceinline__ int64_t umod(int64_t a, int64_t b) {
  return ((a | b) >> 31) == 0 ? int64_t(uint32_t(a) % uint32_t(b)) : a % b;
}

__device__ __forceinline__ int pad16(int p) { return p + (p >> 4); }
__host__ __device__ constexpr int padded_len(int L) { return L + (L >> 4); }

template <typename TT>
__device__ __forceinline__ TT ldg(const TT* p) {
  return __ldg(p);
}

}  // namespace mb
