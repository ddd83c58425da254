// Mixed batches: thousands of independent 1-D transforms of any kind and
// power-of-two length, run by one persistent kernel launched from a CUDA
// graph.
//
// Planning (host).  Jobs are grouped by (kind, direction, length).  Each
// group of transforms whose DFT fits in one CTA is cut into work items of up
// to `cpb` transforms (the tile shape: the items of a length-L group use
// L/16 threads per transform, so a 512-thread CTA holds 512*16/L of them);
// every longer transform (64 K points at most) is one work item by itself.
// Items are ordered by estimated cost, largest first, so the long ones start
// early and the short ones fill the tail.
//
// Execution (device).  Every resident CTA takes the next item from an
// atomic counter until the list is exhausted.  Short items run the same
// load -> Stockham passes -> store code as the axis passes, with each
// transform's own input and output pointers.  Long items (2^14 .. 2^16
// complex points) run by default on one CTA each: two Stockham passes over
// global memory through the CTA's private scratch slice, with the kind's
// element-wise steps fused into them where they need no (k, L-k) pairing
// and run as sweeps of the CTA before or after them otherwise.  With
// MINFFT_B200_MIXED_CLUSTER=1 (where the device can co-schedule the clusters)
// they run instead on clusters of eight CTAs entirely in distributed shared
// memory (mixed_cluster_kernel, run_cluster_big): the clusters take the long
// items first, one per cluster, then every CTA takes short items on its own.
// That form moves each element through HBM once but measured slower.
//
// No CTA ever waits on a CTA outside its own cluster (the queues are a
// single atomicAdd per item; the CTAs of a cluster are co-resident by
// construction), so the kernel cannot deadlock whatever the residency.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdio.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "kernel_registry.h"
#include "line_ops.cuh"
#include "minfft_b200.h"

#define MB_EXPORT extern "C" __attribute__((visibility("default")))

namespace mb {
void set_last_error(int code, const char* msg);
void host_table(int kind, int64_t N, std::vector<cpx>& h);
cudaError_t dev_malloc(void** p, size_t bytes);  // every device allocation of the library (plan.cu)
template <class T>
cudaError_t dev_malloc(T** p, size_t bytes) {
  return dev_malloc(reinterpret_cast<void**>(p), bytes);
}
}  // namespace mb

namespace mb {
namespace mixed {

constexpr int kThreads = 512;
constexpr int kSlots = 18;           // table slots by log2 length, 0 .. 17
constexpr int kSmallMaxLog2L = 13;   // one-CTA DFTs up to 8192 points
constexpr int kBigMaxLog2L = 16;     // two passes over global memory up to 65536
constexpr int kOffsetsBytes = 1024;  // tile offsets of the long-item passes (<= 64 transforms)

struct Job {
  const void* in;
  void* out;
  int op;
  int log2n;
};

// combo < 0: length-1 transforms (a scale or a type change per job)
struct Item {
  int combo;
  int log2L;
  int flags;
  int count;
  int first;  // index into the job order
  int big;
  int op;
  int pad;
};

struct Params {
  const Job* jobs;
  const int* order;
  const Item* items;
  int nitems;
  int nbig;            // items [0, nbig) are long items (cluster form), the rest short ones
  unsigned* counter;   // [0]: next short item, [1]: next long item (cluster form)
  cpx* scratch;
  int64_t scratch_stride;  // complex elements per CTA (two buffers)
  const cpx* tw[kSlots];    // w_L^m, by log2 L
  const cpx* rft[kSlots];   // real-DFT roots, by log2 N
  const cpx* t23[kSlots];   // type-2/3 roots, by log2 N
  const cpx* t4a[kSlots];   // type-4 pre-rotation, by log2 N
  const cpx* t4b[kSlots];   // type-4 post-rotation, by log2 N
  const cpx* sthi[kSlots];  // coarse roots of a long length, by log2 L
  const cpx* stlo[kSlots];  // fine roots of a long length, by log2 L
};

__host__ __device__ constexpr int small_radix(int L) { return L < 16 ? L : 16; }
__host__ __device__ constexpr int log2c(int v) { return v <= 1 ? 0 : 1 + log2c(v / 2); }
__host__ __device__ constexpr int small_cpb(int L) { return kThreads / (L / small_radix(L)); }

// ---------------------------------------------------------------- device
template <int L, class LoadOp, class StoreOp>
__device__ __noinline__ void run_small(const Params& mp, const Item& it, unsigned char* smem) {
  constexpr int R = small_radix(L);
  constexpr int TPT = L / R;
  constexpr int CPB = kThreads / TPT;
  const int c = threadIdx.x / TPT, j = threadIdx.x % TPT;
  const bool active = c < it.count;
  Job job{};
  if (active) job = mp.jobs[mp.order[it.first + c]];
  const int log2N = (it.combo == K_CPLX) ? it.log2L : it.log2L + 1;
  AxisParams p;
  memset(&p, 0, sizeof(p));
  p.in = job.in;
  p.out = job.out;
  p.nbatch = it.count;
  p.d0 = p.d1 = 1;
  p.in_n = 1;
  p.out_k = 1;
  p.tw = mp.tw[it.log2L];
  p.st_ns = 1;
  p.st_div = 1;
  p.cpb = CPB;
  p.flags = it.flags;
  p.lp = tile_pitch(L, R, CPB, 0);
  switch (it.combo) {
    case K_R2C:
      p.t1 = mp.rft[log2N];
      if ((reinterpret_cast<uintptr_t>(job.in) % sizeof(cpx)) == 0) p.flags |= F_VEC;
      break;
    case K_C2R:
      p.t2 = mp.rft[log2N];
      if ((reinterpret_cast<uintptr_t>(job.out) % sizeof(cpx)) == 0) p.flags |= F_VEC;
      break;
    case K_DCT2:
    case K_DCT3:
      p.t1 = mp.t23[log2N];
      p.t2 = mp.rft[log2N];
      break;
    case K_T4:
      p.t1 = mp.t4a[log2N];
      p.t2 = mp.t4b[log2N];
      break;
    default: break;
  }
  Ctx x;
  x.b = c;
  x.b0 = 0;
  x.oin = 0;
  x.oout = 0;
  x.c = c;
  x.j = j;
  x.active = active;
  Tile t{reinterpret_cast<cpx*>(smem + kOffsetsBytes), p.lp};
  TileOffsets to{nullptr, nullptr, it.count};
  cpx v[R];
  LoadOp::template run<L, R>(p, x, t, v);
  run_passes<L, R, 1>(v, j, c, t, p.tw);
  StoreOp::template run<L, R>(p, x, t, to, v);
}

// One Stockham pass over global memory of a long transform of length 2^LG,
// sub-DFTs of length RP, span NS (1 or the length of the first pass).
// Ld / St: the load and store stages (complex by default; the fused type-2
// permutation and type-4 pre-rotation in the first pass, the fused type-3
// de-interleave and type-4 post-rotation in the last, with the line's real
// length kn and direct root tables t1, t2).
template <int LG, int RP, int NS, class Ld = LoadCplx, class St = StoreCplx>
__device__ __forceinline__ void big_pass(const Params& mp, const void* src, void* dst, int flags,
                                         unsigned char* smem, int64_t kn = 0, const cpx* t1 = nullptr,
                                         const cpx* t2 = nullptr) {
  constexpr int Lc = 1 << LG;
  constexpr int R = 16;
  constexpr int TPT = RP / R;
  constexpr int CPB = kThreads / TPT;
  constexpr int NJ = Lc / RP;
  static_assert(CPB * 2 * sizeof(int64_t) <= kOffsetsBytes, "offsets region");
  AxisParams p;
  memset(&p, 0, sizeof(p));
  p.in = src;
  p.out = dst;
  p.nbatch = NJ;
  p.d0 = NS;
  p.d1 = Lc / (NS * RP);
  p.is0 = 1;
  p.is1 = NS;
  p.is2 = Lc;
  p.in_n = Lc / RP;
  p.os0 = 1;
  p.os1 = NS * RP;
  p.os2 = Lc;
  p.out_k = NS;
  p.st_ns = NS;
  p.st_div = 1;
  p.st_shift = 0;
  p.st_lobits = (LG + 1) / 2;
  p.st_hi = mp.sthi[LG];
  p.st_lo = mp.stlo[LG];
  p.tw = mp.tw[log2c(RP)];
  p.cpb = CPB;
  p.colmode = 1;
  p.flags = flags | (NS == 1 ? F_STAGE_ROWS : 0);
  p.lp = tile_pitch(RP, R, CPB, 1);
  p.kn = kn;
  p.t1 = t1;
  p.t2 = t2;
  int64_t* offs = reinterpret_cast<int64_t*>(smem);
  Tile t{reinterpret_cast<cpx*>(smem + kOffsetsBytes), p.lp};
  const int c = threadIdx.x % CPB, j = threadIdx.x / CPB;
  for (int round = 0; round * CPB < NJ; ++round) {
    const int64_t base = int64_t(round) * CPB;
    if (threadIdx.x < CPB) {
      int64_t b0, oi, oo;
      batch_offsets(p, base + threadIdx.x < NJ ? base + threadIdx.x : 0, b0, oi, oo);
      offs[threadIdx.x] = oi;
      offs[CPB + threadIdx.x] = oo;
    }
    __syncthreads();
    const int left = int(NJ - base);
    TileOffsets to{offs, offs + CPB, left < CPB ? left : CPB};
    Ctx x;
    x.c = c;
    x.j = j;
    x.b = base + c;
    x.active = x.b < NJ;
    x.b0 = umod(x.b, p.d0);
    x.oin = offs[c];
    x.oout = offs[CPB + c];
    cpx v[R];
    Ld::template run<RP, R>(p, x, t, v);
    run_passes<RP, R, 1>(v, j, c, t, p.tw);
    St::template run<RP, R>(p, x, t, to, v);
    __syncthreads();
  }
}

// A line step over one long item by the whole CTA: each thread takes items
// tid, tid + blockDim.x, ... and issues the loads of kBatch of them before
// computing and storing any, so the CTA keeps several loads per thread in
// flight instead of one (this walk is a single CTA's, not a grid's).
template <class Op>
__device__ __forceinline__ void cta_line(const LineParams& lp) {
  constexpr int kBatch = sizeof(typename Op::In) <= 3 * sizeof(cpx) ? 4 : 2;
  const int64_t total = Op::count(lp);
  const int64_t step = blockDim.x;
  // one line (outer = inner = 1): item e is point e of the line
  int64_t e = threadIdx.x;
  for (; e + (kBatch - 1) * step < total; e += kBatch * step) {
    typename Op::In v[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) v[u] = Op::load_at(lp, ItemIdx{0, e + u * step, 0});
#pragma unroll
    for (int u = 0; u < kBatch; ++u) Op::finish_at(lp, ItemIdx{0, e + u * step, 0}, v[u]);
  }
  for (; e < total; e += step) Op::finish_at(lp, ItemIdx{0, e, 0}, Op::load_at(lp, ItemIdx{0, e, 0}));
}

template <int LG>
__device__ __noinline__ void run_big(const Params& mp, const Item& it, unsigned char* smem) {
  constexpr int Lc = 1 << LG;
  constexpr int B1 = (LG + 1) / 2, B2 = LG - B1;
  constexpr int R1 = 1 << B1, R2 = 1 << B2;
  const Job job = mp.jobs[mp.order[it.first]];
  cpx* S1 = mp.scratch + int64_t(blockIdx.x) * mp.scratch_stride;
  cpx* S2 = S1 + mp.scratch_stride / 2;
  const int log2N = (it.combo == K_CPLX) ? LG : LG + 1;
  LineParams lp;
  memset(&lp, 0, sizeof(lp));
  lp.outer = 1;
  lp.inner = 1;
  lp.L = Lc;
  lp.in_sn = 1;
  lp.out_sn = 1;
  lp.flags = it.flags;
  const int64_t N = int64_t(1) << log2N;  // the real length (real kinds)
  const cpx* src = static_cast<const cpx*>(job.in);
  // element-wise pre-processing into S1 where it needs the pair (k, L-k)
  // (the type-2 permutation and type-4 pre-rotation are fused into the
  // first pass instead)
  if (it.combo == K_C2R || it.combo == K_DCT3) {
    lp.in = job.in;
    lp.out = S1;
    if (it.combo == K_C2R) {
      lp.t2 = mp.rft[log2N];
      cta_line<Op_c2r_pack>(lp);
    } else {
      lp.t1 = mp.t23[log2N];
      lp.t2 = mp.rft[log2N];
      cta_line<Op_dct3_pack>(lp);
    }
    src = S1;
    __syncthreads();
  }
  cpx* mid = (src == S1) ? S2 : S1;
  const bool inv_cplx = (it.combo == K_CPLX) && (it.flags & F_CONJ_IN);
  const int kf = it.flags & F_DST;
  if (it.combo == K_DCT2)
    big_pass<LG, R1, 1, LoadDCT2Chain>(mp, job.in, mid, kf, smem, N);
  else if (it.combo == K_T4)
    big_pass<LG, R1, 1, LoadT4Direct>(mp, job.in, mid, kf, smem, N, mp.t4a[log2N]);
  else
    big_pass<LG, R1, 1>(mp, src, mid, inv_cplx ? F_CONJ_IN : 0, smem);
  __syncthreads();
  // the last pass writes the output itself for the complex DFT, the
  // inverse real DFT and the fused type-3 de-interleave and type-4
  // post-rotation; the real DFT and the DCT-2 unpack the pairs afterwards
  const bool pairs = it.combo == K_R2C || it.combo == K_DCT2;
  cpx* fin = pairs ? (mid == S1 ? S2 : S1) : static_cast<cpx*>(job.out);
  const bool conj_out = inv_cplx || it.combo == K_C2R;
  if (it.combo == K_DCT3)
    big_pass<LG, R2, R1, LoadCplx, StoreDCT3Chain>(mp, mid, job.out, kf, smem, N);
  else if (it.combo == K_T4)
    big_pass<LG, R2, R1, LoadCplx, StoreT4Direct>(mp, mid, job.out, kf, smem, N, nullptr, mp.t4b[log2N]);
  else
    big_pass<LG, R2, R1>(mp, mid, fin, conj_out ? F_CONJ_OUT : 0, smem);
  __syncthreads();
  if (pairs) {
    lp.in = fin;
    lp.out = job.out;
    if (it.combo == K_R2C) {
      lp.t1 = mp.rft[log2N];
      cta_line<Op_r2c_unpack>(lp);
    } else {
      lp.t1 = mp.t23[log2N];
      lp.t2 = mp.rft[log2N];
      cta_line<Op_dct2_post>(lp);
    }
  }
}

// length-1 transforms: y = 2x (type 2), x (type 3), sqrt(2) x (type 4),
// (x, 0) (real DFT), Re z (inverse real DFT), z (complex DFT)
__device__ __noinline__ void run_unit(const Params& mp, const Item& it) {
  for (int c = threadIdx.x; c < it.count; c += blockDim.x) {
    const Job job = mp.jobs[mp.order[it.first + c]];
    switch (job.op) {
      case MINFFT_B200_DFT:
      case MINFFT_B200_INVDFT: *static_cast<cpx*>(job.out) = *static_cast<const cpx*>(job.in); break;
      case MINFFT_B200_REALDFT: *static_cast<cpx*>(job.out) = cmk(*static_cast<const real*>(job.in), real(0)); break;
      case MINFFT_B200_INVREALDFT: *static_cast<real*>(job.out) = static_cast<const cpx*>(job.in)->x; break;
      case MINFFT_B200_DCT2:
      case MINFFT_B200_DST2: *static_cast<real*>(job.out) = 2 * *static_cast<const real*>(job.in); break;
      case MINFFT_B200_DCT3:
      case MINFFT_B200_DST3: *static_cast<real*>(job.out) = *static_cast<const real*>(job.in); break;
      default:
        *static_cast<real*>(job.out) = real(1.414213562373095048801688724209698079) * *static_cast<const real*>(job.in);
        break;
    }
  }
}

template <class Ld, class St>
__device__ __forceinline__ void run_small_any(const Params& mp, const Item& it, unsigned char* smem) {
  switch (it.log2L) {
    case 0: run_small<1, Ld, St>(mp, it, smem); break;
    case 1: run_small<2, Ld, St>(mp, it, smem); break;
    case 2: run_small<4, Ld, St>(mp, it, smem); break;
    case 3: run_small<8, Ld, St>(mp, it, smem); break;
    case 4: run_small<16, Ld, St>(mp, it, smem); break;
    case 5: run_small<32, Ld, St>(mp, it, smem); break;
    case 6: run_small<64, Ld, St>(mp, it, smem); break;
    case 7: run_small<128, Ld, St>(mp, it, smem); break;
    case 8: run_small<256, Ld, St>(mp, it, smem); break;
    case 9: run_small<512, Ld, St>(mp, it, smem); break;
    case 10: run_small<1024, Ld, St>(mp, it, smem); break;
    case 11: run_small<2048, Ld, St>(mp, it, smem); break;
    case 12: run_small<4096, Ld, St>(mp, it, smem); break;
    case 13: run_small<8192, Ld, St>(mp, it, smem); break;
    default: break;
  }
}

__global__ void __launch_bounds__(kThreads, MinBlocks<16>::value) mixed_kernel(const __grid_constant__ Params mp) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = int(atomicAdd(mp.counter, 1u));
    __syncthreads();
    const int idx = s_item;
    __syncthreads();
    if (idx >= mp.nitems) break;
    const Item it = mp.items[idx];
    if (it.big) {
      switch (it.log2L) {
        case 14: run_big<14>(mp, it, smem); break;
        case 15: run_big<15>(mp, it, smem); break;
        case 16: run_big<16>(mp, it, smem); break;
        default: break;
      }
    } else if (it.combo < 0) {
      run_unit(mp, it);
    } else {
      switch (it.combo) {
        case K_CPLX: run_small_any<LoadCplx, StoreCplx>(mp, it, smem); break;
        case K_R2C: run_small_any<LoadR2C, StoreR2C>(mp, it, smem); break;
        case K_C2R: run_small_any<LoadC2R, StoreC2R>(mp, it, smem); break;
        case K_DCT2: run_small_any<LoadDCT2, StoreDCT2>(mp, it, smem); break;
        case K_DCT3: run_small_any<LoadDCT3, StoreDCT3>(mp, it, smem); break;
        default: run_small_any<LoadT4, StoreT4>(mp, it, smem); break;
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------- long items on a cluster
// A long item (L = 2^14 .. 2^16 complex points) is computed by a cluster of
// kCluster CTAs entirely in their shared memory (the four-step split
// n = 256*n1 + n2, k = k1 + N1*k2, N1 = L/256): CTA r holds the 32 columns
// n2 = 32r .. 32r+31 of all N1 rows, computes their length-N1 DFTs over n1
// (with the kind's pre-processing fused into the global loads) and the
// twiddles w_L^(n2 k1); after a cluster barrier it gathers, through
// distributed shared memory, rows k1 = r*N1/8 .. (r+1)*N1/8-1 from all eight
// CTAs and computes their length-256 DFTs over n2, then applies the kind's
// post-processing (reading the partner outputs z_{L-k} of the real DFT and
// DCT-2 from the CTA that holds them) and stores.  Each element is read from
// and written to global memory once.
constexpr int kCluster = 8;
constexpr int kN2 = 256;
constexpr int kColsPerCta = kN2 / kCluster;  // 32

// Element n (< L) of the complex sequence whose length-L DFT a long item of
// kind it.combo needs: the pre-processing steps of line_ops.cuh, per element.
__device__ __forceinline__ cpx big_pre(const Params& mp, const Item& it, const Job& job, int LG, int64_t n) {
  const int64_t L = int64_t(1) << LG, N = 2 * L;
  const int log2N = LG + 1;
  const bool dst = (it.flags & F_DST) != 0;
  switch (it.combo) {
    case K_CPLX: {
      cpx x = static_cast<const cpx*>(job.in)[n];
      if (it.flags & F_CONJ_IN) x.y = -x.y;
      return x;
    }
    case K_R2C:
      return static_cast<const cpx*>(job.in)[n];  // the real row as pairs (aligned: checked at planning)
    case K_DCT2: {
      const real* in = static_cast<const real*>(job.in);
      const real sg = dst ? real(-1) : real(1);
      const int64_t i0 = 2 * n, i1 = 2 * n + 1;
      const real a = i0 < L ? in[2 * i0] : sg * in[2 * N - 1 - 2 * i0];
      const real b = i1 < L ? in[2 * i1] : sg * in[2 * N - 1 - 2 * i1];
      return cmk(a, b);
    }
    case K_T4: {
      const real* in = static_cast<const real*>(job.in);
      const real a = in[2 * n], b = in[N - 1 - 2 * n];
      const cpx w = ldg(mp.t4a[log2N] + n);
      if (!dst) return cmul(w, cmk(a, b));
      const cpx q = cmul(w, cmk(a, -b));
      return cmk(-q.x, -q.y);
    }
    default: {  // K_C2R and K_DCT3: packing of the pair (n, L-n), conjugated
      const cpx* zin = static_cast<const cpx*>(job.in);
      const real* rin = static_cast<const real*>(job.in);
      auto z = [&](int64_t k) -> cpx {
        if (it.combo == K_C2R) return zin[k];
        auto rd = [&](int i) { return rin[i]; };
        return LoadDCT3::zval_r(rd, int(k), int(L), dst, mp.t23[log2N]);
      };
      const cpx* rft = mp.rft[log2N];
      if (n == 0) {
        const cpx z0 = z(0), z1 = z(L);
        return cmk(z0.x + z1.x, -(z0.x - z1.x));
      }
      if (2 * n == L) {
        const cpx z0 = z(n);
        return cmk(2 * z0.x, 2 * z0.y);
      }
      cpx ta, tb;
      if (2 * n < L) {
        pack_pair(z(n), z(L - n), ldg(rft + n), ta, tb);
        return cconj(ta);
      }
      pack_pair(z(L - n), z(n), ldg(rft + (L - n)), ta, tb);
      return cconj(tb);
    }
  }
}

// Outputs of a long item for DFT output z_k of a kind without pairing.
__device__ __forceinline__ void big_post_single(const Params& mp, const Item& it, const Job& job, int LG, int64_t k,
                                                cpx zk) {
  const int64_t L = int64_t(1) << LG, N = 2 * L;
  const int log2N = LG + 1;
  const bool dst = (it.flags & F_DST) != 0;
  switch (it.combo) {
    case K_CPLX:
      if (it.flags & F_CONJ_OUT) zk.y = -zk.y;
      static_cast<cpx*>(job.out)[k] = zk;
      break;
    case K_C2R:
      static_cast<cpx*>(job.out)[k] = cconj(zk);  // the real output as pairs (aligned: checked at planning)
      break;
    case K_DCT3: {
      real* out = static_cast<real*>(job.out);
      const cpx w = cconj(zk);
      const int64_t i0 = 2 * k, i1 = 2 * k + 1;
      const real a = (dst && i0 >= L) ? -w.x : w.x;
      const real b = (dst && i1 >= L) ? -w.y : w.y;
      out[i0 < L ? 2 * i0 : 2 * N - 1 - 2 * i0] = a;
      out[i1 < L ? 2 * i1 : 2 * N - 1 - 2 * i1] = b;
      break;
    }
    default: {  // K_T4
      real* out = static_cast<real*>(job.out);
      const cpx* t4b = mp.t4b[log2N];
      const cpx a = cmul(ldg(t4b + 2 * k), zk);
      const cpx b = cmul(ldg(t4b + (N - 1 - 2 * k)), cconj(zk));
      out[2 * k] = 2 * (dst ? a.y : a.x);
      out[N - 1 - 2 * k] = 2 * (dst ? b.y : b.x);
      break;
    }
  }
}

// Outputs of the pairing kinds (real DFT, DCT-2) from z_k and z_{L-k}, for
// 0 <= k <= L/2 (k = 0 also covers X_L; zb is unused there and at k = L/2).
__device__ __forceinline__ void big_post_pair(const Params& mp, const Item& it, const Job& job, int LG, int64_t k,
                                              cpx za, cpx zb) {
  const int64_t L = int64_t(1) << LG, N = 2 * L;
  const int log2N = LG + 1;
  const cpx* rft = mp.rft[log2N];
  if (it.combo == K_R2C) {
    cpx* out = static_cast<cpx*>(job.out);
    if (k == 0) {
      out[0] = cmk(za.x + za.y, real(0));
      out[L] = cmk(za.x - za.y, real(0));
    } else if (2 * k == L) {
      out[k] = cconj(za);
    } else {
      cpx xa, xb;
      unpack_pair(za, zb, ldg(rft + k), xa, xb);
      out[k] = xa;
      out[L - k] = xb;
    }
    return;
  }
  real* out = static_cast<real*>(job.out);
  const bool dst = (it.flags & F_DST) != 0;
  const cpx* t23 = mp.t23[log2N];
  if (k == 0) {
    const real r2 = real(1.414213562373095048801688724209698079);
    out[dst ? N - 1 : 0] = 2 * (za.x + za.y);
    out[dst ? L - 1 : L] = r2 * (za.x - za.y);
  } else if (2 * k == L) {
    StoreDCT2::emit(out, 1, int(k), int(N), dst, cconj(za), ldg(t23 + k));
  } else {
    cpx xa, xb;
    unpack_pair2(za, zb, ldg(rft + k), xa, xb);
    StoreDCT2::emit2(out, 1, int(k), int(N), dst, xa, ldg(t23 + k));
    StoreDCT2::emit2(out, 1, int(L - k), int(N), dst, xb, ldg(t23 + (L - k)));
  }
}

// Row k1 of step 2 held by CTA `rank` at local index kk < K1.  The pairing
// kinds (real DFT, DCT-2) need z_k beside z_{L-k}: with k = k1 + N1*k2, the
// partner sits in row N1 - k1 (rows 0 and N1/2 are their own partners), so
// their CTAs take the rows in mirrored pairs (base + p, N1 - base - p),
// base = rank*K1/2 (CTA 0: rows 0 and N1/2, then its pairs) and every partner
// is local.  The other kinds take K1 consecutive rows, so that their stores
// run along k1.
template <int N1, int K1>
__device__ __forceinline__ int step2_row(bool pairs, int rank, int kk) {
  if (!pairs) return rank * K1 + kk;
  const int p = kk >> 1, base = rank * (K1 / 2);
  if (rank == 0 && p == 0) return (kk & 1) ? N1 / 2 : 0;
  return (kk & 1) ? N1 - (base + p) : base + p;
}

// One long item on the cluster.  Two cluster barriers: after step 1 (every
// CTA's columns are in its tile) and after the gather of step 2 (no CTA reads
// another's tile any more, so each may overwrite its own, for step 2's
// exchanges and for the next item).  `next` is the index of the cluster's next
// item, which cluster rank 0 has written to its slot before this item began;
// it is read once the first barrier has made it visible.
template <int LG>
__device__ __noinline__ int run_cluster_big(const Params& mp, const Item& it, unsigned char* smem, const int* next) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  constexpr int L = 1 << LG;
  constexpr int N1 = L / kN2;                 // 64, 128, 256
  constexpr int TPT1 = kThreads / kColsPerCta;  // 16 threads per column in step 1
  constexpr int R1 = N1 / TPT1;               // 4, 8, 16
  constexpr int K1 = N1 / kCluster;           // rows k1 per CTA in step 2: 8, 16, 32
  constexpr int TPT2 = kThreads / K1;         // 64, 32, 16
  constexpr int R2 = kN2 / TPT2;              // 4, 8, 16
  static_assert(R1 >= 4 && R2 >= 4 && TPT1 * kColsPerCta == kThreads && K1 >= 4, "shape");
  const int rank = int(cl.block_rank());
  const Job job = mp.jobs[mp.order[it.first]];
  cpx* tile = reinterpret_cast<cpx*>(smem + kOffsetsBytes);
  const int lp1 = tile_pitch(N1, R1, kColsPerCta, 1);
  const int lp2 = tile_pitch(kN2, R2, K1, 1);
  const int lobits = (LG + 1) / 2;
  const int64_t lomask = (int64_t(1) << lobits) - 1;
  const bool pairs = it.combo == K_R2C || it.combo == K_DCT2;

  // ---- step 1: DFTs over n1 of the columns n2 = 32*rank + c
  {
    const int c = threadIdx.x % kColsPerCta, j = threadIdx.x / kColsPerCta;
    const int n2 = rank * kColsPerCta + c;
    Tile t{tile, lp1};
    cpx v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) v[r] = big_pre(mp, it, job, LG, int64_t(kN2) * (j + r * TPT1) + n2);
    run_passes<N1, R1, 1>(v, j, c, t, mp.tw[log2c(N1)]);
    // v[r] = output k1 = j + r*TPT1; twiddle w_L^(n2 k1)
#pragma unroll
    for (int r = 0; r < R1; ++r) {
      const int64_t g = int64_t(n2) * (j + r * TPT1);
      v[r] = cmul(v[r], cmul(ldg(mp.sthi[LG] + (g >> lobits)), ldg(mp.stlo[LG] + (g & lomask))));
    }
    __syncthreads();
    scatter_natural<N1, R1>(v, j, c, t);
  }
  cl.sync();
  const int nxt = *cl.map_shared_rank(next, 0);

  // ---- step 2: DFTs over n2 of the CTA's K1 rows
  const int kk = threadIdx.x % K1, j2 = threadIdx.x / K1;
  const int k1 = step2_row<N1, K1>(pairs, rank, kk);
  cpx v[R2];
#pragma unroll
  for (int r = 0; r < R2; ++r) {
    const int n2 = j2 + r * TPT2;
    const cpx* src = cl.map_shared_rank(tile, n2 / kColsPerCta);
    v[r] = src[(n2 % kColsPerCta) * lp1 + pad16(k1)];
  }
  cl.sync();  // every remote read of this CTA's tile is done
  Tile t2{tile, lp2};
  run_passes<kN2, R2, 1>(v, j2, kk, t2, mp.tw[log2c(kN2)]);
  // v[r] = z_k, k = k1 + N1*k2, k2 = j2 + r*TPT2
  if (pairs) {
    __syncthreads();
    scatter_natural<kN2, R2>(v, j2, kk, t2);
    __syncthreads();
    // partner row: the other member of the pair (rows 0 and N1/2: the row itself)
    const int pkk = (rank == 0 && kk < 2) ? kk : (kk ^ 1);
#pragma unroll
    for (int r = 0; r < R2; ++r) {
      const int k2 = j2 + r * TPT2;
      const int64_t k = int64_t(k1) + int64_t(N1) * k2;
      if (2 * k > L) continue;
      cpx zb = czero();
      if (k != 0 && 2 * k != L) {
        const int pk2 = k1 == 0 ? kN2 - k2 : kN2 - 1 - k2;
        zb = tile[pkk * lp2 + pad16(pk2)];
      }
      big_post_pair(mp, it, job, LG, k, v[r], zb);
    }
  } else {
#pragma unroll
    for (int r = 0; r < R2; ++r) big_post_single(mp, it, job, LG, int64_t(k1) + int64_t(N1) * (j2 + r * TPT2), v[r]);
  }
  __syncthreads();  // the local tile may be reused
  return nxt;
}

// Shared memory a CTA needs for its part of a long item.
__host__ __device__ inline size_t cluster_big_smem() {
  size_t m = 0;
  for (int lg = 14; lg <= kBigMaxLog2L; ++lg) {
    const int N1 = (1 << lg) / kN2, R1 = N1 / (kThreads / kColsPerCta);
    const int K1 = N1 / kCluster, R2 = kN2 / (kThreads / K1);
    const size_t a = size_t(kColsPerCta) * tile_pitch(N1, R1, kColsPerCta, 1) * sizeof(cpx);
    const size_t b = size_t(K1) * tile_pitch(kN2, R2, K1, 1) * sizeof(cpx);
    m = m > a ? m : a;
    m = m > b ? m : b;
  }
  return kOffsetsBytes + 16 * ((m + 15) / 16);
}

// The persistent kernel in cluster form: long items first, each on a whole
// cluster (cluster rank 0 takes the next one from counter[1] and the others
// read its index through distributed shared memory), then every CTA takes
// short items from counter[0] on its own.
__global__ void __launch_bounds__(kThreads, MinBlocks<16>::value) mixed_cluster_kernel(const __grid_constant__ Params mp) {
  namespace cg = cooperative_groups;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_item;
  __shared__ int s_next[2];  // cluster rank 0: the cluster's next long item, by item parity
  cg::cluster_group cl = cg::this_cluster();
  const bool lead = cl.block_rank() == 0 && threadIdx.x == 0;
  if (lead) s_next[0] = int(atomicAdd(mp.counter + 1, 1u));
  cl.sync();
  int idx = *cl.map_shared_rank(&s_next[0], 0);
  for (int n = 0; idx < mp.nbig; ++n) {
    // the index after this one, read by the cluster after this item's first
    // barrier (the slot it replaces was read during the previous item)
    if (lead) s_next[(n + 1) & 1] = int(atomicAdd(mp.counter + 1, 1u));
    const Item it = mp.items[idx];
    switch (it.log2L) {
      case 14: idx = run_cluster_big<14>(mp, it, smem, &s_next[(n + 1) & 1]); break;
      case 15: idx = run_cluster_big<15>(mp, it, smem, &s_next[(n + 1) & 1]); break;
      default: idx = run_cluster_big<16>(mp, it, smem, &s_next[(n + 1) & 1]); break;
    }
  }
  cl.sync();  // rank 0's slot has been read by all before anyone moves on
  for (;;) {
    if (threadIdx.x == 0) s_item = mp.nbig + int(atomicAdd(mp.counter, 1u));
    __syncthreads();
    const int idx = s_item;
    __syncthreads();
    if (idx >= mp.nitems) break;
    const Item it = mp.items[idx];
    if (it.combo < 0) {
      run_unit(mp, it);
    } else {
      switch (it.combo) {
        case K_CPLX: run_small_any<LoadCplx, StoreCplx>(mp, it, smem); break;
        case K_R2C: run_small_any<LoadR2C, StoreR2C>(mp, it, smem); break;
        case K_C2R: run_small_any<LoadC2R, StoreC2R>(mp, it, smem); break;
        case K_DCT2: run_small_any<LoadDCT2, StoreDCT2>(mp, it, smem); break;
        case K_DCT3: run_small_any<LoadDCT3, StoreDCT3>(mp, it, smem); break;
        default: run_small_any<LoadT4, StoreT4>(mp, it, smem); break;
      }
    }
    __syncthreads();
  }
  cl.sync();  // no CTA leaves while another may still read its shared memory
}

// shared memory of the kernel: offsets + the largest tile of any item
size_t kernel_smem() {
  size_t m = 0;
  for (int lg = 0; lg <= kSmallMaxLog2L; ++lg) {
    const int L = 1 << lg;
    const int cpb = small_cpb(L);
    m = std::max(m, size_t(cpb) * tile_pitch(L, small_radix(L), cpb, 0) * sizeof(cpx));
  }
  for (int rp : {64, 128, 256}) {
    const int cpb = kThreads / (rp / 16);
    m = std::max(m, size_t(cpb) * tile_pitch(rp, 16, cpb, 1) * sizeof(cpx));
  }
  return kOffsetsBytes + 16 * ((m + 15) / 16);
}

}  // namespace mixed
}  // namespace mb

// ==================================================================== host
using mb::cpx;
using mb::real;
using namespace mb::mixed;

struct minfft_b200_mixed {
  int device = 0;
  int count = 0;
  std::vector<Job> jobs;
  std::vector<int> order;
  std::vector<Item> items;
  Params params;
  void* d_jobs = nullptr;
  void* d_order = nullptr;
  void* d_items = nullptr;
  unsigned* d_counter = nullptr;
  cpx* d_scratch = nullptr;
  std::vector<void*> tables;
  int grid = 0;
  int per_sm = 1;
  size_t smem = 0;
  int split = 1;  // jobs per short item = slots / split
  bool cluster = false;  // long items on clusters (mixed_cluster_kernel)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

bool ok(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  char buf[256];
  snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
  mb::set_last_error(e == cudaErrorMemoryAllocation ? MINFFT_B200_ENOMEM : MINFFT_B200_ECUDA, buf);
  return false;
}

int fail(int code, const char* msg) {
  mb::set_last_error(code, msg);
  return code;
}

int ilog2i(int64_t v) {
  int r = 0;
  while ((int64_t(1) << r) < v) ++r;
  return r;
}

int combo_of(int op) {
  switch (op) {
    case MINFFT_B200_DFT:
    case MINFFT_B200_INVDFT: return mb::K_CPLX;
    case MINFFT_B200_REALDFT: return mb::K_R2C;
    case MINFFT_B200_INVREALDFT: return mb::K_C2R;
    case MINFFT_B200_DCT2:
    case MINFFT_B200_DST2: return mb::K_DCT2;
    case MINFFT_B200_DCT3:
    case MINFFT_B200_DST3: return mb::K_DCT3;
    default: return mb::K_T4;
  }
}

int flags_of(int op) {
  if (op == MINFFT_B200_INVDFT) return mb::F_CONJ_IN | mb::F_CONJ_OUT;
  if (op == MINFFT_B200_DST2 || op == MINFFT_B200_DST3 || op == MINFFT_B200_DST4) return mb::F_DST;
  return 0;
}

const cpx* upload(minfft_b200_mixed* m, int kind, int64_t N) {
  std::vector<cpx> h;
  mb::host_table(kind, N, h);
  void* d = nullptr;
  if (!ok(mb::dev_malloc(&d, h.size() * sizeof(cpx)), "cudaMalloc(table)")) return nullptr;
  m->tables.push_back(d);
  if (!ok(cudaMemcpy(d, h.data(), h.size() * sizeof(cpx), cudaMemcpyHostToDevice), "cudaMemcpy(table)"))
    return nullptr;
  return static_cast<const cpx*>(d);
}

void release_graph(minfft_b200_mixed* m) {
  if (m->exec) cudaGraphExecDestroy(m->exec);
  if (m->graph) cudaGraphDestroy(m->graph);
  m->exec = nullptr;
  m->graph = nullptr;
}

// Cut the job groups into items (short groups: slots/split jobs per item),
// order them by cost, upload, and capture counter reset + kernel in a graph.
bool build_items(minfft_b200_mixed* m) {
  std::map<std::tuple<int, int, int, int>, std::vector<int>> groups;  // (big, combo, flags, log2L) -> jobs
  for (int i = 0; i < m->count; ++i) {
    const Job& j = m->jobs[i];
    const int combo = combo_of(j.op);
    const int64_t n = int64_t(1) << j.log2n;
    if (n == 1) {
      groups[std::make_tuple(0, -1, 0, 0)].push_back(i);
      continue;
    }
    const int lgL = combo == mb::K_CPLX ? j.log2n : j.log2n - 1;
    groups[std::make_tuple(lgL > kSmallMaxLog2L ? 1 : 0, combo, flags_of(j.op), lgL)].push_back(i);
  }
  std::vector<std::pair<double, Item>> its;
  m->order.clear();
  for (auto& g : groups) {
    const int big = std::get<0>(g.first), combo = std::get<1>(g.first), flags = std::get<2>(g.first),
              lgL = std::get<3>(g.first);
    const std::vector<int>& js = g.second;
    const int L = 1 << lgL;
    int per = big ? 1 : (combo < 0 ? kThreads : std::max(1, small_cpb(L) / m->split));
    for (size_t s = 0; s < js.size(); s += per) {
      Item it{};
      it.combo = combo;
      it.log2L = lgL;
      it.flags = flags;
      it.count = int(std::min<size_t>(per, js.size() - s));
      it.first = int(m->order.size());
      it.big = big;
      it.op = m->jobs[js[s]].op;
      for (int k = 0; k < it.count; ++k) m->order.push_back(js[s + k]);
      // cost: points processed (x2 passes and pre/post for the long ones)
      const double cost = double(L) * std::max(1, lgL) * (big ? 3.0 : 1.0) * (big ? 1 : it.count);
      its.push_back(std::make_pair(cost, it));
    }
  }
  std::stable_sort(its.begin(), its.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
  // long items first (the cluster form takes them from their own queue)
  std::stable_partition(its.begin(), its.end(), [](const auto& a) { return a.second.big != 0; });
  m->items.clear();
  int nbig = 0;
  for (auto& p : its) {
    m->items.push_back(p.second);
    nbig += p.second.big ? 1 : 0;
  }
  if (m->d_order) cudaFree(m->d_order);
  if (m->d_items) cudaFree(m->d_items);
  m->d_order = m->d_items = nullptr;
  if (!ok(mb::dev_malloc(&m->d_order, std::max<size_t>(1, m->order.size()) * sizeof(int)), "cudaMalloc(order)") ||
      !ok(mb::dev_malloc(&m->d_items, std::max<size_t>(1, m->items.size()) * sizeof(Item)), "cudaMalloc(items)"))
    return false;
  if (!m->order.empty() &&
      !ok(cudaMemcpy(m->d_order, m->order.data(), m->order.size() * sizeof(int), cudaMemcpyHostToDevice),
          "cudaMemcpy(order)"))
    return false;
  if (!m->items.empty() &&
      !ok(cudaMemcpy(m->d_items, m->items.data(), m->items.size() * sizeof(Item), cudaMemcpyHostToDevice),
          "cudaMemcpy(items)"))
    return false;
  m->params.order = static_cast<const int*>(m->d_order);
  m->params.items = static_cast<const Item*>(m->d_items);
  m->params.nitems = int(m->items.size());
  m->params.nbig = m->cluster ? nbig : 0;
  // graph: reset the queue counter, run the persistent kernel
  release_graph(m);
  cudaStream_t cs;
  if (!ok(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "cudaStreamCreate")) return false;
  bool good = ok(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
  if (good) {
    cudaMemsetAsync(m->d_counter, 0, 2 * sizeof(unsigned), cs);
    void* args[1] = {&m->params};
    if (m->cluster) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(m->grid);
      cfg.blockDim = dim3(kThreads);
      cfg.dynamicSmemBytes = m->smem;
      cfg.stream = cs;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = kCluster;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      cudaLaunchKernelExC(&cfg, (const void*)mixed_cluster_kernel, args);
    } else {
      cudaLaunchKernel((const void*)mixed_kernel, dim3(m->grid), dim3(kThreads), args, m->smem, cs);
    }
    good = ok(cudaStreamEndCapture(cs, &m->graph), "cudaStreamEndCapture");
  }
  if (good) good = ok(cudaGraphInstantiate(&m->exec, m->graph, 0), "cudaGraphInstantiate");
  cudaStreamDestroy(cs);
  return good;
}

}  // namespace

MB_EXPORT void minfft_b200_mixed_free(minfft_b200_mixed* m) {
  if (!m) return;
  release_graph(m);
  for (void* t : m->tables) cudaFree(t);
  cudaFree(m->d_jobs);
  cudaFree(m->d_order);
  cudaFree(m->d_items);
  cudaFree(m->d_counter);
  cudaFree(m->d_scratch);
  delete m;
}

MB_EXPORT minfft_b200_mixed* minfft_b200_mixed_plan(int count, const minfft_b200_job* jobs) {
  if (count < 1 || !jobs) {
    fail(MINFFT_B200_EINVAL, "mixed plan: need at least one job");
    return nullptr;
  }
  minfft_b200_mixed* m = new (std::nothrow) minfft_b200_mixed();
  if (!m) {
    fail(MINFFT_B200_ENOMEM, "mixed plan: host allocation failed");
    return nullptr;
  }
  m->count = count;
  m->jobs.resize(count);
  int max_big = 0;
  std::vector<int> need_tw(kSlots, 0), need_n(kSlots, 0), need_st(kSlots, 0);
  std::vector<int> need_kind(kSlots * mb::K_COUNT, 0);
  for (int i = 0; i < count; ++i) {
    const minfft_b200_job& j = jobs[i];
    const int64_t n = j.n;
    if (j.op < MINFFT_B200_DFT || j.op > MINFFT_B200_DST4 || n < 1 || (n & (n - 1)) || !j.in || !j.out) {
      char buf[160];
      snprintf(buf, sizeof(buf), "mixed plan: job %d has a bad transform code, length or pointer", i);
      fail(MINFFT_B200_EINVAL, buf);
      minfft_b200_mixed_free(m);
      return nullptr;
    }
    const int combo = combo_of(j.op);
    const int lgn = ilog2i(n);
    const int lgL = (combo == mb::K_CPLX) ? lgn : std::max(lgn - 1, 0);
    if (lgL > kBigMaxLog2L) {
      fail(MINFFT_B200_EINVAL, "mixed plan: lengths above 65536 complex points (131072 real) are not supported");
      minfft_b200_mixed_free(m);
      return nullptr;
    }
    // complex arrays are accessed as aligned pairs; so are the real arrays a
    // long real DFT reads (or a long inverse writes) as complex values
    const bool cin = combo == mb::K_CPLX || combo == mb::K_C2R || (combo == mb::K_R2C && lgL > kSmallMaxLog2L);
    const bool cout = combo == mb::K_CPLX || combo == mb::K_R2C || (combo == mb::K_C2R && lgL > kSmallMaxLog2L);
    if ((cin && reinterpret_cast<uintptr_t>(j.in) % sizeof(cpx)) ||
        (cout && reinterpret_cast<uintptr_t>(j.out) % sizeof(cpx))) {
      fail(MINFFT_B200_EINVAL, "mixed plan: complex data must be aligned to its size");
      minfft_b200_mixed_free(m);
      return nullptr;
    }
    m->jobs[i] = Job{j.in, j.out, j.op, lgn};
    if (n == 1) continue;
    if (lgL > kSmallMaxLog2L) {
      max_big = std::max(max_big, lgL);
      need_st[lgL] = 1;
      need_tw[(lgL + 1) / 2] = 1;  // scratch form: its two passes
      need_tw[lgL - (lgL + 1) / 2] = 1;
      need_tw[lgL - ilog2i(kN2)] = 1;  // cluster form: the L/256-point column DFTs
      need_tw[ilog2i(kN2)] = 1;        // and the 256-point row DFTs
    } else {
      need_tw[lgL] = 1;
    }
    need_kind[combo * kSlots + lgn] = 1;
  }
  if (!ok(cudaGetDevice(&m->device), "cudaGetDevice")) {
    minfft_b200_mixed_free(m);
    return nullptr;
  }
  Params& P = m->params;
  memset(&P, 0, sizeof(P));
  bool good = true;
  for (int lg = 0; lg < kSlots && good; ++lg) {
    const int64_t L = int64_t(1) << lg;
    if (need_tw[lg]) good = (P.tw[lg] = upload(m, mb::tables::TB_TW, L)) != nullptr;
    if (good && need_st[lg]) {
      good = (P.sthi[lg] = upload(m, mb::tables::TB_STHI, L)) && (P.stlo[lg] = upload(m, mb::tables::TB_STLO, L));
    }
    for (int combo = 1; combo < mb::K_COUNT && good; ++combo) {
      if (!need_kind[combo * kSlots + lg]) continue;
      const int64_t N = L;
      if (combo == mb::K_R2C || combo == mb::K_C2R || combo == mb::K_DCT2 || combo == mb::K_DCT3)
        if (!P.rft[lg]) good = (P.rft[lg] = upload(m, mb::tables::TB_RFT, N)) != nullptr;
      if (good && (combo == mb::K_DCT2 || combo == mb::K_DCT3) && !P.t23[lg])
        good = (P.t23[lg] = upload(m, mb::tables::TB_T23, N)) != nullptr;
      if (good && combo == mb::K_T4 && !P.t4a[lg])
        good = (P.t4a[lg] = upload(m, mb::tables::TB_T4PRE, N)) && (P.t4b[lg] = upload(m, mb::tables::TB_T4POST, N));
    }
  }
  int sms = 148;
  if (good) good = ok(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device), "device query");
  m->smem = kernel_smem();
  if (good)
    good = ok(cudaFuncSetAttribute((const void*)mixed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(m->smem)),
              "cudaFuncSetAttribute");
  int occ = 1;
  if (good)
    good = ok(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void*)mixed_kernel, kThreads, m->smem),
              "occupancy query");
  m->per_sm = std::max(1, occ);
  m->grid = sms * m->per_sm;
  // long items: the cluster form with MINFFT_B200_MIXED_CLUSTER=1, where the
  // device can co-schedule clusters of eight CTAs with this shared memory
  // (measured slower than the per-CTA scratch form on the 20000-job batch,
  // so not the default)
  const char* ce = getenv("MINFFT_B200_MIXED_CLUSTER");
  if (good && max_big > 0 && ce && ce[0] == '1') {
    const size_t csmem = std::max(kernel_smem(), cluster_big_smem());
    int nclusters = 0;
    if (cudaFuncSetAttribute((const void*)mixed_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(csmem)) == cudaSuccess) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(kCluster);
      cfg.blockDim = dim3(kThreads);
      cfg.dynamicSmemBytes = csmem;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = kCluster;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      if (cudaOccupancyMaxActiveClusters(&nclusters, (const void*)mixed_cluster_kernel, &cfg) != cudaSuccess)
        nclusters = 0;
    }
    cudaGetLastError();
    if (nclusters > 0) {
      m->cluster = true;
      m->smem = csmem;
      m->grid = nclusters * kCluster;
      m->per_sm = std::max(1, m->grid / sms);
    }
  }
  if (good) good = ok(mb::dev_malloc(&m->d_jobs, count * sizeof(Job)), "cudaMalloc(jobs)");
  if (good)
    good = ok(cudaMemcpy(m->d_jobs, m->jobs.data(), count * sizeof(Job), cudaMemcpyHostToDevice), "cudaMemcpy(jobs)");
  if (good) good = ok(mb::dev_malloc(&m->d_counter, 2 * sizeof(unsigned)), "cudaMalloc(counter)");
  if (good && max_big > 0 && !m->cluster) {
    P.scratch_stride = int64_t(2) << kBigMaxLog2L;
    good = ok(mb::dev_malloc(&m->d_scratch, size_t(m->grid) * P.scratch_stride * sizeof(cpx)), "cudaMalloc(scratch)");
  }
  P.jobs = static_cast<const Job*>(m->d_jobs);
  P.counter = m->d_counter;
  P.scratch = m->d_scratch;
  if (good) good = build_items(m);
  if (!good) {
    minfft_b200_mixed_free(m);
    return nullptr;
  }
  return m;
}

MB_EXPORT int minfft_b200_mixed_execute(minfft_b200_mixed* m, void* stream) {
  if (!m || !m->exec) return fail(MINFFT_B200_EINVAL, "mixed execute: NULL plan");
  return ok(cudaGraphLaunch(m->exec, static_cast<cudaStream_t>(stream)), "cudaGraphLaunch") ? MINFFT_B200_OK
                                                                                             : MINFFT_B200_ECUDA;
}

MB_EXPORT int minfft_b200_mixed_items(const minfft_b200_mixed* m) { return m ? int(m->items.size()) : -1; }

// Time the plan's tile shapes (jobs per short work item: all slots, 1/2,
// 1/4, 1/8 of them) and persistent grid sizes (1 .. max CTAs per SM), keep
// the fastest.  Runs the batch several times (outputs are overwritten).
MB_EXPORT int minfft_b200_mixed_autotune(minfft_b200_mixed* m, int reps) {
  if (!m) return fail(MINFFT_B200_EINVAL, "mixed autotune: NULL plan");
  if (reps < 1) reps = 3;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device);
  const int max_per_sm = m->per_sm;
  cudaStream_t st;
  if (!ok(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate")) return MINFFT_B200_ECUDA;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int best_split = m->split, best_per = m->per_sm;
  const int grid_cap = m->grid;  // scratch is sized for this many CTAs
  // the cluster form keeps every co-resident cluster (its grid is the
  // occupancy query's cluster count, not a multiple of the SMs)
  auto grid_for = [&](int per) {
    return m->cluster ? grid_cap : std::min(grid_cap, sms * per);
  };
  for (int split : {1, 2, 4, 8}) {
    for (int per = 1; per <= (m->cluster ? 1 : max_per_sm); ++per) {
      m->split = split;
      m->grid = grid_for(per);
      if (!build_items(m)) continue;
      cudaGraphLaunch(m->exec, st);
      cudaEventRecord(e0, st);
      for (int r = 0; r < reps; ++r) cudaGraphLaunch(m->exec, st);
      cudaEventRecord(e1, st);
      cudaEventSynchronize(e1);
      float ms = 0;
      if (cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && ms > 0 && ms < best) {
        best = ms;
        best_split = split;
        best_per = per;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  m->split = best_split;
  m->grid = grid_for(best_per);
  return build_items(m) ? MINFFT_B200_OK : MINFFT_B200_ECUDA;
}
