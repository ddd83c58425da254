// Persistent, software-pipelined axis pass.
//
// Same arithmetic as axis_pass_kernel (the Stockham core and the store stages
// are shared), different data movement: each CTA stays resident and walks a
// strided list of tiles (cpb transforms each).  While tile i is being
// computed from shared-memory stage i%2, the raw input of tile i+1 is already
// streaming into the other stage with cp.async (16-, 8- or 4-byte copies that
// bypass registers), so HBM traffic overlaps the butterflies and the shared
// memory exchanges instead of alternating with them.  The stage that held a
// tile's raw input then serves as that tile's Stockham exchange buffer and
// staging area for the store, and is refilled with tile i+2 once the tile is
// done.
//
// Tiles.  Row mode (transforms are contiguous rows): tile t holds transforms
// t*cpb .. t*cpb+cpb-1, copied row by row.  Column mode: a tile holds cpb
// adjacent columns of one d0 block (tiles never straddle blocks), copied as
// runs of cpb adjacent elements per row.
#pragma once

#include "axis_pass.cuh"

namespace mb {

// ------------------------------------------------------------ async copies
template <int CH>
__device__ __forceinline__ void cp_async(unsigned dst, const void* src) {
  if constexpr (CH == 16) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
  } else if constexpr (CH == 8) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(src) : "memory");
  }
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Copy `runs` runs of `run_bytes` bytes (a multiple of CH) from global
// addresses src0 + run*src_stride (or per-run offsets) to dst0 + run*dst_stride.
template <int CH>
__device__ __forceinline__ void copy_runs(unsigned dst0, int dst_stride, const char* src0, int64_t src_stride,
                                          const int64_t* run_off, int runs, int run_bytes) {
  const int cpr = run_bytes / CH;
  const int total = runs * cpr;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int run = i / cpr, k = i - run * cpr;
    const char* src = run_off ? src0 + run_off[run] + int64_t(k) * CH : src0 + run * src_stride + int64_t(k) * CH;
    cp_async<CH>(dst0 + unsigned(run * dst_stride + k * CH), src);
  }
}

// ------------------------------------------------------------- raw tiles
// Raw input of a tile in shared memory: element e of transform c at
// (row mode) c*e_raw + e or (column mode) e*cpb + c, in units of the raw type.
struct RawTile {
  const unsigned char* base;
  int cpb, colmode, e_raw;
  template <class T>
  __device__ __forceinline__ T at(int c, int e) const {
    const int i = colmode ? e * cpb + c : c * e_raw + e;
    return reinterpret_cast<const T*>(base)[i];
  }
};

// Kinds of the pipelined kernel: raw element type, raw elements per
// transform, and the read from the raw tile into registers (element
// n = j + r*(L/R) of the length-L complex DFT).
struct PCplx {
  using Raw = cpx;
  static constexpr int e_raw(int L) { return L; }
  template <int L, int R>
  static __device__ __forceinline__ void read(const AxisParams& p, const Ctx& x, const RawTile& rt, const Tile&,
                                              cpx (&v)[R]) {
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = x.active ? rt.at<cpx>(x.c, x.j + r * (L / R)) : czero();
    if (p.flags & F_CONJ_IN) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r].y = -v[r].y;
    }
    if (p.st_ns > 1) hbm_pretwiddle<L, R>(v, p, x.b0, x.j);
  }
};

struct PR2C {
  using Raw = real;
  static constexpr int e_raw(int L) { return 2 * L; }
  template <int L, int R>
  static __device__ __forceinline__ void read(const AxisParams&, const Ctx& x, const RawTile& rt, const Tile&,
                                              cpx (&v)[R]) {
    // row mode only: the real row read as complex pairs
    const cpx* row = reinterpret_cast<const cpx*>(rt.base) + x.c * L;
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = x.active ? row[x.j + r * (L / R)] : czero();
  }
};

struct PDCT2 {
  using Raw = real;
  static constexpr int e_raw(int L) { return 2 * L; }
  template <int L, int R>
  static __device__ __forceinline__ void read(const AxisParams& p, const Ctx& x, const RawTile& rt, const Tile&,
                                              cpx (&v)[R]) {
    const real sg = (p.flags & F_DST) ? real(-1) : real(1);
    constexpr int N = 2 * L;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int m = x.j + r * (L / R);
      const int i0 = 2 * m, i1 = 2 * m + 1;
      const real a = i0 < L ? rt.at<real>(x.c, 2 * i0) : sg * rt.at<real>(x.c, 2 * N - 1 - 2 * i0);
      const real b = i1 < L ? rt.at<real>(x.c, 2 * i1) : sg * rt.at<real>(x.c, 2 * N - 1 - 2 * i1);
      v[r] = x.active ? cmk(a, b) : czero();
    }
  }
};

struct PT4 {
  using Raw = real;
  static constexpr int e_raw(int L) { return 2 * L; }
  template <int L, int R>
  static __device__ __forceinline__ void read(const AxisParams& p, const Ctx& x, const RawTile& rt, const Tile&,
                                              cpx (&v)[R]) {
    const bool dst = (p.flags & F_DST) != 0;
    constexpr int N = 2 * L;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int n = x.j + r * (L / R);
      const real a = rt.at<real>(x.c, 2 * n);
      const real b = rt.at<real>(x.c, N - 1 - 2 * n);
      const cpx e = ldg(p.t1 + n);
      cpx o;
      if (!dst) {
        o = cmul(e, cmk(a, b));
      } else {
        const cpx q = cmul(e, cmk(a, -b));
        o = cmk(-q.x, -q.y);
      }
      v[r] = x.active ? o : czero();
    }
  }
};

// Pairing kinds: every thread first reads the spectrum pairs (z_k, z_{L-k})
// it owns into registers, then -- after a barrier, because the packed values
// overwrite the raw tile in place -- writes the packed, conjugated inputs to
// the exchange layout and gathers its first-pass elements.
template <int L, int R, class Zf>
__device__ __forceinline__ void pair_pack_stage(const AxisParams& p, const Ctx& x, const Tile& t, const Zf& zf,
                                                cpx (&v)[R]) {
  constexpr int TPT = L / R;
  constexpr int NP = (L / 2) / TPT + 1;  // pair indices per thread (upper bound)
  cpx za[NP], zb[NP];
#pragma unroll
  for (int i = 0; i < NP; ++i) {
    const int k = x.j + i * TPT;
    za[i] = czero();
    zb[i] = czero();
    if (k <= L / 2 && x.active) {
      za[i] = zf(k);
      zb[i] = zf(L - k);
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NP; ++i) {
    const int k = x.j + i * TPT;
    if (k > L / 2) continue;
    if (k == 0) {
      t.s[t.idx(x.c, 0)] = cmk(za[i].x + zb[i].x, -(za[i].x - zb[i].x));
    } else if (2 * k == L) {
      t.s[t.idx(x.c, k)] = cmk(2 * za[i].x, 2 * za[i].y);
    } else {
      cpx ta, tb;
      pack_pair(za[i], zb[i], ldg(p.t2 + k), ta, tb);
      t.s[t.idx(x.c, k)] = cconj(ta);
      t.s[t.idx(x.c, L - k)] = cconj(tb);
    }
  }
  __syncthreads();
  gather_natural<L, R>(v, x.j, x.c, t);
}

struct PC2R {
  using Raw = cpx;
  static constexpr int e_raw(int L) { return L + 1; }
  template <int L, int R>
  static __device__ __forceinline__ void read(const AxisParams& p, const Ctx& x, const RawTile& rt, const Tile& t,
                                              cpx (&v)[R]) {
    pair_pack_stage<L, R>(p, x, t, [&](int k) { return rt.at<cpx>(x.c, k); }, v);
  }
};

struct PDCT3 {
  using Raw = real;
  static constexpr int e_raw(int L) { return 2 * L; }
  template <int L, int R>
  static __device__ __forceinline__ void read(const AxisParams& p, const Ctx& x, const RawTile& rt, const Tile& t,
                                              cpx (&v)[R]) {
    const bool dst = (p.flags & F_DST) != 0;
    auto rd = [&](int i) { return rt.at<real>(x.c, i); };
    pair_pack_stage<L, R>(p, x, t, [&](int k) { return LoadDCT3::zval_r(rd, k, L, dst, p.t1); }, v);
  }
};

// Shared memory of the pipelined kernel: per stage, the tile's input and
// output offsets (2*cpb int64), then the two stages.
__host__ __device__ inline size_t pipe_offsets_bytes(int cpb) { return 16 * ((4 * size_t(cpb) * sizeof(int64_t) + 15) / 16); }
__host__ __device__ inline size_t pipe_stage_bytes(int L, int R, int cpb, int colmode, int e_raw, size_t raw_size) {
  const size_t a = size_t(cpb) * tile_pitch(L, R, cpb, colmode) * sizeof(cpx);
  const size_t b = size_t(cpb) * e_raw * raw_size;
  return 16 * (((a > b ? a : b) + 15) / 16);
}
__host__ __device__ inline size_t pipe_smem(int L, int R, int cpb, int colmode, int e_raw, size_t raw_size) {
  return pipe_offsets_bytes(cpb) + 2 * pipe_stage_bytes(L, R, cpb, colmode, e_raw, raw_size);
}

template <int L, int R, class PLoad, class StoreOp>
__global__ void __launch_bounds__(512, MinBlocks<R>::value) axis_pipe_kernel(const AxisParams p) {
  constexpr int TPT = L / R;
  using Raw = typename PLoad::Raw;
  constexpr int ER = PLoad::e_raw(L);
  pdl_release();
  pdl_wait();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int64_t* offs = reinterpret_cast<int64_t*>(smem_raw);  // [stage][in|out][cpb]
  unsigned char* stages = smem_raw + pipe_offsets_bytes(p.cpb);
  const int cpb = p.cpb;

  int c, j;
  if (p.colmode) {
    c = threadIdx.x % cpb;
    j = threadIdx.x / cpb;
  } else {
    j = threadIdx.x % TPT;
    c = threadIdx.x / TPT;
  }

  // first transform and count of a tile
  auto tile_span = [&](int64_t t, int64_t& b_first, int& nvalid) {
    if (p.colmode) {
      const int64_t blk = udiv(t, p.gpb), g = t - blk * p.gpb;
      const int64_t start = g * cpb;
      b_first = blk * p.d0 + start;
      nvalid = int((p.d0 - start) < cpb ? (p.d0 - start) : cpb);
    } else {
      b_first = t * cpb;
      const int64_t left = p.nbatch - b_first;
      nvalid = int(left < cpb ? left : cpb);
    }
  };

  // start the asynchronous copy of tile t's raw input into stage s
  auto issue = [&](int64_t t, int s) {
    if (t < p.ntiles) {
      int64_t bf;
      int nv;
      tile_span(t, bf, nv);
      int64_t* oin = offs + s * 2 * cpb;
      int64_t* oout = oin + cpb;
      for (int cc = threadIdx.x; cc < cpb; cc += blockDim.x) {
        int64_t b0, oi = 0, oo = 0;
        if (cc < nv) batch_offsets(p, bf + cc, b0, oi, oo);
        oin[cc] = oi * int64_t(sizeof(Raw));
        oout[cc] = oo;
      }
      __syncthreads();
      const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(stages + size_t(s) * p.stage_bytes));
      const char* src = static_cast<const char*>(p.in);
      if (!p.colmode) {
        // one run per transform: ER contiguous raw elements (C2R: the last
        // spectrum element of each row goes separately, see below)
        const int run_elems = (ER % 2 == 1) ? ER - 1 : ER;
        const int rb = run_elems * int(sizeof(Raw));
        if (p.chunk == 16)
          copy_runs<16>(dst, ER * int(sizeof(Raw)), src, 0, oin, nv, rb);
        else if (p.chunk == 8)
          copy_runs<8>(dst, ER * int(sizeof(Raw)), src, 0, oin, nv, rb);
        else
          copy_runs<4>(dst, ER * int(sizeof(Raw)), src, 0, oin, nv, rb);
        if (ER % 2 == 1) {
          for (int cc = threadIdx.x; cc < nv; cc += blockDim.x)
            cp_async<sizeof(Raw) >= 16 ? 16 : (sizeof(Raw) >= 8 ? 8 : 4)>(
                dst + unsigned((cc * ER + ER - 1) * sizeof(Raw)), src + oin[cc] + (ER - 1) * int64_t(sizeof(Raw)));
        }
      } else {
        // one run per element row: nv adjacent columns; a partial tile is
        // copied element by element (elements are always naturally aligned)
        const int rb = nv * int(sizeof(Raw));
        const int64_t stride = p.in_n * int64_t(sizeof(Raw));
        const char* s0 = src + oin[0];
        const int ch = (nv == cpb) ? p.chunk : int(sizeof(Raw));
        const int ds = cpb * int(sizeof(Raw));
        if (ch == 16)
          copy_runs<16>(dst, ds, s0, stride, nullptr, ER, rb);
        else if (ch == 8)
          copy_runs<8>(dst, ds, s0, stride, nullptr, ER, rb);
        else
          copy_runs<4>(dst, ds, s0, stride, nullptr, ER, rb);
      }
    }
    cp_commit();
  };

  const int64_t stride_t = gridDim.x;
  issue(blockIdx.x, 0);
  issue(blockIdx.x + stride_t, 1);
  int it = 0;
  for (int64_t t = blockIdx.x; t < p.ntiles; t += stride_t, ++it) {
    const int s = it & 1;
    cp_wait<1>();
    __syncthreads();
    int64_t bf;
    int nv;
    tile_span(t, bf, nv);
    int64_t* oin = offs + s * 2 * cpb;
    TileOffsets to{oin, oin + cpb, nv};
    unsigned char* st = stages + size_t(s) * p.stage_bytes;
    Tile tl{reinterpret_cast<cpx*>(st), p.lp};
    RawTile rt{st, cpb, p.colmode, ER};
    Ctx x;
    x.c = c;
    x.j = j;
    x.b = bf + c;
    x.active = c < nv;
    x.b0 = umod(x.b, p.d0);
    x.oin = 0;
    x.oout = to.out_off[c];
    cpx v[R];
    PLoad::template read<L, R>(p, x, rt, tl, v);
    run_passes<L, R, 1>(v, x.j, x.c, tl, p.tw);
    StoreOp::template run<L, R>(p, x, tl, to, v);
    __syncthreads();
    issue(t + 2 * stride_t, s);
  }
  cp_wait<0>();
}

}  // namespace mb
