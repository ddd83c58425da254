// Streamed column pass: a persistent, TMA-fed form of the complex axis pass
// for strided columns (the column passes of multi-dimensional transforms and
// the passes of a Stockham FFT over HBM).
//
// Tile.  W = 128 / sizeof(cpx) adjacent columns (transforms) of one block,
// all L elements of each: 8 columns in double, 16 in single, so every
// element row of the tile is one 128-byte line.  In shared memory the tile
// is stored row by row, element n of column c at n*W + c -- exactly the
// layout a 2-D bulk tensor copy (box of 2W reals x up to 256 rows) writes.
//
// Threads.  Thread t owns column c = t % W and holds elements j + r*(L/R)
// (j = t / W) of it in registers, as in the one-tile kernel.  The threads
// of one shared-memory wavefront (a quarter warp of 16-byte accesses in
// double, a half warp of 8-byte accesses in single) are the W columns of
// one element row, so every load, Stockham scatter and gather of the tile
// touches one whole 128-byte line: no padding and no bank conflicts,
// whatever the element permutation.
//
// Pipeline.  Each CTA stays resident and walks tiles blockIdx.x,
// blockIdx.x + gridDim.x, ...; S stages of shared memory hold the tiles in
// flight.  Thread 0 issues a tile's copy into a free stage with an mbarrier
// expecting its bytes; the CTA waits on the barrier, computes the tile in
// place (the stage doubles as the exchange buffer) and stores from
// registers, then refills the stage with the tile S steps ahead.  So while
// one tile is transformed, the next S - 1 are already on their way from
// HBM.  Where the strides do not allow a tensor copy (a row pitch that is
// not a multiple of 16 bytes), every thread copies its share of the tile
// with cp.async and the barrier counts the threads' arrivals instead.
//
// Waits are bounded: a wait that runs out sets *status, the CTA stops
// issuing, waits (bounded) for the copies it has in flight and returns.
#pragma once

#include <cuda.h>

#include "axis_pass.cuh"

namespace mb {

constexpr long long kStreamSpinLimit = 1LL << 22;

__host__ __device__ constexpr int stream_cols() { return int(128 / sizeof(cpx)); }

// Bytes of one stage for length L: the tile, plus one spare element per
// column for the transposed staging of row-contiguous outputs.
__host__ __device__ inline int stream_stage_bytes(int L) {
  const int W = stream_cols();
  return (W * (L + 1) * int(sizeof(cpx)) + 127) / 128 * 128;
}
__host__ __device__ inline size_t stream_smem(int L, int stages) {
  return 128 + size_t(stages) * stream_stage_bytes(L);
}

__device__ __forceinline__ void smbar_init(uint32_t mbar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

__device__ __forceinline__ bool smbar_wait(uint32_t mbar, uint32_t phase, long long limit) {
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

// In-place Stockham pass of the streamed tile (layout n*W + c).
template <int L, int R, int RP, int NS, int W>
__device__ __forceinline__ void stream_scatter(const cpx (&v)[R], int j, int c, cpx* s) {
  constexpr int S = R / RP;
#pragma unroll
  for (int q = 0; q < S; ++q) {
    const int jp = j + q * (L / R);
    const int base = (jp / NS) * (NS * RP) + (jp & (NS - 1));
#pragma unroll
    for (int r = 0; r < RP; ++r) s[(base + r * NS) * W + c] = v[q + r * S];
  }
}

template <int L, int R, int W>
__device__ __forceinline__ void stream_gather(cpx (&v)[R], int j, int c, const cpx* s) {
  constexpr int TPT = L / R;
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = s[(j + r * TPT) * W + c];
}

template <int L, int R, int NS, int W>
__device__ __forceinline__ void stream_passes(cpx (&v)[R], int j, int c, cpx* s, const cpx* __restrict__ tw) {
  constexpr int RP = (L / NS >= R) ? R : (L / NS);
  pass_compute<L, R, RP, NS>(v, j, tw);
  if constexpr (NS * RP < L) {
    __syncthreads();
    stream_scatter<L, R, RP, NS, W>(v, j, c, s);
    __syncthreads();
    stream_gather<L, R, W>(v, j, c, s);
    stream_passes<L, R, NS * RP, W>(v, j, c, s, tw);
  }
}

// Streamed pass flags (AxisParams::flags bits above the kind flags).
enum : int {
  F_STREAM_TMA = 1 << 8,  // the tile copies are tensor copies (else per-thread cp.async)
};

template <int L, int R>
__global__ void __launch_bounds__(stream_cols() * (L / R), 1)
    stream_pass_kernel(const AxisParams p, const __grid_constant__ CUtensorMap tmap) {
  constexpr int W = stream_cols();
  constexpr int TPT = L / R;
  constexpr int NT = W * TPT;
  constexpr int BOX = L < 256 ? L : 256;
  constexpr int C = int(sizeof(cpx));
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem);  // one per stage (at most 8)
  int* bad = reinterpret_cast<int*>(smem + 64);
  unsigned char* stages = smem + 128;
  const int S = p.cpb;  // stages
  const int tid = threadIdx.x;
  const int c = tid % W, j = tid / W;
  const bool tma = (p.flags & F_STREAM_TMA) != 0;
  const uint32_t mbar0 = static_cast<uint32_t>(__cvta_generic_to_shared(mbar));
  const uint32_t st0 = static_cast<uint32_t>(__cvta_generic_to_shared(stages));
  const int64_t gpd = (p.d0 + W - 1) / W;  // tiles per block of adjacent columns
  const int64_t ntiles = p.ntiles;

  pdl_release();
  pdl_wait();
  if (tid == 0) {
    for (int s = 0; s < S; ++s) smbar_init(mbar0 + 8 * s, tma ? 1 : NT);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *bad = 0;
  }
  __syncthreads();

  // tile t -> first column, block indices
  auto tile_pos = [&](int64_t t, int64_t& col0, int64_t& b1, int64_t& b2) {
    const int64_t rest = udiv(t, gpd);
    col0 = (t - rest * gpd) * W;
    b2 = udiv(rest, p.d1);
    b1 = rest - b2 * p.d1;
  };

  // start the copy of tile t into stage s
  auto issue = [&](int64_t t, int s) {
    if (t >= ntiles) return;
    int64_t col0, b1, b2;
    tile_pos(t, col0, b1, b2);
    const uint32_t mb = mbar0 + 8 * s;
    const uint32_t dst = st0 + uint32_t(s) * uint32_t(p.stage_bytes);
    if (tma) {
      if (tid == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(L * W * C) : "memory");
#pragma unroll
        for (int n0 = 0; n0 < L; n0 += BOX) {
          asm volatile(
              "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
              "[%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst + uint32_t(n0 * W * C)),
              "l"(&tmap), "r"(int(2 * col0)), "r"(n0), "r"(int(b1)), "r"(int(b2)), "r"(mb)
              : "memory");
        }
      }
    } else {
      // every thread: elements e = tid + i*NT of the tile (row n = e / W,
      // column e % W), the columns beyond the block left unread
      const int nv = int(p.d0 - col0 < W ? p.d0 - col0 : W);
      const char* src = static_cast<const char*>(p.in) + (b1 * p.is1 + b2 * p.is2 + col0 * p.is0) * C;
#pragma unroll
      for (int i = 0; i < R; ++i) {
        const int e = tid + i * NT;
        const int n = e / W, cc = e % W;
        if (cc < nv) {
          const char* g = src + (int64_t(n) * p.in_n + cc * p.is0) * C;
          const uint32_t d = dst + uint32_t(e * C);
          if constexpr (C == 16)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(g) : "memory");
          else
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(g) : "memory");
        }
      }
      asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(mb) : "memory");
    }
  };

  for (int s = 0; s < S; ++s) issue(blockIdx.x + int64_t(s) * gridDim.x, s);

  const bool cj_in = (p.flags & F_CONJ_IN) != 0, cj_out = (p.flags & F_CONJ_OUT) != 0;
  const bool rows_out = (p.flags & F_STAGE_ROWS) != 0;
  int it = 0;
  bool ok = true;
  int64_t t = blockIdx.x;
  for (; t < ntiles; t += gridDim.x, ++it) {
    const int s = it % S;
    const uint32_t phase = uint32_t(it / S) & 1u;
    if (!smbar_wait(mbar0 + 8 * s, phase, kStreamSpinLimit)) atomicExch(bad, 1);
    __syncthreads();
    if (*bad) {
      ok = false;
      break;
    }
    cpx* tile = reinterpret_cast<cpx*>(stages + size_t(s) * p.stage_bytes);
    int64_t col0, b1, b2;
    tile_pos(t, col0, b1, b2);
    const int64_t col = col0 + c;
    const bool active = col < p.d0;

    cpx v[R];
    stream_gather<L, R, W>(v, j, c, tile);
    if (cj_in) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r].y = -v[r].y;
    }
    if (p.st_ns > 1) hbm_pretwiddle<L, R>(v, p, col, j);
    stream_passes<L, R, 1, W>(v, j, c, tile, p.tw);
    if (cj_out) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r].y = -v[r].y;
    }
    cpx* out = static_cast<cpx*>(p.out);
    const int64_t ob = b1 * p.os1 + b2 * p.os2;
    if (!rows_out) {
      if (active) {
        cpx* q = out + ob + col * p.os0 + int64_t(j) * p.out_k;
        const int64_t st = int64_t(TPT) * p.out_k;
#pragma unroll
        for (int r = 0; r < R; ++r) q[r * st] = v[r];
      }
    } else {
      // outputs of a column contiguous (out_k = 1): transpose through the
      // stage (column c at c*(L+1)), then store with k running fastest
      __syncthreads();
#pragma unroll
      for (int r = 0; r < R; ++r) tile[c * (L + 1) + j + r * TPT] = v[r];
      __syncthreads();
      const int nv = int(p.d0 - col0 < W ? p.d0 - col0 : W);
#pragma unroll
      for (int i = 0; i < R; ++i) {
        const int e = tid + i * NT;
        const int cc = e / L, k = e % L;
        if (cc < nv) out[ob + (col0 + cc) * p.os0 + int64_t(k) * p.out_k] = tile[cc * (L + 1) + k];
      }
    }
    __syncthreads();  // the stage is free: refill it with the tile S steps ahead
    if (tma && tid == 0) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    issue(t + int64_t(S) * gridDim.x, s);
  }

  if (!ok) {
    if (tid == 0 && p.status) atomicExch(p.status, 1);
    // copies already issued into the stages must land before the CTA's
    // shared memory is released: wait for each outstanding stage (bounded)
    for (int k = 0; k < S; ++k, ++it, t += gridDim.x) {
      if (t >= ntiles) break;
      smbar_wait(mbar0 + 8 * (it % S), uint32_t(it / S) & 1u, kStreamSpinLimit);
    }
  }
}

}  // namespace mb

namespace mb {

// -------------------------------------------------------- streamed rows
// The row-mode counterpart: persistent CTAs walk tiles of cpb transforms
// whose input rows are contiguous; each row of a tile arrives in a stage of
// shared memory by one bulk copy (cp.async.bulk, no tensor map) or, where
// the row's bytes or addresses break the 16-byte rules, by per-thread
// cp.async, counted by the stage's mbarrier.  The kind's own load stage
// (LoadR2C, LoadDCT2, LoadT4, LoadC2R, LoadDCT3, LoadC2RQ, LoadCplx) then
// reads the row from the stage instead of global memory -- the same index
// arithmetic on a shared-memory base -- and the stage is refilled with the
// tile S steps ahead right away, so the next tiles' rows stream in while this
// one is transformed in the padded exchange tile and stored by the kind's
// store stage.  Waits are bounded as in the column form.
__host__ __device__ inline size_t stream_rows_offsets_bytes(int cpb) {
  return 16 * ((2 * size_t(cpb) * sizeof(int64_t) + 15) / 16);
}
__host__ __device__ inline size_t stream_rows_tile_bytes(int L, int R, int cpb) {
  return (size_t(cpb) * tile_pitch(L, R, cpb, 0) * sizeof(cpx) + 127) / 128 * 128;
}
__host__ __device__ inline size_t stream_rows_smem(int L, int R, int cpb, int stages, int row_pitch) {
  return 128 + (stream_rows_offsets_bytes(cpb) + 127) / 128 * 128 + stream_rows_tile_bytes(L, R, cpb) +
         size_t(stages) * cpb * row_pitch;
}

template <int L, int R, class LoadOp, class StoreOp>
__global__ void __launch_bounds__(512, 1) stream_rows_kernel(const AxisParams p) {
  constexpr int TPT = L / R;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem);
  int* bad = reinterpret_cast<int*>(smem + 64);
  const int cpb = p.cpb, S = p.nstages;
  int64_t* offs = reinterpret_cast<int64_t*>(smem + 128);
  unsigned char* tile_raw = smem + 128 + (stream_rows_offsets_bytes(cpb) + 127) / 128 * 128;
  unsigned char* stages = tile_raw + stream_rows_tile_bytes(L, R, cpb);
  const int stage_bytes = cpb * p.row_pitch;
  const int tid = threadIdx.x;
  const bool bulk = (p.flags & F_STREAM_TMA) != 0;
  const uint32_t mbar0 = static_cast<uint32_t>(__cvta_generic_to_shared(mbar));
  const uint32_t st0 = static_cast<uint32_t>(__cvta_generic_to_shared(stages));
  const int64_t ntiles = p.ntiles;
  constexpr int esz = LoadOp::kComplexIn ? int(sizeof(cpx)) : int(sizeof(real));

  pdl_release();
  pdl_wait();
  if (tid == 0) {
    for (int s = 0; s < S; ++s) smbar_init(mbar0 + 8 * s, bulk ? 1 : int(blockDim.x));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *bad = 0;
  }
  __syncthreads();

  auto issue = [&](int64_t t, int s) {
    if (t >= ntiles) return;
    const int64_t b0t = t * cpb;
    const int nv = int(p.nbatch - b0t < cpb ? p.nbatch - b0t : cpb);
    const uint32_t mb = mbar0 + 8 * s;
    const uint32_t dst = st0 + uint32_t(s) * uint32_t(stage_bytes);
    const char* in = static_cast<const char*>(p.in);
    if (bulk) {
      if (tid == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(nv * p.row_bytes)
                     : "memory");
        for (int c = 0; c < nv; ++c) {
          int64_t b0, oi, oo;
          batch_offsets(p, b0t + c, b0, oi, oo);
          asm volatile(
              "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                  dst + uint32_t(c * p.row_pitch)),
              "l"(in + oi * esz), "r"(p.row_bytes), "r"(mb)
              : "memory");
        }
      }
    } else {
      const int ch = p.chunk;
      const int cpr = p.row_bytes / ch;
      for (int e = tid; e < nv * cpr; e += blockDim.x) {
        const int c = e / cpr, k = e - c * cpr;
        int64_t b0, oi, oo;
        batch_offsets(p, b0t + c, b0, oi, oo);
        const char* g = in + oi * esz + int64_t(k) * ch;
        const uint32_t d = dst + uint32_t(c * p.row_pitch + k * ch);
        if (ch == 16)
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(g) : "memory");
        else if (ch == 8)
          asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(g) : "memory");
        else
          asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(g) : "memory");
      }
      asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(mb) : "memory");
    }
  };

  for (int s = 0; s < S; ++s) issue(blockIdx.x + int64_t(s) * gridDim.x, s);

  Tile tl{reinterpret_cast<cpx*>(tile_raw), p.lp};
  int it = 0;
  bool ok = true;
  int64_t t = blockIdx.x;
  for (; t < ntiles; t += gridDim.x, ++it) {
    const int s = it % S;
    if (!smbar_wait(mbar0 + 8 * s, uint32_t(it / S) & 1u, kStreamSpinLimit)) atomicExch(bad, 1);
    __syncthreads();
    if (*bad) {
      ok = false;
      break;
    }
    const int64_t b0t = t * cpb;
    const int nv = int(p.nbatch - b0t < cpb ? p.nbatch - b0t : cpb);
    for (int c = tid; c < cpb; c += blockDim.x) {
      int64_t b0, oi, oo;
      batch_offsets(p, b0t + c < p.nbatch ? b0t + c : 0, b0, oi, oo);
      offs[c] = oi;
      offs[cpb + c] = oo;
    }
    __syncthreads();
    TileOffsets to{offs, offs + cpb, nv};
    Ctx x;
    x.j = tid % TPT;
    x.c = tid / TPT;
    x.b = b0t + x.c;
    x.active = x.c < nv;
    x.b0 = umod(x.b, p.d0);
    x.oin = int64_t(x.c) * (p.row_pitch / esz);
    x.oout = offs[cpb + x.c];
    // the kind's load stage, on the rows in the stage
    AxisParams pl = p;
    pl.in = stages + size_t(s) * stage_bytes;
    pl.in_n = 1;
    pl.is0 = p.row_pitch / esz;
    pl.flags |= F_VEC | F_SRC_SMEM;
    cpx v[R];
    LoadOp::template run<L, R>(pl, x, tl, v);
    __syncthreads();  // every read of the stage is done: refill it
    if (bulk && tid == 0) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    issue(t + int64_t(S) * gridDim.x, s);
    run_passes<L, R, 1>(v, x.j, x.c, tl, p.tw);
    StoreOp::template run<L, R>(p, x, tl, to, v);
    __syncthreads();
  }
  if (!ok) {
    if (tid == 0 && p.status) atomicExch(p.status, 1);
    for (int k = 0; k < S; ++k, ++it, t += gridDim.x) {
      if (t >= ntiles) break;
      smbar_wait(mbar0 + 8 * (it % S), uint32_t(it / S) & 1u, kStreamSpinLimit);
    }
  }
}

}  // namespace mb
