// Tensor-core split-precision axis pass (tc_pass.cu): batched complex DFTs
// of length 256 along one axis, two radix-16 stages as DFT-matrix
// contractions on tcgen05 with FP16 or BF16 split operands and FP32
// accumulation.  Single-precision library only.
#pragma once

#include <stddef.h>
#include <stdint.h>

#include <vector>

namespace mb {

enum TcFormat : int {
  TC_F16 = 0,   // two FP16 terms per operand, three products
  TC_BF16 = 1,  // three BF16 terms per operand, six products
};

struct TcParams {
  const void* bmat;  // split DFT-16 operands, tc_bmat_bytes(fmt) bytes (tc_bmat_host)
  int* status;       // set to 1 when a CTA gave up waiting for its tensor-core work
  // Test hook (zero in normal launches): with withhold = 1 the first stage
  // of each CTA's first tile issues no MMA and no commit, so its wait -- limited
  // to wait_polls polls -- runs out and the status path is exercised without
  // any fault.
  long long wait_polls;
  int withhold;
};

constexpr int kTcLength = 256;

// Kernel for format fmt and tb transforms per CTA (8 or 16); nullptr in the
// double-precision library or for an unsupported tb.  Launch with
// tc_threads(tb) threads and tc_smem(fmt, tb) bytes of dynamic shared
// memory; the CTAs are persistent (CTA k takes tiles of tb transforms k,
// k + gridDim.x, ...), so any grid up to (nbatch + tb - 1) / tb CTAs covers
// the batch.  Arguments (AxisParams, TcParams).
const void* tc_kernel(int fmt, int tb);
size_t tc_smem(int fmt, int tb);

// The streamed form (persistent CTAs of 128 threads, tiles of 8 transforms
// fed through `stages` shared-memory stages by tensor copies or cp.async;
// arguments (AxisParams with cpb = stages, TcParams, CUtensorMap)): column
// tiles (8 adjacent transforms, unit stride between them) or row tiles
// (8 transforms of contiguous points).  nullptr in the double library.
const void* tc_stream_kernel_fn(int fmt, bool rows);
size_t tc_stream_smem(int fmt, int stages);
int tc_stream_stage_bytes();
constexpr int kTcStreamThreads = 128;
constexpr int kTcStreamTile = 8;
constexpr int kTcStreamTmemCols = 64;  // a leading and a correction accumulator of 32 columns
inline int tc_threads(int tb) { return 16 * tb; }
// Tensor-memory columns a CTA allocates: per 8 transforms, a leading and a
// correction accumulator of 32 FP32 columns each.
inline int tc_tmem_columns(int tb) { return 64 * (tb / 8); }

// Split terms per operand and the bytes of the B operand image.
inline int tc_terms(int fmt) { return fmt == TC_F16 ? 2 : 3; }
inline size_t tc_bmat_bytes(int fmt) { return size_t(tc_terms(fmt)) * 32 * 32 * 2; }

// Host image of the B operands: for each split term, the real 32 x 32 form
// [[C, S], [-S, C]] of the forward 16-point DFT matrix (row n = output
// column of the contraction, K-major), laid out as the canonical
// no-swizzle K-major UMMA operand (tc_operand_offset).
void tc_bmat_host(int fmt, std::vector<uint16_t>& out);

// Byte offset of element (row m, column k) of a K-major 16-bit operand with
// 32 columns: 8 x 8 core matrices of 128 contiguous bytes, column blocks of
// 8 one core matrix (128 bytes) apart, row blocks of 8 four core matrices
// (512 bytes) apart.
__host__ __device__ inline int tc_operand_offset(int m, int k) {
  return (m >> 3) * 512 + (k >> 3) * 128 + (m & 7) * 16 + (k & 7) * 2;
}

// Splits v into tc_terms(fmt) 16-bit terms (bit patterns), largest first,
// each the correctly rounded value of the remainder.
void tc_split_host(int fmt, float v, uint16_t* terms);

}  // namespace mb
