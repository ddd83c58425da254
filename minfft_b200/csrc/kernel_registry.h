// Kernel registry: every instantiated axis-pass kernel, addressed by the
// (load stage, store stage) combination and log2 of its in-CTA DFT length.
#pragma once

namespace mb {

enum Combo : int {
  K_CPLX = 0,   // complex -> complex (DFT, inverse DFT via conjugation, HBM passes)
  K_R2C,        // real DFT with fused unpacking
  K_C2R,        // inverse real DFT with fused packing
  K_DCT2,       // DCT-2 / DST-2 with fused permutation, unpacking and post-rotation
  K_DCT3,       // DCT-3 / DST-3 with fused pre-rotation, packing and de-interleave
  K_T4,         // DCT-4 / DST-4 with fused pre- and post-rotation
  K_R2CQ,       // real DFT of 4 rows j + Q*m, then the first radix-4 stage of the column DFT across them
  K_C2RQ,       // last radix-4 stage of an inverse column DFT across 4 rows, then their inverse real DFT
  K_T4IN,       // first pass of a 1-D type-4 chain over HBM: the pre-rotation fused into its load
  K_T4OUT,      // last pass of a 1-D type-4 chain over HBM: the post-rotation fused into its store
  K_COUNT
};

constexpr int kMaxLog2L = 13;  // largest in-CTA DFT: 8192 points

// Returns the kernel function for combo, log2(L) and per-thread radix R (8 or
// 16; lengths below 16 use R = L), or nullptr where the configuration does not
// exist (more than 512 threads per transform).
const void* axis_kernel(int combo, int log2L, int R = 16);

// The persistent, software-pipelined form of the same kernels (pipe_pass.cuh),
// for log2(L) = 1 .. 13, or nullptr.
const void* pipe_kernel(int combo, int log2L, int R = 16);

// The streamed complex column pass (stream_pass.cuh) for log2(L) = 4 .. 9 and
// radix R (16, or 8 where the CTA stays within 512 threads), or nullptr.
const void* stream_kernel(int log2L, int R);

// The streamed row pass (stream_pass.cuh) of kind `combo` for log2(L) = 6 ..
// 12 (11 for the split-column kinds), radix 16, or nullptr.
const void* stream_rows_kernel_fn(int combo, int log2L);

// Root tables kept on the device by plans: w_N^m (m < N); the real-DFT
// table w_N^k (k < N/4); the type-2/3 table w_4N^n (n < N/2); the type-4
// tables w_2N^n (n < N/2) and w_8N^(2q+1) (q < N); and the coarse/fine pair
// of a long length (w_N^(a << lobits), w_N^c), lobits = ceil(log2 N / 2).
namespace tables {
enum TableKind : int { TB_TW = 0, TB_RFT, TB_T23, TB_T4PRE, TB_T4POST, TB_STHI, TB_STLO };
}

// Radix actually used by a kernel of length L requested with radix R.
inline int effective_radix(int L, int R) { return L < R ? L : R; }

// Raw input element size and raw elements per transform of the pipelined
// kernel of `combo` (complex or real input, L, L+1 or 2L elements).
int pipe_raw_size(int combo);
int pipe_raw_elems(int combo, int L);

}  // namespace mb
