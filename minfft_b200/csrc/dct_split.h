// Split column DFT of the 2-D DCT-2/DST-2 and DCT-3/DST-3 (dct_split.cu):
// kernel parameters and the kernel table.
#pragma once

#include <stddef.h>

#include "common.cuh"

namespace mb {

struct DctqParams {
  const void* in;
  void* out;
  cpx* mid;           // blocks: (h, q, j, n) at ((h*4 + q)*Q + j)*N + n
  int64_t H, Nr, N, Q;
  int flags;          // F_DST
  int lp;             // tile pitch of the kernel's shared-memory tile
  int W;              // column pass: adjacent columns per CTA
  const cpx* tw_row;  // w_L^m, L = N/2 (row DFTs)
  const cpx* rft_row; // w_N^k (row real DFT)
  const cpx* t23_row; // w_4N^n (row type-2/3 roots)
  const cpx* tw_c;    // w_Lc^m (the radix-4 stage's twiddles)
  const cpx* tw_q;    // w_Q^m (column DFTs)
  const cpx* rft_c;   // w_Nr^k (column real DFT)
  const cpx* t23_c;   // w_4Nr^n (column type-2/3 roots)
};

// which = 0 row pass forward, 1 column pass forward, 2 column pass inverse,
// 3 row pass inverse; log2 of the row half-length L (6 .. 10) or of the
// column block length Q (6 .. 9); nullptr otherwise.  Launch with one
// argument (DctqParams); rows: grid H*Q, 8*L/16 threads, dctq_row_smem(L)
// bytes; columns: grid H*2*(N/W), 2*W*Q/16 threads, dctq_col_smem(Q, W).
const void* dctq_kernel(int which, int log2len);
size_t dctq_row_smem(int L);
size_t dctq_col_smem(int QL, int W);

}  // namespace mb
