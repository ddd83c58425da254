// Interface of the standalone line kernels (line_kernels.cu).
#pragma once

#include <stdint.h>

#include "common.cuh"

namespace mb {

struct LineParams {
  const void* in;
  void* out;
  int64_t outer, inner;
  int64_t L;  // complex length of the lines (element count for LK_UNIT)
  int64_t in_so, in_sn, out_so, out_sn;
  const cpx* t1;
  const cpx* t2;
  // optional coarse/fine form of t1 and t2 for long lines: entry i of table
  // k is the root w^e, e = mul_k*i + add_k, read as hi_k[e >> bits_k] *
  // lo_k[e & (2^bits_k - 1)] instead of a table of the full line length
  const cpx* hi1;
  const cpx* lo1;
  const cpx* hi2;
  const cpx* lo2;
  int bits1, mul1, add1;
  int bits2, mul2, add2;
  int flags;
  int mode;
  real scale;
};

enum LineKernel : int {
  LK_DCT2_PRE = 0,
  LK_T4_PRE,
  LK_C2R_PACK,
  LK_DCT3_PACK,
  LK_R2C_UNPACK,
  LK_DCT2_POST,
  LK_DCT3_POST,
  LK_T4_POST,
  LK_UNIT,
  LK_COUNT
};

enum UnitMode : int { UNIT_SCALE_REAL = 0, UNIT_REAL_TO_CPLX, UNIT_CPLX_TO_REAL, UNIT_COPY_CPLX };

const void* line_kernel(int which);

}  // namespace mb
