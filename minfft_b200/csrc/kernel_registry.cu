// Dispatch from (combo, log2 L) to the instantiated axis-pass kernels; the
// instantiations live in one translation unit per combo (kernels_*.cu) so
// they compile in parallel.
#include "kernel_registry.h"

#include "common.cuh"

namespace mb {

const void* axis_kernel_cplx(int log2L, int radix16);
const void* axis_kernel_r2c(int log2L, int radix16);
const void* axis_kernel_c2r(int log2L, int radix16);
const void* axis_kernel_dct2(int log2L, int radix16);
const void* axis_kernel_dct3(int log2L, int radix16);
const void* axis_kernel_t4(int log2L, int radix16);
const void* axis_kernel_r2cq(int log2L, int radix16);
const void* axis_kernel_c2rq(int log2L, int radix16);
const void* axis_kernel_t4in(int log2L, int radix16);
const void* axis_kernel_t4out(int log2L, int radix16);

const void* pipe_kernel_cplx(int log2L, int radix16);
const void* pipe_kernel_r2c(int log2L, int radix16);
const void* pipe_kernel_c2r(int log2L, int radix16);
const void* pipe_kernel_dct2(int log2L, int radix16);
const void* pipe_kernel_dct3(int log2L, int radix16);
const void* pipe_kernel_t4(int log2L, int radix16);

const void* pipe_kernel(int combo, int log2L, int R) {
  if (log2L < 1) return nullptr;
  switch (combo) {
    case K_CPLX: return pipe_kernel_cplx(log2L, R >= 16);
    case K_R2C: return pipe_kernel_r2c(log2L, R >= 16);
    case K_C2R: return pipe_kernel_c2r(log2L, R >= 16);
    case K_DCT2: return pipe_kernel_dct2(log2L, R >= 16);
    case K_DCT3: return pipe_kernel_dct3(log2L, R >= 16);
    case K_T4: return pipe_kernel_t4(log2L, R >= 16);
    default: return nullptr;
  }
}

int pipe_raw_size(int combo) {
  return (combo == K_CPLX || combo == K_C2R) ? int(sizeof(cpx)) : int(sizeof(real));
}

int pipe_raw_elems(int combo, int L) {
  switch (combo) {
    case K_CPLX: return L;
    case K_C2R: return L + 1;
    default: return 2 * L;
  }
}

const void* axis_kernel(int combo, int log2L, int R) {
  switch (combo) {
    case K_CPLX: return axis_kernel_cplx(log2L, R >= 16);
    case K_R2C: return axis_kernel_r2c(log2L, R >= 16);
    case K_C2R: return axis_kernel_c2r(log2L, R >= 16);
    case K_DCT2: return axis_kernel_dct2(log2L, R >= 16);
    case K_DCT3: return axis_kernel_dct3(log2L, R >= 16);
    case K_T4: return axis_kernel_t4(log2L, R >= 16);
    case K_R2CQ: return axis_kernel_r2cq(log2L, R >= 16);
    case K_C2RQ: return axis_kernel_c2rq(log2L, R >= 16);
    case K_T4IN: return axis_kernel_t4in(log2L, R >= 16);
    case K_T4OUT: return axis_kernel_t4out(log2L, R >= 16);
    default: return nullptr;
  }
}

}  // namespace mb
