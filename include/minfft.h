/*
 * minfft.h -- public C interface of the B200 transform engine.
 *
 * Source-compatible drop-in for the header of the minimalist FFT library
 * aimukhin/minfft (reference file minfft.h).  Every type and prototype below
 * has the same name, argument order and meaning as there, so code written
 * against that library (C, C++, or its Fortran bind(C) module) links against
 * libminfft_b200.so (double) or libminfft_b200_single.so (MINFFT_SINGLE)
 * without changes.
 *
 * What differs is where the work runs: every transform executes as CUDA
 * kernels on the current GPU.  Data pointers may be device, managed or host
 * addresses (host data is staged through device memory and the call returns
 * when the result is back in host memory).  Extensions -- streams, batching,
 * error reporting, the split-precision tensor-core mode and the mixed-batch
 * launcher -- live in minfft_b200.h.
 */
#ifndef MINFFT_H
#define MINFFT_H

#ifdef __cplusplus
extern "C" {
#endif

/* precision and complex type selection: reference minfft.h:14-31 */
#ifdef complex
#if MINFFT_SINGLE
typedef float minfft_real;
typedef float complex minfft_cmpl;
#else
typedef double minfft_real;
typedef double complex minfft_cmpl;
#endif
#else
#if MINFFT_SINGLE
typedef float minfft_real;
#else
typedef double minfft_real;
#endif
/* interleaved (re, im) pair, binary-compatible with float2/double2 */
typedef minfft_real minfft_cmpl[2];
#endif

/* opaque plan ("auxiliary data"): reference minfft.h:33 */
typedef struct minfft_aux minfft_aux;

/*
 * Transforms: reference minfft.h:35-44 (minfft.c:287, 503, 582, 662, 735,
 * 784, 834, 884, 931, 978).  Arguments: input x, output y, plan a.  In-place
 * (x == y) and out-of-place calls are both allowed; out of place, the input
 * is left intact -- including the multi-dimensional inverse real DFT, which
 * the reference is allowed to clobber (README "Inverse real DFT").
 * Definitions are unnormalised and FFTW-compatible (reference README.md
 * "Transforms").
 */
void minfft_dft(minfft_cmpl *x, minfft_cmpl *y, const minfft_aux *a);
void minfft_invdft(minfft_cmpl *x, minfft_cmpl *y, const minfft_aux *a);
void minfft_realdft(minfft_real *x, minfft_cmpl *z, const minfft_aux *a);
void minfft_invrealdft(minfft_cmpl *z, minfft_real *y, const minfft_aux *a);
void minfft_dct2(minfft_real *x, minfft_real *y, const minfft_aux *a);
void minfft_dst2(minfft_real *x, minfft_real *y, const minfft_aux *a);
void minfft_dct3(minfft_real *x, minfft_real *y, const minfft_aux *a);
void minfft_dst3(minfft_real *x, minfft_real *y, const minfft_aux *a);
void minfft_dct4(minfft_real *x, minfft_real *y, const minfft_aux *a);
void minfft_dst4(minfft_real *x, minfft_real *y, const minfft_aux *a);

/*
 * Plan makers: reference minfft.h:46-61 (minfft.c:1057-1335).  Dimensions
 * are in C order (last index fastest).  A maker returns NULL when a length
 * is not a positive power of two, when d < 1, or when device memory cannot
 * be allocated.  One plan serves the forward and inverse transform of its
 * kind: dft/invdft, realdft/invrealdft, dct2/dst2/dct3/dst3 (t2t3), and
 * dct4/dst4 (t4).  The plan holds device-resident twiddle tables and scratch
 * buffers; like the reference's, one plan must not run two transforms at once.
 */
minfft_aux *minfft_mkaux_dft_1d(int N);
minfft_aux *minfft_mkaux_dft_2d(int N1, int N2);
minfft_aux *minfft_mkaux_dft_3d(int N1, int N2, int N3);
minfft_aux *minfft_mkaux_dft(int d, int *Ns);
minfft_aux *minfft_mkaux_realdft_1d(int N);
minfft_aux *minfft_mkaux_realdft_2d(int N1, int N2);
minfft_aux *minfft_mkaux_realdft_3d(int N1, int N2, int N3);
minfft_aux *minfft_mkaux_realdft(int d, int *Ns);
minfft_aux *minfft_mkaux_t2t3_1d(int N);
minfft_aux *minfft_mkaux_t2t3_2d(int N1, int N2);
minfft_aux *minfft_mkaux_t2t3_3d(int N1, int N2, int N3);
minfft_aux *minfft_mkaux_t2t3(int d, int *Ns);
minfft_aux *minfft_mkaux_t4_1d(int N);
minfft_aux *minfft_mkaux_t4_2d(int N1, int N2);
minfft_aux *minfft_mkaux_t4_3d(int N1, int N2, int N3);
minfft_aux *minfft_mkaux_t4(int d, int *Ns);

/* release a plan and its device memory; NULL is ignored (reference minfft.c:1338-1347) */
void minfft_free_aux(minfft_aux *a);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* MINFFT_H */
