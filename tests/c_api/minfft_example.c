/*
 * A C program written against the minfft C API exactly as the reference
 * library documents it (reference README.md "Interface"): host arrays, the
 * plan makers, the transforms and minfft_free_aux, with nothing from the B200
 * engine's extensions.  It builds unchanged against any library that exports
 * the minfft.h symbols.  The tests build it against the engine (run on a GPU)
 * and against the CPU oracle, which checks this program itself.
 *
 * Checks (relative L2 against sums of the definitions in long double, with
 * the roots of unity tabulated once):
 *   1-D complex DFT, N = 1024, and the inverse back to N x;
 *   2-D real DFT, 64 x 128 -> 64 x 65, and the inverse back to N1 N2 x;
 *   1-D DCT-2, N = 256, then DCT-3 back to 2N x;
 *   1-D DCT-4, N = 256, applied twice: 2N x.
 * Bars: 1e-13 in double, 1e-6 log2(N) in single (MINFFT_SINGLE).
 * Exit status: 0 all checks pass, 1 a result is off, 2 a plan maker returned
 * NULL (for the engine: no usable GPU).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "minfft.h"

#define PI 3.141592653589793238462643383279502884L

static unsigned long long g_state = 12345u;

/* uniform in [-1, 1) from a 64-bit LCG */
static double uniform(void)
{
    g_state = g_state * 6364136223846793005ull + 1442695040888963407ull;
    return (double)(g_state >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

static double bar(long n)
{
#if MINFFT_SINGLE
    return 1e-6 * log2((double)n);
#else
    (void)n;
    return 1e-13;
#endif
}

/* relative L2 distance between n reals a (scaled by s) and b */
static double rel_l2(const minfft_real *a, const long double *b, long n, long double s)
{
    long double num = 0, den = 0;
    long i;
    for (i = 0; i < n; ++i) {
        long double d = (long double)a[i] * s - b[i];
        num += d * d;
        den += b[i] * b[i];
    }
    return (double)sqrtl(num / den);
}

/* cos and sin of 2 pi m / M for m < M, in long double */
static void roots(long M, long double **c, long double **s)
{
    long m;
    *c = malloc((size_t)M * sizeof(long double));
    *s = malloc((size_t)M * sizeof(long double));
    if (!*c || !*s) {
        fprintf(stderr, "out of host memory\n");
        exit(3);
    }
    for (m = 0; m < M; ++m) {
        (*c)[m] = cosl(2 * PI * m / M);
        (*s)[m] = sinl(2 * PI * m / M);
    }
}

static int failures = 0;

static void check(const char *what, double err, long n)
{
    int ok = err <= bar(n);
    printf("%-44s rel L2 %.3e (bar %.1e) %s\n", what, err, bar(n), ok ? "ok" : "FAIL");
    if (!ok) ++failures;
}

static void *alloc(long n, size_t size)
{
    void *p = malloc((size_t)n * size);
    if (!p) {
        fprintf(stderr, "out of host memory\n");
        exit(3);
    }
    return p;
}

static int complex_dft(void)
{
    enum { N = 1024 };
    minfft_cmpl *x = alloc(N, sizeof(minfft_cmpl)), *y = alloc(N, sizeof(minfft_cmpl)),
                *z = alloc(N, sizeof(minfft_cmpl));
    long double *ref = alloc(2 * N, sizeof(long double)), *xin = alloc(2 * N, sizeof(long double)), *c, *s;
    minfft_aux *a;
    long k, n;
    roots(N, &c, &s);
    for (n = 0; n < N; ++n) {
        x[n][0] = (minfft_real)uniform();
        x[n][1] = (minfft_real)uniform();
        xin[2 * n] = x[n][0];
        xin[2 * n + 1] = x[n][1];
    }
    a = minfft_mkaux_dft_1d(N);
    if (!a) return 2;
    minfft_dft(x, y, a);
    minfft_invdft(y, z, a);
    minfft_free_aux(a);
    for (k = 0; k < N; ++k) {
        long double re = 0, im = 0;
        for (n = 0; n < N; ++n) { /* x_n e^(-2 pi i k n / N) */
            const long m = (k * n) % N;
            re += xin[2 * n] * c[m] + xin[2 * n + 1] * s[m];
            im += xin[2 * n + 1] * c[m] - xin[2 * n] * s[m];
        }
        ref[2 * k] = re;
        ref[2 * k + 1] = im;
    }
    check("dft 1024", rel_l2(&y[0][0], ref, 2 * N, 1), N);
    check("invdft(dft(x)) / N", rel_l2(&z[0][0], xin, 2 * N, 1.0L / N), N);
    free(x), free(y), free(z), free(ref), free(xin), free(c), free(s);
    return 0;
}

static int real_dft_2d(void)
{
    enum { N1 = 64, N2 = 128, H = N2 / 2 + 1 };
    minfft_real *x = alloc(N1 * N2, sizeof(minfft_real)), *y = alloc(N1 * N2, sizeof(minfft_real));
    minfft_cmpl *z = alloc(N1 * H, sizeof(minfft_cmpl));
    long double *ref = alloc(2 * N1 * H, sizeof(long double)), *xin = alloc(N1 * N2, sizeof(long double)), *c, *s;
    minfft_aux *a;
    long k1, k2, n1, n2;
    roots(N1 * N2, &c, &s);
    for (n1 = 0; n1 < N1 * N2; ++n1) {
        x[n1] = (minfft_real)uniform();
        xin[n1] = x[n1];
    }
    a = minfft_mkaux_realdft_2d(N1, N2);
    if (!a) return 2;
    minfft_realdft(x, z, a);
    for (k1 = 0; k1 < N1; ++k1)
        for (k2 = 0; k2 < H; ++k2) {
            long double re = 0, im = 0;
            for (n1 = 0; n1 < N1; ++n1)
                for (n2 = 0; n2 < N2; ++n2) { /* e^(-2 pi i (k1 n1 / N1 + k2 n2 / N2)) */
                    const long m = (((k1 * n1) % N1) * N2 + ((k2 * n2) % N2) * N1) % (N1 * N2);
                    re += xin[n1 * N2 + n2] * c[m];
                    im -= xin[n1 * N2 + n2] * s[m];
                }
            ref[2 * (k1 * H + k2)] = re;
            ref[2 * (k1 * H + k2) + 1] = im;
        }
    check("realdft 64 x 128", rel_l2(&z[0][0], ref, 2 * N1 * H, 1), N1 * N2);
    minfft_invrealdft(z, y, a);
    minfft_free_aux(a);
    check("invrealdft(realdft(x)) / (N1 N2)", rel_l2(y, xin, N1 * N2, 1.0L / (N1 * N2)), N1 * N2);
    free(x), free(y), free(z), free(ref), free(xin), free(c), free(s);
    return 0;
}

static int trig(void)
{
    enum { N = 256 };
    minfft_real *x = alloc(N, sizeof(minfft_real)), *y = alloc(N, sizeof(minfft_real)),
                *z = alloc(N, sizeof(minfft_real));
    long double *ref = alloc(N, sizeof(long double)), *xin = alloc(N, sizeof(long double)), *c, *s;
    minfft_aux *a;
    long k, n;
    roots(16 * N, &c, &s); /* cos(pi j / (8N)) = c[j] */
    for (n = 0; n < N; ++n) {
        x[n] = (minfft_real)uniform();
        xin[n] = x[n];
    }
    a = minfft_mkaux_t2t3_1d(N);
    if (!a) return 2;
    minfft_dct2(x, y, a);
    minfft_dct3(y, z, a);
    minfft_free_aux(a);
    for (k = 0; k < N; ++k) {
        long double acc = 0; /* cos(pi (n + 1/2) k / N) = cos(pi (8n + 4) k / (8N)) */
        for (n = 0; n < N; ++n) acc += xin[n] * c[((8 * n + 4) * k) % (16 * N)];
        ref[k] = 2 * acc;
    }
    check("dct2 256", rel_l2(y, ref, N, 1), N);
    check("dct3(dct2(x)) / 2N", rel_l2(z, xin, N, 1.0L / (2 * N)), N);
    a = minfft_mkaux_t4_1d(N);
    if (!a) return 2;
    minfft_dct4(x, y, a);
    minfft_dct4(y, z, a);
    minfft_free_aux(a);
    for (k = 0; k < N; ++k) {
        long double acc = 0; /* cos(pi (n + 1/2) (k + 1/2) / N) = cos(pi (2n + 1) (2k + 1) 2 / (8N)) */
        for (n = 0; n < N; ++n) acc += xin[n] * c[(2 * (2 * n + 1) * (2 * k + 1)) % (16 * N)];
        ref[k] = 2 * acc;
    }
    check("dct4 256", rel_l2(y, ref, N, 1), N);
    check("dct4(dct4(x)) / 2N", rel_l2(z, xin, N, 1.0L / (2 * N)), N);
    free(x), free(y), free(z), free(ref), free(xin), free(c), free(s);
    return 0;
}

int main(void)
{
    if (complex_dft() || real_dft_2d() || trig()) {
        printf("a plan maker returned NULL\n");
        return 2;
    }
    minfft_free_aux(NULL); /* NULL is ignored, as in the reference */
    return failures ? 1 : 0;
}
