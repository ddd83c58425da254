/*
 * CPU oracle for the minfft transform family -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is a restatement, in plain C, of the algorithms of the reference
 * library (aimukhin/minfft, file minfft.c).  It is the checker the GPU engine
 * is compared against; nothing in the product links it.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * It exports the same 27 symbols as the reference header minfft.h, so a single
 * ctypes binding drives the reference build, this restatement and the GPU
 * library alike.  Build twice: plain (double) and with -DMINFFT_SINGLE=1.
 *
 * Parity pin: tests/test_oracle.py checks this file against golden vectors
 * produced by the compiled reference (tests/golden/, generator
 * tests/golden/make_golden.py) and, where oracle/_ref/ exists, against the
 * compiled reference directly.
 *
 * Algorithm map (reference minfft.c line numbers):
 *   unit roots with octant folding ........ ncos/nsin            989-1018
 *   split-radix DIF complex DFT ........... rs_dft_1d/rs_invdft_1d 77-488
 *   transposing multi-D recursion ......... mkcx/mkrx             33-72
 *   real DFT (half-length complex + unpack) s_realdft_1d          511-579
 *   inverse real DFT (pack + half-length) . invrealdft_1d         600-659
 *   multi-D real / inverse real DFT ....... minfft_(inv)realdft   582-597, 662-687
 *   DCT-2/DST-2, DCT-3/DST-3, DCT-4/DST-4 . s_dct2_1d..s_dst4_1d  692-969
 *   plan makers ........................... make_aux, mkaux_*     1024-1347
 */
#include <stdlib.h>
#include <string.h>
#include <math.h>

#if defined(_WIN32)
#define ORACLE_API __declspec(dllexport)
#else
#define ORACLE_API __attribute__((visibility("default")))
#endif

#if MINFFT_SINGLE
typedef float real_t;
#else
typedef double real_t;
#endif

typedef struct { real_t re, im; } cpx;

/* pi and sqrt(2) rounded once to the working precision (minfft.c:12-14) */
static const real_t k_pi = (real_t)3.141592653589793238462643383279502884L;
static const real_t k_sqrt2 = (real_t)1.414213562373095048801688724209698079L;

/* ------------------------------------------------------------------ */
/* complex helpers                                                    */
/* ------------------------------------------------------------------ */

static cpx c_make(real_t re, real_t im) { cpx z; z.re = re; z.im = im; return z; }
static cpx c_add(cpx a, cpx b) { return c_make(a.re + b.re, a.im + b.im); }
static cpx c_sub(cpx a, cpx b) { return c_make(a.re - b.re, a.im - b.im); }
static cpx c_mul(cpx a, cpx b) { return c_make(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
/* a * conj(b) */
static cpx c_mulc(cpx a, cpx b) { return c_make(a.re * b.re + a.im * b.im, a.im * b.re - a.re * b.im); }
static cpx c_conj(cpx a) { return c_make(a.re, -a.im); }
/* multiply by +i */
static cpx c_ipos(cpx a) { return c_make(-a.im, a.re); }

/* ------------------------------------------------------------------ */
/* unit roots: (cos, sin)(2*pi*n/N) with the angle folded into the    */
/* first octant before libm is called (minfft.c:989-1018).  The       */
/* angle 2*pi*n/N is formed in the working precision, as there.  The  */
/* folding tests 2n >= N, 4n >= N, 8n > N equal the reference's for   */
/* N >= 8 and also terminate for N < 8.                               */
/* ------------------------------------------------------------------ */

static cpx unit_root(long n, long N)
{
    cpx r;
    real_t s;
    if (n < 0) {                       /* odd symmetry of sin */
        r = unit_root(-n, N);
        r.im = -r.im;
        return r;
    }
    if (2 * n >= N) {                  /* rotate by pi */
        r = unit_root(n - N / 2, N);
        r.re = -r.re;
        r.im = -r.im;
        return r;
    }
    if (4 * n >= N) {                  /* rotate by pi/2 */
        r = unit_root(n - N / 4, N);
        s = r.re;
        r.re = -r.im;
        r.im = s;
        return r;
    }
    if (8 * n > N) {                   /* reflect about pi/4 */
        r = unit_root(N / 4 - n, N);
        s = r.re;
        r.re = r.im;
        r.im = s;
        return r;
    }
    {
        real_t ang = 2 * k_pi * (real_t)n / (real_t)N;
        r.re = (real_t)cos(ang);
        r.im = (real_t)sin(ang);
    }
    return r;
}

/* ------------------------------------------------------------------ */
/* plan tree (minfft.c:17-22): length, work buffer, root table, and   */
/* two children.  For a multi-D plan `inner` covers the trailing      */
/* dimensions and `outer` the leading one, as in the reference.       */
/* ------------------------------------------------------------------ */

struct minfft_aux {
    int n;                     /* elements transformed by this node */
    void *work;                /* scratch buffer */
    cpx *roots;                /* precomputed unit roots */
    struct minfft_aux *inner;  /* sub1 */
    struct minfft_aux *outer;  /* sub2 */
};
typedef struct minfft_aux minfft_aux;

ORACLE_API void minfft_free_aux(minfft_aux *a);

static minfft_aux *node_new(int n)
{
    minfft_aux *a = (minfft_aux *)calloc(1, sizeof(minfft_aux));
    if (a) a->n = n;
    return a;
}

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* ------------------------------------------------------------------ */
/* split-radix decimation-in-frequency complex DFT                    */
/* (minfft.c:77-272 forward, 293-488 inverse).  One level splits the  */
/* input into sums (length M/2) and two twiddled differences          */
/* (length M/4 each); the leaves scatter with growing output stride.  */
/* `sign` = -1 forward, +1 inverse.  Root table of level M sits at    */
/* offset (N - M) of the top-level table, 2 roots per quad index.     */
/* ------------------------------------------------------------------ */

static void sr_leaf(int M, const cpx *x, cpx *y, long sy, int sign)
{
    /* direct butterflies for M = 1, 2, 4, 8 (minfft.c:82-231) */
    if (M == 1) {
        y[0] = x[0];
    } else if (M == 2) {
        cpx a = x[0], b = x[1];
        y[0] = c_add(a, b);
        y[sy] = c_sub(a, b);
    } else if (M == 4) {
        cpx s0 = c_add(x[0], x[2]), s1 = c_add(x[1], x[3]);
        cpx d0 = c_sub(x[0], x[2]), d1 = c_ipos(c_sub(x[1], x[3]));
        y[0] = c_add(s0, s1);
        y[2 * sy] = c_sub(s0, s1);
        if (sign < 0) {
            y[sy] = c_sub(d0, d1);
            y[3 * sy] = c_add(d0, d1);
        } else {
            y[sy] = c_add(d0, d1);
            y[3 * sy] = c_sub(d0, d1);
        }
    } else { /* M == 8: radix-2 split into two length-4 halves */
        const real_t h = (real_t)0.707106781186547524400844362104849039L;
        cpx e[4], o[4], eo[4], oo[4];
        int k;
        for (k = 0; k < 4; ++k) {
            e[k] = x[2 * k];
            o[k] = x[2 * k + 1];
        }
        sr_leaf(4, e, eo, 1, sign);
        sr_leaf(4, o, oo, 1, sign);
        /* odd half times w8^k: w8^1 = h(1, sign), w8^2 = (0, sign), w8^3 = h(-1, sign) */
        oo[1] = c_make(h * (oo[1].re - sign * oo[1].im), h * (oo[1].im + sign * oo[1].re));
        oo[2] = c_mul(oo[2], c_make(0, (real_t)sign));
        oo[3] = c_make(-h * (oo[3].re + sign * oo[3].im), h * (sign * oo[3].re - oo[3].im));
        for (k = 0; k < 4; ++k) {
            y[k * sy] = c_add(eo[k], oo[k]);
            y[(k + 4) * sy] = c_sub(eo[k], oo[k]);
        }
    }
}

static void sr_dft(int M, const cpx *x, cpx *t, cpx *y, long sy, const cpx *w, int sign)
{
    int q, n;
    if (M <= 8) {
        sr_leaf(M, x, y, sy, sign);
        return;
    }
    q = M / 4;
    for (n = 0; n < q; ++n) {
        cpx a = x[n], b = x[n + q], c = x[n + 2 * q], d = x[n + 3 * q];
        cpx dif = c_sub(a, c);
        cpx rot = c_ipos(c_sub(b, d));
        cpx lo, hi;
        t[n] = c_add(a, c);
        t[n + q] = c_add(b, d);
        if (sign < 0) {
            lo = c_mul(c_sub(dif, rot), w[2 * n]);
            hi = c_mul(c_add(dif, rot), w[2 * n + 1]);
        } else {
            lo = c_mulc(c_add(dif, rot), w[2 * n]);
            hi = c_mulc(c_sub(dif, rot), w[2 * n + 1]);
        }
        t[n + 2 * q] = lo;
        t[n + 3 * q] = hi;
    }
    /* sub-tables: level M/2 at w + M/2, level M/4 at w + 3M/4 (in cpx units) */
    sr_dft(M / 2, t, t, y, 2 * sy, w + M / 2, sign);
    sr_dft(q, t + 2 * q, t + 2 * q, y + sy, 4 * sy, w + 3 * q, sign);
    sr_dft(q, t + 3 * q, t + 3 * q, y + 3 * sy, 4 * sy, w + 3 * q, sign);
}

typedef void (*cx_line_fn)(const cpx *, cpx *, long, const minfft_aux *);
typedef void (*rx_line_fn)(const real_t *, real_t *, long, const minfft_aux *);

static void line_dft(const cpx *x, cpx *y, long sy, const minfft_aux *a)
{
    sr_dft(a->n, x, (cpx *)a->work, y, sy, a->roots, -1);
}

static void line_invdft(const cpx *x, cpx *y, long sy, const minfft_aux *a)
{
    sr_dft(a->n, x, (cpx *)a->work, y, sy, a->roots, +1);
}

/* transposing multi-D recursion (minfft.c:33-48 complex, 57-72 real):  */
/* each leading-index hyperplane is transformed into work[] with stride */
/* n_outer, then rows of work[] are transformed along the leading axis. */
static void nd_complex(const cpx *x, cpx *y, long sy, const minfft_aux *a, cx_line_fn f)
{
    if (a->outer == NULL) {
        f(x, y, sy, a);
    } else {
        long n_in = a->inner->n, n_out = a->outer->n, i;
        cpx *w = (cpx *)a->work;
        for (i = 0; i < n_out; ++i) nd_complex(x + i * n_in, w + i, n_out, a->inner, f);
        for (i = 0; i < n_in; ++i) f(w + i * n_out, y + sy * i, sy * n_in, a->outer);
    }
}

static void nd_real(const real_t *x, real_t *y, long sy, const minfft_aux *a, rx_line_fn f)
{
    if (a->outer == NULL) {
        f(x, y, sy, a);
    } else {
        long n_in = a->inner->n, n_out = a->outer->n, i;
        real_t *w = (real_t *)a->work;
        for (i = 0; i < n_out; ++i) nd_real(x + i * n_in, w + i, n_out, a->inner, f);
        for (i = 0; i < n_in; ++i) f(w + i * n_out, y + sy * i, sy * n_in, a->outer);
    }
}

ORACLE_API void minfft_dft(cpx *x, cpx *y, const minfft_aux *a) { nd_complex(x, y, 1, a, line_dft); }
ORACLE_API void minfft_invdft(cpx *x, cpx *y, const minfft_aux *a) { nd_complex(x, y, 1, a, line_invdft); }

/* ------------------------------------------------------------------ */
/* real DFT of length N (minfft.c:511-579): N reals read as N/2       */
/* complex, a half-length complex DFT, then an unpacking pass that    */
/* separates the even/odd spectra with roots w_N^k (k < N/4).         */
/* ------------------------------------------------------------------ */

static void line_realdft(const real_t *x, cpx *z, long sz, const minfft_aux *a)
{
    long N = a->n, h, k;
    const cpx *T;
    if (N == 1) {
        z[0] = c_make(x[0], 0);
        return;
    }
    if (N == 2) {
        real_t p = x[0], q = x[1];
        z[0] = c_make(p + q, 0);
        z[sz] = c_make(p - q, 0);
        return;
    }
    h = N / 2;
    sr_dft((int)h, (const cpx *)x, (cpx *)a->inner->work, (cpx *)a->work, 1, a->inner->roots, -1);
    T = (const cpx *)a->work;
    z[0] = c_make(T[0].re + T[0].im, 0);
    z[sz * h] = c_make(T[0].re - T[0].im, 0);
    for (k = 1; k < N / 4; ++k) {
        cpx p = T[k], m = c_conj(T[h - k]);
        cpx u = c_make((p.re + m.re) / 2, (p.im + m.im) / 2);
        cpx d = c_sub(p, m);
        /* root / (2i) = (w.im, -w.re) / 2 */
        cpx wr = c_make(a->roots[k].im, -a->roots[k].re);
        cpx v = c_mul(d, wr);
        v.re /= 2;
        v.im /= 2;
        z[sz * k] = c_add(u, v);
        z[sz * (h - k)] = c_conj(c_sub(u, v));
    }
    z[sz * (N / 4)] = c_conj(T[N / 4]);
}

ORACLE_API void minfft_realdft(real_t *x, cpx *z, const minfft_aux *a)
{
    if (a->outer == NULL) {
        line_realdft(x, z, 1, a);
    } else {
        /* rows of the last axis into work[] transposed, then the (d-1)-D */
        /* complex DFT of every frequency column (minfft.c:582-597)       */
        long n_last = a->inner->n, n_lead = a->outer->n, n_half = n_last / 2 + 1, i;
        cpx *w = (cpx *)a->work;
        for (i = 0; i < n_lead; ++i) line_realdft(x + i * n_last, w + i, n_lead, a->inner);
        for (i = 0; i < n_half; ++i) nd_complex(w + i * n_lead, z + i, n_half, a->outer, line_dft);
    }
}

/* inverse real DFT of length N (minfft.c:600-659), unnormalised */
static void line_invrealdft(const cpx *z, real_t *y, const minfft_aux *a)
{
    long N = a->n, h, k;
    cpx *t;
    if (N == 1) {
        y[0] = z[0].re;
        return;
    }
    if (N == 2) {
        real_t p = z[0].re, q = z[1].re;
        y[0] = p + q;
        y[1] = p - q;
        return;
    }
    h = N / 2;
    t = (cpx *)a->work;
    t[0] = c_make(z[0].re + z[h].re, z[0].re - z[h].re);
    for (k = 1; k < N / 4; ++k) {
        cpx p = z[k], m = c_conj(z[h - k]);
        cpx u = c_add(p, m);
        cpx d = c_sub(p, m);
        /* i * conj(root) = (w.im, w.re) */
        cpx wr = c_make(a->roots[k].im, a->roots[k].re);
        cpx v = c_mul(d, wr);
        t[k] = c_add(u, v);
        t[h - k] = c_conj(c_sub(u, v));
    }
    t[N / 4] = c_make(2 * z[N / 4].re, -2 * z[N / 4].im);
    sr_dft((int)h, t, (cpx *)a->inner->work, (cpx *)y, 1, a->inner->roots, +1);
}

ORACLE_API void minfft_invrealdft(cpx *z, real_t *y, const minfft_aux *a)
{
    if (a->outer == NULL) {
        line_invrealdft(z, y, a);
    } else {
        /* transpose z into work[], inverse (d-1)-D DFT of each column back */
        /* into z (input destroyed, as in minfft.c:662-687), then rows      */
        long n_last = a->inner->n, n_lead = a->outer->n, n_half = n_last / 2 + 1, i, k;
        cpx *w = (cpx *)a->work;
        for (i = 0; i < n_lead; ++i)
            for (k = 0; k < n_half; ++k) w[i + n_lead * k] = z[n_half * i + k];
        for (i = 0; i < n_half; ++i) nd_complex(w + i * n_lead, z + i, n_half, a->outer, line_invdft);
        for (i = 0; i < n_lead; ++i) line_invrealdft(z + i * n_half, y + i * n_last, a->inner);
    }
}

/* ------------------------------------------------------------------ */
/* type-2 and type-3 transforms (minfft.c:692-887).  Both reduce to a */
/* real DFT (or its inverse) of the same length N with roots          */
/* w_{4N}^n, n < N/2.  `dst` selects the sine variant.                */
/* ------------------------------------------------------------------ */

static void t2_line(const real_t *x, real_t *y, long sy, const minfft_aux *a, int dst)
{
    long N = a->n, n;
    real_t *v = (real_t *)a->work;
    cpx *V = (cpx *)a->work;
    real_t sg = dst ? -1 : 1;
    if (N == 1) {
        y[0] = 2 * x[0];
        return;
    }
    /* even samples ascending, odd samples descending (DST negates them) */
    for (n = 0; n < N / 2; ++n) {
        v[n] = x[2 * n];
        v[N / 2 + n] = sg * x[N - 1 - 2 * n];
    }
    {
        /* real DFT in the same buffer: copy the input row aside first */
        real_t *row = v + N + 2;
        memcpy(row, v, (size_t)N * sizeof(real_t));
        line_realdft(row, V, 1, a->inner);
    }
    if (!dst) {
        y[0] = 2 * V[0].re;
        for (n = 1; n < N / 2; ++n) {
            cpx r = c_mul(V[n], a->roots[n]);
            y[sy * n] = 2 * r.re;
            y[sy * (N - n)] = -2 * r.im;
        }
        y[sy * (N / 2)] = k_sqrt2 * V[N / 2].re;
    } else {
        y[sy * (N - 1)] = 2 * V[0].re;
        for (n = 1; n < N / 2; ++n) {
            cpx r = c_mul(V[n], a->roots[n]);
            y[sy * (n - 1)] = -2 * r.im;
            y[sy * (N - n - 1)] = 2 * r.re;
        }
        y[sy * (N / 2 - 1)] = k_sqrt2 * V[N / 2].re;
    }
}

static void t3_line(const real_t *x, real_t *y, long sy, const minfft_aux *a, int dst)
{
    long N = a->n, n;
    cpx *Z = (cpx *)a->work;
    real_t *out = (real_t *)a->work + N + 2;
    if (N == 1) {
        y[0] = x[0];
        return;
    }
    if (!dst) {
        Z[0] = c_make(x[0], 0);
        for (n = 1; n < N / 2; ++n) Z[n] = c_conj(c_mul(c_make(x[n], x[N - n]), a->roots[n]));
        Z[N / 2] = c_make(k_sqrt2 * x[N / 2], 0);
    } else {
        Z[0] = c_make(x[N - 1], 0);
        for (n = 1; n < N / 2; ++n) Z[n] = c_conj(c_mul(c_make(x[N - n - 1], x[n - 1]), a->roots[n]));
        Z[N / 2] = c_make(k_sqrt2 * x[N / 2 - 1], 0);
    }
    line_invrealdft(Z, out, a->inner);
    for (n = 0; n < N / 2; ++n) {
        y[sy * 2 * n] = out[n];
        y[sy * (N - 1 - 2 * n)] = dst ? -out[N / 2 + n] : out[N / 2 + n];
    }
}

static void line_dct2(const real_t *x, real_t *y, long sy, const minfft_aux *a) { t2_line(x, y, sy, a, 0); }
static void line_dst2(const real_t *x, real_t *y, long sy, const minfft_aux *a) { t2_line(x, y, sy, a, 1); }
static void line_dct3(const real_t *x, real_t *y, long sy, const minfft_aux *a) { t3_line(x, y, sy, a, 0); }
static void line_dst3(const real_t *x, real_t *y, long sy, const minfft_aux *a) { t3_line(x, y, sy, a, 1); }

ORACLE_API void minfft_dct2(real_t *x, real_t *y, const minfft_aux *a) { nd_real(x, y, 1, a, line_dct2); }
ORACLE_API void minfft_dst2(real_t *x, real_t *y, const minfft_aux *a) { nd_real(x, y, 1, a, line_dst2); }
ORACLE_API void minfft_dct3(real_t *x, real_t *y, const minfft_aux *a) { nd_real(x, y, 1, a, line_dct3); }
ORACLE_API void minfft_dst3(real_t *x, real_t *y, const minfft_aux *a) { nd_real(x, y, 1, a, line_dst3); }

/* ------------------------------------------------------------------ */
/* type-4 transforms (minfft.c:890-981): pre-rotation by w_{2N}^n,    */
/* complex DFT of length N/2, post-rotation by w_{8N}^(2m+1).         */
/* ------------------------------------------------------------------ */

static void t4_line(const real_t *x, real_t *y, long sy, const minfft_aux *a, int dst)
{
    long N = a->n, h, n;
    cpx *t = (cpx *)a->work;
    cpx *T = t + N / 2;
    const cpx *pre = a->roots, *post = a->roots + N / 2;
    if (N == 1) {
        y[0] = k_sqrt2 * x[0];
        return;
    }
    h = N / 2;
    for (n = 0; n < h; ++n) {
        if (!dst) {
            t[n] = c_mul(pre[n], c_make(x[2 * n], x[N - 1 - 2 * n]));
        } else {
            cpx r = c_mul(pre[n], c_make(x[2 * n], -x[N - 1 - 2 * n]));
            t[n] = c_make(-r.re, -r.im);
        }
    }
    sr_dft((int)h, t, (cpx *)a->inner->work, T, 1, a->inner->roots, -1);
    for (n = 0; n < h; ++n) {
        cpx e0 = post[2 * n], e1 = post[2 * n + 1];
        cpx q0 = T[n], q1 = c_conj(T[h - 1 - n]);
        if (!dst) {
            y[sy * 2 * n] = 2 * c_mul(e0, q0).re;
            y[sy * (2 * n + 1)] = 2 * c_mul(e1, q1).re;
        } else {
            y[sy * 2 * n] = 2 * c_mul(e0, q0).im;
            y[sy * (2 * n + 1)] = 2 * c_mul(e1, q1).im;
        }
    }
}

static void line_dct4(const real_t *x, real_t *y, long sy, const minfft_aux *a) { t4_line(x, y, sy, a, 0); }
static void line_dst4(const real_t *x, real_t *y, long sy, const minfft_aux *a) { t4_line(x, y, sy, a, 1); }

ORACLE_API void minfft_dct4(real_t *x, real_t *y, const minfft_aux *a) { nd_real(x, y, 1, a, line_dct4); }
ORACLE_API void minfft_dst4(real_t *x, real_t *y, const minfft_aux *a) { nd_real(x, y, 1, a, line_dst4); }

/* ------------------------------------------------------------------ */
/* plan makers (minfft.c:1024-1335).  Every maker returns NULL on a   */
/* non-positive or non-power-of-two length and on allocation failure; */
/* unlike the reference, a partly built tree is always zero-filled so */
/* the cleanup path never frees an uninitialised pointer, and d < 1   */
/* is rejected instead of recursing without bound.                    */
/* ------------------------------------------------------------------ */

ORACLE_API minfft_aux *minfft_mkaux_dft_1d(int N)
{
    minfft_aux *a;
    cpx *w;
    int M, n;
    if (!is_pow2(N)) return NULL;
    a = node_new(N);
    if (!a) return NULL;
    if (N >= 16) {
        a->work = malloc((size_t)N * sizeof(cpx));
        a->roots = (cpx *)malloc((size_t)N * sizeof(cpx));
        if (!a->work || !a->roots) goto fail;
        /* per level M = N, N/2, ..., 16: {w_M^-n, w_M^-3n}, n < M/4 */
        w = a->roots;
        for (M = N; M >= 16; M /= 2)
            for (n = 0; n < M / 4; ++n) {
                *w++ = unit_root(-n, M);
                *w++ = unit_root(-3 * n, M);
            }
    }
    return a;
fail:
    minfft_free_aux(a);
    return NULL;
}

ORACLE_API minfft_aux *minfft_mkaux_realdft_1d(int N)
{
    minfft_aux *a;
    int n;
    if (!is_pow2(N)) return NULL;
    a = node_new(N);
    if (!a) return NULL;
    if (N >= 4) {
        a->work = malloc((size_t)(N / 2) * sizeof(cpx));
        a->roots = (cpx *)malloc((size_t)(N / 4) * sizeof(cpx));
        a->inner = minfft_mkaux_dft_1d(N / 2);
        if (!a->work || !a->roots || !a->inner) goto fail;
        for (n = 0; n < N / 4; ++n) a->roots[n] = unit_root(-n, N);
    }
    return a;
fail:
    minfft_free_aux(a);
    return NULL;
}

ORACLE_API minfft_aux *minfft_mkaux_t2t3_1d(int N)
{
    minfft_aux *a;
    int n;
    if (!is_pow2(N)) return NULL;
    a = node_new(N);
    if (!a) return NULL;
    if (N >= 2) {
        /* N+2 reals for the in-buffer real DFT plus N reals of row copy */
        a->work = malloc((size_t)(2 * N + 4) * sizeof(real_t));
        a->roots = (cpx *)malloc((size_t)(N / 2) * sizeof(cpx));
        if (!a->work || !a->roots) goto fail;
        for (n = 0; n < N / 2; ++n) a->roots[n] = unit_root(-n, 4 * N);
    }
    a->inner = minfft_mkaux_realdft_1d(N);
    if (!a->inner) goto fail;
    return a;
fail:
    minfft_free_aux(a);
    return NULL;
}

ORACLE_API minfft_aux *minfft_mkaux_t4_1d(int N)
{
    minfft_aux *a;
    int n;
    if (!is_pow2(N)) return NULL;
    a = node_new(N);
    if (!a) return NULL;
    if (N >= 2) {
        a->work = malloc((size_t)N * sizeof(cpx));
        a->roots = (cpx *)malloc((size_t)(N / 2 + N) * sizeof(cpx));
        a->inner = minfft_mkaux_dft_1d(N / 2);
        if (!a->work || !a->roots || !a->inner) goto fail;
        for (n = 0; n < N / 2; ++n) a->roots[n] = unit_root(-n, 2 * N);
        for (n = 0; n < N; ++n) a->roots[N / 2 + n] = unit_root(-(2 * n + 1), 8 * N);
    }
    return a;
fail:
    minfft_free_aux(a);
    return NULL;
}

/* generic multi-D tree: inner = trailing d-1 dims, outer = 1-D of the */
/* leading dim, work = product * elem_size (minfft.c:1024-1054)        */
static minfft_aux *make_nd(int d, const int *Ns, size_t elem, minfft_aux *(*mk1)(int))
{
    minfft_aux *a;
    long p = 1;
    int i;
    if (d < 1 || Ns == NULL) return NULL;
    if (d == 1) return mk1(Ns[0]);
    for (i = 0; i < d; ++i) {
        if (!is_pow2(Ns[i])) return NULL;
        p *= Ns[i];
    }
    a = node_new((int)p);
    if (!a) return NULL;
    a->work = malloc((size_t)p * elem);
    if (!a->work) goto fail;
    a->inner = make_nd(d - 1, Ns + 1, elem, mk1);
    if (!a->inner) goto fail;
    a->outer = mk1(Ns[0]);
    if (!a->outer) goto fail;
    return a;
fail:
    minfft_free_aux(a);
    return NULL;
}

ORACLE_API minfft_aux *minfft_mkaux_dft(int d, int *Ns) { return make_nd(d, Ns, sizeof(cpx), minfft_mkaux_dft_1d); }
ORACLE_API minfft_aux *minfft_mkaux_t2t3(int d, int *Ns) { return make_nd(d, Ns, sizeof(real_t), minfft_mkaux_t2t3_1d); }
ORACLE_API minfft_aux *minfft_mkaux_t4(int d, int *Ns) { return make_nd(d, Ns, sizeof(real_t), minfft_mkaux_t4_1d); }

ORACLE_API minfft_aux *minfft_mkaux_realdft(int d, int *Ns)
{
    /* inner = 1-D real DFT of the last dim, outer = (d-1)-D complex DFT */
    /* of the leading dims, work = (N_last/2+1) * prod(leading) complex  */
    /* (minfft.c:1159-1189)                                              */
    minfft_aux *a;
    long p = 1;
    int i;
    if (d < 1 || Ns == NULL) return NULL;
    if (d == 1) return minfft_mkaux_realdft_1d(Ns[0]);
    for (i = 0; i < d; ++i)
        if (!is_pow2(Ns[i])) return NULL;
    for (i = 0; i < d - 1; ++i) p *= Ns[i];
    a = node_new((int)(p * Ns[d - 1]));
    if (!a) return NULL;
    a->work = malloc((size_t)(Ns[d - 1] / 2 + 1) * (size_t)p * sizeof(cpx));
    if (!a->work) goto fail;
    a->inner = minfft_mkaux_realdft_1d(Ns[d - 1]);
    if (!a->inner) goto fail;
    a->outer = minfft_mkaux_dft(d - 1, Ns);
    if (!a->outer) goto fail;
    return a;
fail:
    minfft_free_aux(a);
    return NULL;
}

#define DIMS2(f)                                                  \
    ORACLE_API minfft_aux *f##_2d(int N1, int N2)                 \
    {                                                             \
        int Ns[2];                                                \
        Ns[0] = N1;                                               \
        Ns[1] = N2;                                               \
        return f(2, Ns);                                          \
    }                                                             \
    ORACLE_API minfft_aux *f##_3d(int N1, int N2, int N3)         \
    {                                                             \
        int Ns[3];                                                \
        Ns[0] = N1;                                               \
        Ns[1] = N2;                                               \
        Ns[2] = N3;                                               \
        return f(3, Ns);                                          \
    }

DIMS2(minfft_mkaux_dft)
DIMS2(minfft_mkaux_realdft)
DIMS2(minfft_mkaux_t2t3)
DIMS2(minfft_mkaux_t4)

ORACLE_API void minfft_free_aux(minfft_aux *a)
{
    if (a == NULL) return;
    free(a->work);
    free(a->roots);
    minfft_free_aux(a->inner);
    minfft_free_aux(a->outer);
    free(a);
}
