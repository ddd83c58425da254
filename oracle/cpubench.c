/*
 * CPU timing driver for the minfft C API -- TEST/BENCH INFRASTRUCTURE ONLY.
 *
 * dlopen()s any library that exports the minfft.h symbols (the compiled
 * reference in oracle/_ref/, or the restatement liboracle*.so) and times a
 * batch of independent transforms with OpenMP: one plan ("aux") per thread,
 * since a minfft aux is not re-entrant (its work buffer is written through a
 * const pointer, reference minfft.c:40,269), and `omp for` over the batch.
 * This is how bench.py measures the reference's CPU path on the host cores.
 */
#include <dlfcn.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define CB_API __attribute__((visibility("default")))

/* transform codes, shared with the Python side */
enum { OP_DFT, OP_INVDFT, OP_REALDFT, OP_INVREALDFT, OP_DCT2, OP_DST2, OP_DCT3, OP_DST3, OP_DCT4, OP_DST4, OP_COUNT };
/* plan families */
enum { FAM_DFT, FAM_REALDFT, FAM_T2T3, FAM_T4 };

typedef void *(*mk_fn)(int, int *);
typedef void (*tx_fn)(void *, void *, const void *);
typedef void (*free_fn)(void *);

static const char *k_op_names[OP_COUNT] = {"minfft_dft",  "minfft_invdft", "minfft_realdft", "minfft_invrealdft",
                                           "minfft_dct2", "minfft_dst2",   "minfft_dct3",    "minfft_dst3",
                                           "minfft_dct4", "minfft_dst4"};
static const char *k_mk_names[4] = {"minfft_mkaux_dft", "minfft_mkaux_realdft", "minfft_mkaux_t2t3", "minfft_mkaux_t4"};

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* element counts (in reals) of an op's input and output for dims */
static void op_sizes(int op, int d, const int *dims, long *in_r, long *out_r)
{
    long p = 1, lead = 1;
    int i;
    for (i = 0; i < d; ++i) p *= dims[i];
    for (i = 0; i < d - 1; ++i) lead *= dims[i];
    switch (op) {
    case OP_DFT:
    case OP_INVDFT: *in_r = *out_r = 2 * p; break;
    case OP_REALDFT: *in_r = p; *out_r = 2 * lead * (dims[d - 1] / 2 + 1); break;
    case OP_INVREALDFT: *in_r = 2 * lead * (dims[d - 1] / 2 + 1); *out_r = p; break;
    default: *in_r = *out_r = p; break;
    }
}

/*
 * Run `warm` untimed and then `reps` timed sweeps over `batch` independent
 * inputs; every batch entry goes through ops[0], ops[1], ... in sequence, the
 * output of one op feeding the next.  Returns the wall time of the timed
 * sweeps in seconds, or a negative code on error.
 * `threads` <= 0 means all OpenMP threads.  `single` = 1 when the library
 * was built with MINFFT_SINGLE.
 */
CB_API double cpubench_run(const char *lib, int single, int family, int nops, const int *ops, int d, const int *dims,
                           long batch, int threads, int warm, int reps, unsigned seed)
{
    void *h = dlopen(lib, RTLD_NOW | RTLD_LOCAL);
    mk_fn mk;
    free_fn fr;
    tx_fn fns[8];
    long sz[9];
    size_t esz = single ? sizeof(float) : sizeof(double);
    char *bufs[9];
    int i, k, err = 0;
    double t0, t1;
    if (!h) return -1;
    if (nops < 1 || nops > 8 || family < 0 || family > 3) return -2;
    mk = (mk_fn)dlsym(h, k_mk_names[family]);
    fr = (free_fn)dlsym(h, "minfft_free_aux");
    if (!mk || !fr) return -3;
    for (k = 0; k < nops; ++k) {
        long a, b;
        if (ops[k] < 0 || ops[k] >= OP_COUNT) return -2;
        fns[k] = (tx_fn)dlsym(h, k_op_names[ops[k]]);
        if (!fns[k]) return -3;
        op_sizes(ops[k], d, dims, &a, &b);
        if (k == 0) sz[0] = a;
        sz[k + 1] = b;
    }
    for (k = 0; k <= nops; ++k) {
        bufs[k] = (char *)malloc((size_t)batch * sz[k] * esz);
        if (!bufs[k]) {
            for (i = 0; i < k; ++i) free(bufs[i]);
            return -4;
        }
    }
    /* seeded uniform [-1, 1) input, filled in parallel (first touch) */
#pragma omp parallel for schedule(static)
    for (i = 0; i < batch; ++i) {
        unsigned s = seed * 2654435761u + (unsigned)i * 40503u + 1u;
        long j;
        for (j = 0; j < sz[0]; ++j) {
            double v;
            s = s * 1664525u + 1013904223u;
            v = (s >> 8) * (1.0 / 8388608.0) - 1.0;
            if (single) ((float *)bufs[0])[(size_t)i * sz[0] + j] = (float)v;
            else ((double *)bufs[0])[(size_t)i * sz[0] + j] = v;
        }
        for (k = 1; k <= nops; ++k) memset(bufs[k] + (size_t)i * sz[k] * esz, 0, (size_t)sz[k] * esz);
    }
    if (threads > 0) omp_set_num_threads(threads);
    if (warm < 0) warm = 0;
    t0 = t1 = 0;
#pragma omp parallel reduction(+ : err)
    {
        void *aux = mk(d, (int *)dims);
        int r;
        long b;
        if (!aux) err += 1;
        for (r = 0; r < warm + reps; ++r) {
#pragma omp barrier
#pragma omp master
            if (r == warm) t0 = now_s();
#pragma omp for schedule(static)
            for (b = 0; b < batch; ++b) {
                int q;
                if (!aux) continue;
                for (q = 0; q < nops; ++q)
                    fns[q](bufs[q] + (size_t)b * sz[q] * esz, bufs[q + 1] + (size_t)b * sz[q + 1] * esz, aux);
            }
        }
#pragma omp barrier
#pragma omp master
        t1 = now_s();
        fr(aux);
    }
    for (k = 0; k <= nops; ++k) free(bufs[k]);
    dlclose(h);
    if (err) return -5;
    return t1 - t0;
}

CB_API int cpubench_max_threads(void) { return omp_get_max_threads(); }
