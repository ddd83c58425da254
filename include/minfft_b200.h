/*
 * minfft_b200.h -- extensions of the B200 transform engine beyond the
 * reference API in minfft.h.  The reference library (aimukhin/minfft) has no
 * counterpart for anything declared here: it is single-threaded, synchronous,
 * returns no error codes and has no batch interface.
 *
 * Conventions: functions returning int return 0 on success or a
 * MINFFT_B200_E* code; the code of the last failure on the calling thread is
 * also kept for minfft_b200_last_error().  Pointers named "stream" are
 * cudaStream_t values.
 */
#ifndef MINFFT_B200_H
#define MINFFT_B200_H

#include "minfft.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- errors */
enum {
    MINFFT_B200_OK = 0,
    MINFFT_B200_EINVAL = 1,      /* bad argument: NULL plan, wrong plan kind, bad size */
    MINFFT_B200_ENOMEM = 2,      /* device or host allocation failed */
    MINFFT_B200_ECUDA = 3,       /* a CUDA runtime call failed */
    MINFFT_B200_EUNSUPPORTED = 4,/* valid request this build cannot run */
    MINFFT_B200_ETIMEOUT = 5     /* a bounded device-side wait gave up */
};

/* Code of the most recent failure on this thread (0 if none) and clear it.
 * minfft.h's transforms return void, so this is how a caller learns that a
 * call was rejected (e.g. invdft given a t4 plan) or that CUDA failed. */
int minfft_b200_last_error(void);
/* Text of the most recent failure on this thread ("" if none). */
const char *minfft_b200_last_error_message(void);

/* --------------------------------------------------------------- streams */
/* Work on device pointers is enqueued on the plan's stream and returns
 * without waiting; calls with host pointers stage through device memory and
 * return when the result is in host memory.  The default stream is the
 * legacy default stream (0). */
int minfft_b200_set_stream(minfft_aux *a, void *stream);
void *minfft_b200_get_stream(const minfft_aux *a);
int minfft_b200_synchronize(const minfft_aux *a);

/* Host-async mode (off by default; no counterpart in the reference, whose
 * calls return when the output is ready).  With enable != 0, a call on plan
 * `a` whose input and output are both page-locked host arrays (cudaHostAlloc
 * or cudaHostRegister) or device arrays is enqueued on the plan's stream --
 * upload, kernels, download -- and returns at once; the caller waits with
 * minfft_b200_synchronize(a) (or the stream) before reading the output or
 * overwriting the input.  Calls on pageable host memory stay synchronous.
 * Consecutive calls on one plan reuse its staging buffers in stream order,
 * so plans on different streams overlap their copies in both directions. */
int minfft_b200_set_host_async(minfft_aux *a, int enable);

/* ------------------------------------------------------------ transforms */
/* Transform codes for the generic entry points below. */
enum {
    MINFFT_B200_DFT = 0,
    MINFFT_B200_INVDFT = 1,
    MINFFT_B200_REALDFT = 2,
    MINFFT_B200_INVREALDFT = 3,
    MINFFT_B200_DCT2 = 4,
    MINFFT_B200_DST2 = 5,
    MINFFT_B200_DCT3 = 6,
    MINFFT_B200_DST3 = 7,
    MINFFT_B200_DCT4 = 8,
    MINFFT_B200_DST4 = 9
};

/* Run transform `op` on `howmany` arrays stored back to back, each shaped
 * as the plan's dimensions (input and output strides are the sizes of one
 * input / output array).  howmany = 1 is exactly the minfft.h call. */
int minfft_b200_execute_batch(int op, void *x, void *y, int howmany, const minfft_aux *a);

/* Bytes of one input / output array of `op` for plan `a` (-1 on error). */
long long minfft_b200_input_bytes(int op, const minfft_aux *a);
long long minfft_b200_output_bytes(int op, const minfft_aux *a);

/* Device bytes held by the plan (tables and scratch). */
long long minfft_b200_plan_bytes(const minfft_aux *a);

/* Number of kernel launches one call of `op` enqueues (after planning). */
int minfft_b200_launch_count(int op, const minfft_aux *a);

/* ------------------------------------------------------ launch timing */
/* With profiling enabled, every kernel launch of the plan's subsequent
 * calls is bracketed by CUDA events on the plan's stream (no host
 * synchronisation).  Reading the statistics synchronises and folds the
 * recorded timings into one entry per kernel label: number of launches,
 * total milliseconds and algorithmic bytes per launch (inputs read once,
 * outputs written once).  Enabling (or disabling) clears the statistics;
 * enable > 1 also pre-creates events for that many launches. */
int minfft_b200_profile(minfft_aux *a, int enable);
int minfft_b200_profile_count(minfft_aux *a);
int minfft_b200_profile_entry(minfft_aux *a, int i, const char **label, long long *launches, double *total_ms,
                              double *bytes_per_launch);

/* ------------------------------------------------- allocation-free DFT */
/* No counterpart in the reference.  Complex DFT (inverse = 0) or unnormalised
 * inverse DFT (inverse != 0) of length n, a power of two in [4, 262144],
 * from device array x to device array y (complex values of this library's
 * precision; x == y allowed), enqueued on `stream` (NULL: the legacy default
 * stream).  It allocates nothing: for callers that cannot call cudaMalloc
 * -- device memory owned by another allocator's pool, fixed memory budgets,
 * loops where an allocation's latency and implied synchronisation are not
 * acceptable -- and so cannot hold a plan.  Its scratch (4 MiB double /
 * 2 MiB single, plus the call's root tables) is a static device array that
 * every GPU loading the library keeps until exit; all calls share it, so
 * calls that overlap on the GPU race and must be ordered by the caller.  The
 * first call on each device looks up the array's address; make it before
 * any stream capture.  Lengths outside the range return MINFFT_B200_EINVAL
 * with nothing launched. */
int minfft_b200_dft_noalloc(const void *x, void *y, int n, int inverse, void *stream);

/* ----------------------------------------------------------- mixed batch */
/* Thousands of independent 1-D transforms of any kind and power-of-two
 * length in one persistent kernel launched from a CUDA graph.  Each job names
 * a transform code (MINFFT_B200_*), its length n (1 .. 65536 for complex
 * transforms, 1 .. 131072 for the real ones) and device input and output
 * arrays (complex data aligned to its size).  Jobs are grouped by kind and
 * length into work items (up to 512*16/L short transforms per item; one item
 * per transform longer than 8192 complex points, which its CTA computes in
 * two passes through a private scratch slice) and handed out through an
 * atomic queue, largest items first.  The plan owns the root tables, the
 * queue and the scratch; execute only launches the captured graph on
 * `stream`.  Outputs of different jobs must not overlap their inputs. */
typedef struct {
    int op;
    int n;
    const void *in;
    void *out;
} minfft_b200_job;
typedef struct minfft_b200_mixed minfft_b200_mixed;
minfft_b200_mixed *minfft_b200_mixed_plan(int count, const minfft_b200_job *jobs);
int minfft_b200_mixed_execute(minfft_b200_mixed *m, void *stream);
/* Time tile shapes (jobs per short work item) and persistent grid sizes
 * (CTAs per SM) on the plan's own data and keep the fastest. */
int minfft_b200_mixed_autotune(minfft_b200_mixed *m, int reps);
int minfft_b200_mixed_items(const minfft_b200_mixed *m);
void minfft_b200_mixed_free(minfft_b200_mixed *m);

/* ----------------------------------------------- tensor-core precision */
/* Arithmetic of plan `a`'s complex 256-point axis passes, including the
 * 256-point passes over HBM of an axis too long for one thread block (in a
 * tensor-core mode such an axis is split into as many 256-point passes as
 * its pass count allows: 2^26 = 256 x 256 x 1024) (single-precision
 * library; no counterpart in the reference, whose arithmetic is its
 * `minfft_real` type, minfft.h:14-31):
 *   MINFFT_B200_PREC_FP32     FP32 on the CUDA cores (default);
 *   MINFFT_B200_PREC_TC_F16   radix-16 stages as DFT-matrix contractions on
 *                             the tensor cores, each row block-scaled by a
 *                             power of two and split into two FP16 terms
 *                             (three products, FP32 accumulation);
 *   MINFFT_B200_PREC_TC_BF16  the same with three BF16 terms (six products).
 * Every other axis keeps its FP32 kernels.  The double-precision library
 * accepts only MINFFT_B200_PREC_FP32 (MINFFT_B200_EUNSUPPORTED otherwise).
 * Applies to launch lists built afterwards (the plan's lists are rebuilt). */
enum {
    MINFFT_B200_PREC_FP32 = 0,
    MINFFT_B200_PREC_TC_F16 = 1,
    MINFFT_B200_PREC_TC_BF16 = 2
};
int minfft_b200_set_precision(minfft_aux *a, int mode);
int minfft_b200_get_precision(const minfft_aux *a);
/* Waits for plan `a`'s stream and reports whether one of its kernels gave up
 * on a bounded device-side wait (a tensor-core pass waiting for its matrix
 * operations) since the previous call: MINFFT_B200_ETIMEOUT, and that
 * launch's output is incomplete.  Clears the record.  minfft_b200_tc_status
 * is the same call. */
int minfft_b200_device_status(const minfft_aux *a);
int minfft_b200_tc_status(const minfft_aux *a);

/* ------------------------------------------------------------- autotuner */
/* Time the candidate launch configurations (kernel form: one tile per CTA
 * or persistent CTAs with double-buffered asynchronous copies; per-thread
 * radix 8 or 16; transforms per CTA) of every kernel launch of transform `op`
 * on `howmany` arrays of plan
 * `a`, using scratch buffers (`reps` timed runs each), and keep the fastest
 * in a process-wide table that every plan consults when it builds its launch
 * lists.  The table can be saved to and loaded from a text file. */
int minfft_b200_autotune(minfft_aux *a, int op, int howmany, int reps);
int minfft_b200_tune_save(const char *path);
int minfft_b200_tune_load(const char *path);
int minfft_b200_tune_clear(void);
int minfft_b200_tune_size(void);
/* Configuration for launches without a table entry: pipe = 1 persistent
 * pipelined kernels, 0 one tile per CTA, -1 the planner's heuristic; cpb > 0
 * transforms per CTA (reduced until it fits), 0 the heuristic; radix 8 or 16
 * complex values per thread.  Applies to plans built afterwards. */
int minfft_b200_tune_set_default(int pipe, int cpb, int radix);

/* ------------------------------------------------------------ self-check */
/* Plan transform `op` for dims Ns[0..d-1] (times `howmany` arrays; `alias`
 * = input and output share memory) on the host only -- no device needed --
 * and verify every planned kernel launch: the elements it reads and writes
 * stay inside their buffers, launch shapes and shared memory are within
 * limits, and passes that cannot run in place do not.  Returns the number of
 * violations (0 = sound, -1 = bad arguments); `report` receives a
 * description of the first violations or, for a sound plan, the launches'
 * labels in launch order, one per line (truncated to report_len);
 * `launches` the launch count. */
int minfft_b200_plan_selfcheck(int op, int d, const int *Ns, int howmany, int alias, char *report, int report_len,
                               int *launches);
/* The same for a plan in arithmetic mode `precision` (MINFFT_B200_PREC_*). */
int minfft_b200_plan_selfcheck_precision(int op, int d, const int *Ns, int howmany, int alias, int precision,
                                         char *report, int report_len, int *launches);

/* ------------------------------------------------------------ test hooks */
/* Failure injection for tests of the allocation paths (no counterpart in the
 * reference, whose makers call malloc directly, minfft.c:1024-1054).  With
 * k > 0, the k-th device allocation the library attempts after this call
 * fails as cudaMalloc does when device memory is short (nothing is
 * allocated for it); k = 0 turns injection off.  Either way the allocation
 * counter restarts at 0.  Process-wide; meant for single-threaded tests. */
int minfft_b200_test_fail_device_alloc(long long k);
/* Device allocations attempted since the last
 * minfft_b200_test_fail_device_alloc call (or since the library loaded). */
long long minfft_b200_test_device_alloc_count(void);
/* Timeout injection for the tensor-core pass (no counterpart in the
 * reference, which has no device waits).  With polls > 0, every tensor-core
 * launch issued afterwards withholds the matrix operations of its first
 * stage, so that stage's completion wait -- limited to `polls` polls -- runs
 * out: the launch leaves its output incomplete and records the timeout for
 * minfft_b200_device_status (MINFFT_B200_ETIMEOUT).  polls = 0 restores
 * normal launches.  No fault is involved; meant for tests. */
int minfft_b200_test_tc_withhold(long long polls);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* MINFFT_B200_H */
