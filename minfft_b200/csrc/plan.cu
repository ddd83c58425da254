// Host side of the engine: plans ("aux") with device-resident root tables
// and scratch, launch-list planning for every transform kind and
// dimensionality, execution on a CUDA stream, and the C ABI of minfft.h and
// minfft_b200.h.
//
// Planning model.  A transform is a sequence of "axis steps".  Each axis
// step is one batched 1-D transform along one axis of a C-order array,
// executed by
//   * one axis-pass kernel when its half- or full-length complex DFT fits in
//     one CTA (L <= 8192 points along contiguous rows, L <= 4096 along
//     strided columns), with the kind's pre/post-processing fused in; or
//   * a Stockham FFT over HBM: P passes of in-CTA sub-DFTs of length <= 4096,
//     pass p reading with stride L/R_p and pre-multiplying by
//     w_{Ns*R_p}^((j mod Ns)*r) (Ns = product of earlier radices), plus a
//     standalone pre/post kernel for real kinds.
// Multi-dimensional transforms apply the 1-D transform along every axis, as
// the reference's transposing recursion does (minfft.c:33-72, 582-597,
// 662-687); here each axis is processed in place in natural C order instead
// of being transposed, which gives the same result.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <new>
#include <set>
#include <string>
#include <tuple>
#include <vector>

#include "axis_pass.cuh"
#include "kernel_registry.h"
#include "pipe_pass.cuh"
#include "stream_pass.cuh"
#include "dct_split.h"
#include "line_kernels.h"
#include "tc_pass.h"
#include "minfft.h"
#include "minfft_b200.h"

#define MB_EXPORT extern "C" __attribute__((visibility("default")))

using mb::AxisParams;
using mb::cpx;
using mb::LineParams;
using mb::real;

// =============================================================== errors
namespace {

thread_local int g_err = 0;
thread_local char g_msg[512] = "";

void set_error(int code, const char* fmt, ...) {
  g_err = code;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
  va_end(ap);
}

}  // namespace

namespace mb {
// Records a failure for minfft_b200_last_error() (used by other translation units).
void set_last_error(int code, const char* msg) { set_error(code, "%s", msg); }
}  // namespace mb

namespace {

bool cuda_ok(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  set_error(e == cudaErrorMemoryAllocation ? MINFFT_B200_ENOMEM : MINFFT_B200_ECUDA, "%s: %s", what,
            cudaGetErrorString(e));
  return false;
}

// Failure injection for the allocation paths (a test hook, off by default):
// when g_fail_at = k > 0, the k-th device allocation counted from the call
// that set it fails as cudaMalloc does when memory is short.
std::atomic<long long> g_alloc_count{0};
std::atomic<long long> g_fail_at{0};
// Test hook: > 0 makes tensor-core launches withhold their first commit and
// give up after this many polls (see mb::TcParams).
std::atomic<long long> g_tc_withhold{0};

}  // namespace

namespace mb {
// Every device allocation of the library goes through here.
cudaError_t dev_malloc(void** p, size_t bytes) {
  const long long n = ++g_alloc_count;
  const long long k = g_fail_at.load();
  if (k > 0 && n == k) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}
}  // namespace mb

namespace {

// ========================================================== unit roots
// (cos, sin)(2*pi*n/N), with the angle folded into [0, pi/4] before calling
// libm -- the folding of reference minfft.c:989-1018, evaluated in double
// for both precisions so the single-precision tables are correctly rounded.
// The tests are written as 2n >= N, 4n >= N, 8n > N: identical to the
// reference's n >= N/2, n >= N/4, n > N/8 for N >= 8, and still terminating
// for N = 1, 2, 4 (where N/4 or N/8 would be 0).
void unit_root(int64_t n, int64_t N, double* c, double* s) {
  if (n < 0) {
    unit_root(-n, N, c, s);
    *s = -*s;
  } else if (2 * n >= N) {
    unit_root(n - N / 2, N, c, s);
    *c = -*c;
    *s = -*s;
  } else if (4 * n >= N) {
    double cc, ss;
    unit_root(n - N / 4, N, &cc, &ss);
    *c = -ss;
    *s = cc;
  } else if (8 * n > N) {
    double cc, ss;
    unit_root(N / 4 - n, N, &cc, &ss);
    *c = ss;
    *s = cc;
  } else {
    const double pi = 3.141592653589793238462643383279502884;
    const double ang = 2 * pi * (double)n / (double)N;
    *c = std::cos(ang);
    *s = std::sin(ang);
  }
}

// w_N^m = exp(-2*pi*i*m/N)
cpx root_w(int64_t m, int64_t N) {
  double c, s;
  unit_root(-m, N, &c, &s);
  cpx r;
  r.x = (real)c;
  r.y = (real)s;
  return r;
}

int ilog2(int64_t v) {
  int r = 0;
  while ((int64_t(1) << r) < v) ++r;
  return r;
}

bool is_pow2(int64_t v) { return v > 0 && (v & (v - 1)) == 0; }

// =================================================== device properties
struct DeviceInfo {
  int max_smem = 227 * 1024;  // B200 opt-in limit; replaced by the queried value
  int sms = 148;
};

DeviceInfo device_info(int dev) {
  static std::mutex mu;
  static std::map<int, DeviceInfo> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(dev);
  if (it != cache.end()) return it->second;
  DeviceInfo d;
  int v = 0;
  if (dev >= 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess && v > 0)
      d.max_smem = v;
    else
      cudaGetLastError();
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0)
      d.sms = v;
    else
      cudaGetLastError();
  }
  cache[dev] = d;
  return d;
}

bool ensure_smem_attr(const void* fn, size_t bytes) {
  static std::mutex mu;
  static std::map<const void*, size_t> done;
  if (bytes <= 48 * 1024) return true;
  std::lock_guard<std::mutex> lk(mu);
  auto it = done.find(fn);
  if (it != done.end() && it->second >= bytes) return true;
  if (!cuda_ok(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
               "cudaFuncSetAttribute"))
    return false;
  done[fn] = bytes;
  return true;
}

// ------------------------------------------------------------- autotuning
// Launch configuration of an axis pass: kernel form and transforms per CTA
// (per tile for the pipelined form).  The autotuner (minfft_b200_autotune)
// times the candidates of each launch of a plan on the device and records
// the fastest here, keyed by everything that shapes the launch; the planner
// consults this table before falling back to its heuristics.
struct TuneKey {
  int combo, L, colmode, hbm, staged;
  int64_t nbatch, d0, in_n, out_k;
  bool operator<(const TuneKey& o) const {
    return std::tie(combo, L, colmode, hbm, staged, nbatch, d0, in_n, out_k) <
           std::tie(o.combo, o.L, o.colmode, o.hbm, o.staged, o.nbatch, o.d0, o.in_n, o.out_k);
  }
};
struct TuneVal {
  int pipe;
  int cpb;
  int radix;  // registers per thread: 8 or 16 complex values
};

std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune;
TuneVal g_default_override{-1, 0, 16};  // minfft_b200_tune_set_default: form (-1 = heuristic), tile, radix
thread_local const std::map<TuneKey, TuneVal>* t_force = nullptr;  // candidates under test

bool tune_lookup(const TuneKey& k, TuneVal* v) {
  if (t_force) {
    auto it = t_force->find(k);
    if (it != t_force->end()) {
      *v = it->second;
      return true;
    }
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(k);
  if (it == g_tune.end()) return false;
  *v = it->second;
  return true;
}

// ============================================================ programs
enum Buf : int { BUF_X = 0, BUF_Y, BUF_T1, BUF_T2, BUF_T3, BUF_T4, BUF_COUNT };

struct Launch {
  const void* fn = nullptr;
  unsigned grid = 0, block = 0;
  size_t smem = 0;
  int in_buf = BUF_X, out_buf = BUF_Y;
  bool is_line = false;
  bool vec_in = false;   // set F_VEC when the resolved real input is complex-aligned
  bool vec_out = false;  // same for the real output
  bool in_c = false;     // the kernel reads its input as complex values
  bool out_c = false;    // the kernel writes its output as complex values
  bool hbm_pass = false; // a pass of the Stockham FFT over HBM (never in place)
  bool pipe = false;     // persistent pipelined kernel (pipe_pass.cuh)
  bool stream = false;   // persistent TMA-fed column pass (stream_pass.cuh)
  bool stream_rows = false;  // persistent bulk-copy-fed row pass (stream_pass.cuh)
  int tcs = 0;           // tensor-core pass in streamed form: 1 column tiles, 2 row tiles
  int dctq = -1;         // split-column DCT pass (dct_split.cu): mb::dctq_kernel's `which`, else -1
  mb::DctqParams dq{};   // its parameters (in, out, mid resolved at launch)
  int mid_buf = -1;      // its intermediate buffer
  int64_t st_d2 = 1;     // streamed pass: outermost batch extent of its tensor copies
  bool tc = false;       // tensor-core split-precision pass (tc_pass.cu)
  mb::TcParams tcp{};    // its B operands and status word
  int ch_static = 16;    // pipelined kernel: copy chunk allowed by the strides
  int combo = -1;        // axis kernels: mb::Combo; line kernels: mb::LineKernel
  TuneKey key{};         // axis kernels: autotuning key
  int L = 0;             // axis kernels: in-CTA DFT length
  int radix = 16;        // axis kernels: per-thread radix
  AxisParams ap;
  LineParams lp;
  std::string label;  // kernel and shape, for launch-level timing
  double bytes = 0;   // algorithmic bytes: each input element read once, each output written once
};

struct Program {
  std::vector<Launch> launches;
  size_t tbytes[BUF_COUNT] = {0, 0, 0, 0, 0, 0};
};

enum Family : int { FAM_DFT = 0, FAM_REALDFT, FAM_T2T3, FAM_T4 };

int op_family(int op) {
  switch (op) {
    case MINFFT_B200_DFT:
    case MINFFT_B200_INVDFT: return FAM_DFT;
    case MINFFT_B200_REALDFT:
    case MINFFT_B200_INVREALDFT: return FAM_REALDFT;
    case MINFFT_B200_DCT2:
    case MINFFT_B200_DST2:
    case MINFFT_B200_DCT3:
    case MINFFT_B200_DST3: return FAM_T2T3;
    case MINFFT_B200_DCT4:
    case MINFFT_B200_DST4: return FAM_T4;
    default: return -1;
  }
}

using namespace mb::tables;

}  // namespace

// ================================================================ plan
struct minfft_aux {
  int family = 0;
  std::vector<int> dims;
  int64_t total = 1;  // product of dims
  int device = 0;
  cudaStream_t stream = nullptr;
  std::map<std::pair<int, int64_t>, void*> tables;
  void* bufs[BUF_COUNT] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  size_t buf_bytes[BUF_COUNT] = {0, 0, 0, 0, 0, 0};
  std::map<std::tuple<int, int, int>, Program> programs;  // (op, howmany, alias)
  int precision = MINFFT_B200_PREC_FP32;  // arithmetic of the 256-point complex passes
  void* tc_mem = nullptr;                 // tensor-core B operands (both formats)
  int* dev_status = nullptr;              // set by kernels whose bounded device-side wait ran out
  bool host_async = false;                // page-locked host arrays: stream-ordered calls (minfft_b200_set_host_async)
  void* stage_in = nullptr;
  size_t stage_in_bytes = 0;
  void* stage_out = nullptr;
  size_t stage_out_bytes = 0;
  size_t table_bytes = 0;
  bool host_only = false;  // plan without a device (minfft_b200_plan_selfcheck)
  // launch-level timing (minfft_b200_profile)
  bool prof = false;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  struct Pending {
    const Launch* ln;
    size_t e0, e1;
  };
  std::vector<Pending> pending;
  struct Stat {
    std::string label;
    long long launches = 0;
    double ms = 0;
    double bytes = 0;
  };
  std::vector<Stat> stats;
};

namespace {

int64_t st_lobits_for(int64_t Lt) { return (ilog2(Lt) + 1) / 2; }

}  // namespace

namespace mb {
// Host values of root table `kind` for length N (see TableKind).
void host_table(int kind, int64_t N, std::vector<cpx>& h) {
  h.clear();
  switch (kind) {
    case TB_TW:  // w_N^m, m < N
      h.resize(N);
      for (int64_t m = 0; m < N; ++m) h[m] = root_w(m, N);
      break;
    case TB_RFT:  // w_N^k, k < N/4 (real-DFT unpacking, minfft.c:1141-1144)
      h.resize(std::max<int64_t>(N / 4, 1));
      for (int64_t k = 0; k < (int64_t)h.size(); ++k) h[k] = root_w(k, N);
      break;
    case TB_T23:  // w_4N^n, n < N/2 (minfft.c:1229-1232)
      h.resize(std::max<int64_t>(N / 2, 1));
      for (int64_t n = 0; n < (int64_t)h.size(); ++n) h[n] = root_w(n, 4 * N);
      break;
    case TB_T4PRE:  // w_2N^n, n < N/2 (minfft.c:1291-1294)
      h.resize(std::max<int64_t>(N / 2, 1));
      for (int64_t n = 0; n < (int64_t)h.size(); ++n) h[n] = root_w(n, 2 * N);
      break;
    case TB_T4POST:  // w_8N^(2q+1), q < N (minfft.c:1295-1298)
      h.resize(N);
      for (int64_t q = 0; q < N; ++q) h[q] = root_w(2 * q + 1, 8 * N);
      break;
    case TB_STHI: {  // w_N^(a << lobits)
      const int lb = (int)st_lobits_for(N);
      h.resize(std::max<int64_t>(N >> lb, 1));
      for (int64_t q = 0; q < (int64_t)h.size(); ++q) h[q] = root_w(q << lb, N);
      break;
    }
    case TB_STLO: {  // w_N^c, c < 2^lobits
      const int lb = (int)st_lobits_for(N);
      h.resize(int64_t(1) << lb);
      for (int64_t q = 0; q < (int64_t)h.size(); ++q) h[q] = root_w(q, N);
      break;
    }
    default: break;
  }
}
}  // namespace mb

namespace {

// Device table of the given kind for length N (built on first use).
const cpx* table(minfft_aux* a, int kind, int64_t N) {
  auto key = std::make_pair(kind, N);
  auto it = a->tables.find(key);
  if (it != a->tables.end()) return static_cast<const cpx*>(it->second);
  if (a->host_only) {
    // placeholder address: self-check plans are never executed
    static cpx dummy[1];
    a->tables[key] = dummy;
    return dummy;
  }
  std::vector<cpx> h;
  mb::host_table(kind, N, h);
  if (h.empty()) return nullptr;
  void* d = nullptr;
  const size_t bytes = h.size() * sizeof(cpx);
  if (!cuda_ok(mb::dev_malloc(&d, bytes), "cudaMalloc(table)")) return nullptr;
  if (!cuda_ok(cudaMemcpy(d, h.data(), bytes, cudaMemcpyHostToDevice), "cudaMemcpy(table)")) {
    cudaFree(d);
    return nullptr;
  }
  a->tables[key] = d;
  a->table_bytes += bytes;
  return static_cast<const cpx*>(d);
}

// ------------------------------------------------------------ planner
constexpr int kRowCapLog2 = 13;  // in-CTA DFT along contiguous rows: <= 8192
constexpr int kColCapLog2 = 12;  // along strided columns: <= 4096
constexpr int kPassCapLog2 = 12;    // sub-DFTs of the HBM passes: <= 4096
constexpr int kPassCapLog2Cc = 10;  // ... of the CUDA-core (FP32/FP64) chains: <= 1024

// Longest sub-DFT of an HBM pass (log2).  A column pass over HBM holds at
// most 512/(L/16) sub-DFTs per CTA, so lengths of 2048 and 4096 leave two to
// four adjacent columns per CTA (runs of 16-64 bytes per row) and ran at half
// the bandwidth of passes of 1024 points or fewer: the CUDA-core chains take
// a third pass instead (2^21 .. 2^24 points; the f32 2^24 DCT-4 + DST-4 step
// went from 0.350 to 0.238 ms).  Tensor-core chains are built around their
// 256-point passes and keep 4096.  MINFFT_B200_PASS_CAP (8 .. 12) overrides
// both, for measurement.
int pass_cap_log2(int precision) {
  static const int forced = [] {
    const char* e = getenv("MINFFT_B200_PASS_CAP");
    const int c = e ? atoi(e) : 0;
    return (c >= 8 && c <= kPassCapLog2) ? c : 0;
  }();
  if (forced) return forced;
  return precision == MINFFT_B200_PREC_FP32 ? kPassCapLog2Cc : kPassCapLog2;
}

struct AxisStep {
  int combo;        // mb::Combo
  int64_t N;        // axis length (real length for real kinds)
  int64_t outer, inner;
  int64_t in_row, out_row;  // elements between consecutive outer rows
  int flags;
  int in_buf, out_buf;
};

struct Planner {
  minfft_aux* a;
  Program* prog;
  int dev_max_smem;
  int sms;
  bool ok = true;

  void need(int buf, size_t bytes) { prog->tbytes[buf] = std::max(prog->tbytes[buf], bytes); }

  const cpx* tab(int kind, int64_t N) {
    const cpx* t = table(a, kind, N);
    if (!t) ok = false;
    return t;
  }

  // transforms per CTA for an in-CTA DFT of length L
  int choose_cpb(int L, bool colmode, int Rq = 16) {
    const int R = std::min(Rq, L);
    const int tpt = L / R;
    int cpb = std::max(1, 256 / tpt);
    if (colmode) {
      const int want = int(128 / sizeof(cpx));  // 128-byte runs of adjacent columns
      if (cpb < want) cpb = std::max(cpb, std::min(want, std::max(1, 512 / tpt)));
    }
    while (cpb > 1 && mb::axis_pass_smem(L, R, cpb, colmode ? 1 : 0) > (size_t)dev_max_smem) cpb /= 2;
    return cpb;
  }

  // kinds whose load or store stage uses the shared-memory tile (the fused
  // type-4 passes hand each real pair's second value to the mirror element)
  static bool staged(int combo) {
    return combo == mb::K_R2C || combo == mb::K_C2R || combo == mb::K_DCT2 || combo == mb::K_DCT3 ||
           combo == mb::K_R2CQ || combo == mb::K_C2RQ || combo == mb::K_T4IN || combo == mb::K_T4OUT;
  }

  // the fused type-4 passes hold mirror pairs of sub-DFTs in one CTA
  static bool mirror_pairs(int combo) { return combo == mb::K_T4IN || combo == mb::K_T4OUT; }

  // the split-column kinds work on exactly four rows per CTA
  static bool four_rows(int combo) { return combo == mb::K_R2CQ || combo == mb::K_C2RQ; }

  // default kernel form when no tuned configuration exists (the pipelined
  // form is chosen per launch by the autotuner; MINFFT_B200_PIPE=1 makes it
  // the default)
  static bool pipe_default() {
    static const bool on = [] {
      const char* e = getenv("MINFFT_B200_PIPE");
      return e && e[0] == '1';
    }();
    return on;
  }

  int max_threads_cpb(int L, int R = 16) const { return std::max(1, 512 / (L / std::min(R, L))); }

  // largest power of two <= 16 dividing every value
  static int pow2_align(std::initializer_list<int64_t> vals) {
    int a = 16;
    for (int64_t v : vals)
      while (a > 4 && (v % a) != 0) a /= 2;
    return a;
  }

  bool pipe_fits(int combo, int L, int cpb, int colmode, int R = 16) const {
    const int Re = std::min(R, L);
    return L >= 2 && mb::pipe_kernel(combo, ilog2(L), R) && cpb >= 1 && cpb <= max_threads_cpb(L, R) &&
           mb::pipe_smem(L, Re, cpb, colmode, mb::pipe_raw_elems(combo, L), mb::pipe_raw_size(combo)) <=
               (size_t)dev_max_smem;
  }

  bool plain_fits(int combo, int L, int cpb, int flags, int colmode, int R = 16) const {
    const int Re = std::min(R, L);
    const bool tile = (L > Re) || staged(combo) || (flags & mb::F_STAGE_ROWS);
    const size_t sm =
        tile ? mb::axis_pass_smem(L, Re, cpb, colmode) : size_t(16 * ((2 * cpb * sizeof(int64_t) + 15) / 16));
    return mb::axis_kernel(combo, ilog2(L), R) && cpb >= 1 && cpb <= max_threads_cpb(L, R) &&
           (!mirror_pairs(combo) || cpb % 2 == 0) && sm <= (size_t)dev_max_smem;
  }

  // The tensor-core pass covers complex 256-point axes: every in-CTA axis
  // of that length and every 256-point pass of a Stockham chain over HBM
  // (pre-twiddled in FP32 after the first); it always stages the tile
  // through shared memory.
  bool use_tc(int combo, int L, const AxisParams& ap) const {
    return a->precision != MINFFT_B200_PREC_FP32 && combo == mb::K_CPLX && L == mb::kTcLength &&
           (ap.flags & ~(mb::F_CONJ_IN | mb::F_CONJ_OUT | mb::F_STAGE_ROWS)) == 0;
  }

  // Type-4 pre/post-rotations fused into the chain passes (MINFFT_B200_T4FUSE=0
  // keeps them as separate element-wise kernels).
  static bool t4_fuse_enabled() {
    static const bool on = [] {
      const char* e = getenv("MINFFT_B200_T4FUSE");
      return !(e && e[0] == '0');
    }();
    return on;
  }

  // Sub-DFT lengths (log2) of the P passes of a Stockham chain over
  // 2^bits points: as even as possible, the longer ones first; in a
  // tensor-core precision mode, as many 256-point passes (first) as the
  // same number of passes allows, the rest split evenly after them.
  std::vector<int> pass_bits(int bits, int P) const {
    const int tb = ilog2(mb::kTcLength);
    int k = 0;
    if (a->precision != MINFFT_B200_PREC_FP32) {
      for (k = std::min(P, bits / tb); k > 0; --k) {
        const int rest = bits - tb * k, left = P - k;
        if (left == 0 ? rest == 0 : (rest >= left && rest <= left * pass_cap_log2(a->precision))) break;
      }
    }
    std::vector<int> pb(k, tb);
    const int left = P - k, rest = bits - tb * k;
    for (int p = 0; p < left; ++p) pb.push_back(rest / left + (p < rest % left ? 1 : 0));
    return pb;
  }

  // Form of the tensor-core pass: the streamed form (tc_stream_kernel) by
  // default, the one-tile form with MINFFT_B200_TC_FORM=tile; stages of the
  // streamed form from MINFFT_B200_TC_STAGES (2 .. 6; default 2, which fits
  // four CTAs per SM in FP16 and three in BF16).
  static bool tc_stream_default() {
    static const bool on = [] {
      const char* e = getenv("MINFFT_B200_TC_FORM");
      return !(e && strcmp(e, "tile") == 0);
    }();
    return on;
  }
  static int tc_stream_stages(int) {
    static const int n = [] {
      const char* e = getenv("MINFFT_B200_TC_STAGES");
      const int v = e ? atoi(e) : 0;
      return v <= 0 ? 0 : (v < 2 ? 2 : (v > 6 ? 6 : v));
    }();
    return n ? n : 2;
  }

  // Normalised layout of the streamed tensor-core pass: b0 indexes the
  // transforms of a tile (adjacent columns at unit stride, or rows of
  // contiguous points), d0 * d1 divides the batch.
  static bool tc_stream_normalise(int64_t nbatch, AxisParams& ap) {
    if (ap.d0 == 1 && ap.d1 > 1) {
      const int64_t d1 = ap.d1;
      ap.d0 = d1;
      ap.is0 = ap.is1;
      ap.os0 = ap.os1;
      ap.d1 = (nbatch + d1 - 1) / d1;
      ap.is1 = ap.is2;
      ap.os1 = ap.os2;
      ap.is2 = 0;
      ap.os2 = 0;
    }
    if (ap.d0 < 2 || nbatch % (ap.d0 * ap.d1) != 0) return false;
    return ap.colmode ? ap.is0 == 1 : ap.in_n == 1;
  }

  bool add_tc_stream_kernel(int fmt, int L, int64_t nbatch, AxisParams ap, int in_buf, int out_buf,
                            const TuneKey& key) {
    if (!tc_stream_default() || L != mb::kTcLength || !tc_stream_normalise(nbatch, ap)) return false;
    if (!ap.colmode && (ap.flags & mb::F_STAGE_ROWS)) return false;
    const bool rows = !ap.colmode;
    const int stages = tc_stream_stages(fmt);
    Launch ln;
    ln.key = key;
    ln.radix = 16;
    ln.tc = true;
    ln.tcs = rows ? 2 : 1;
    ln.fn = mb::tc_stream_kernel_fn(fmt, rows);
    if (!ln.fn) return false;
    ln.smem = mb::tc_stream_smem(fmt, stages);
    if (ln.smem > (size_t)dev_max_smem) return false;
    if (!a->host_only && !ensure_smem_attr(ln.fn, ln.smem)) {
      ok = false;
      return true;
    }
    if (a->host_only) {
      static uint4 dummy[1];
      ln.tcp.bmat = dummy;
      ln.tcp.status = nullptr;
    } else {
      if (!a->tc_mem) {
        set_error(MINFFT_B200_EINVAL, "tensor-core operands missing (set the precision first)");
        ok = false;
        return true;
      }
      ln.tcp.bmat = static_cast<const char*>(a->tc_mem) + (fmt == mb::TC_F16 ? 0 : mb::tc_bmat_bytes(mb::TC_F16));
      ln.tcp.status = a->dev_status;
    }
    const int W = mb::kTcStreamTile;
    ap.nbatch = nbatch;
    ap.cpb = stages;
    ap.stage_bytes = mb::tc_stream_stage_bytes();
    ap.gpb = (ap.d0 + W - 1) / W;
    ln.st_d2 = nbatch / (ap.d0 * ap.d1);
    ap.ntiles = ap.gpb * ap.d1 * ln.st_d2;
    ap.lp = 0;
    ln.block = unsigned(mb::kTcStreamThreads);
    // resident CTAs per SM, counted here from registers, shared memory,
    // threads and the tensor-memory columns a CTA allocates (the
    // occupancy calculator reports one CTA per SM for kernels that allocate
    // tensor memory)
    int occ = 1;
    if (!a->host_only) {
      cudaFuncAttributes fa;
      int dev = 0, smem_sm = 0, regs_sm = 0;
      if (cudaFuncGetAttributes(&fa, ln.fn) == cudaSuccess && cudaGetDevice(&dev) == cudaSuccess &&
          cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) == cudaSuccess &&
          cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) == cudaSuccess) {
        const int warps = int(ln.block + 31) / 32;
        const int regs_cta = warps * ((fa.numRegs * 32 + 255) / 256 * 256);
        const size_t smem_cta = ln.smem + fa.sharedSizeBytes + 1024;  // + the per-CTA reservation
        occ = std::min({regs_sm / std::max(regs_cta, 1), int(size_t(smem_sm) / smem_cta), 2048 / int(ln.block),
                        512 / mb::kTcStreamTmemCols});
        occ = std::max(occ, 1);
      } else {
        cudaGetLastError();
      }
    }
    ln.grid = unsigned(std::min<int64_t>(ap.ntiles, int64_t(sms) * occ));
    ln.in_buf = in_buf;
    ln.out_buf = out_buf;
    ln.in_c = ln.out_c = true;
    ln.combo = mb::K_CPLX;
    ln.L = L;
    ln.ap = ap;
    ln.bytes = 2.0 * L * sizeof(cpx) * double(nbatch);
    char buf[160];
    snprintf(buf, sizeof(buf), "tc_stream<%s,L=%d,%s> batch=%lld", fmt == mb::TC_F16 ? "f16x3" : "bf16x6", L,
             rows ? "row" : "col", (long long)nbatch);
    ln.label = buf;
    prog->launches.push_back(ln);
    return true;
  }

  void add_tc_kernel(int L, int64_t nbatch, AxisParams ap, int in_buf, int out_buf, const TuneKey& key) {
    const int fmt = a->precision == MINFFT_B200_PREC_TC_BF16 ? mb::TC_BF16 : mb::TC_F16;
    if (add_tc_stream_kernel(fmt, L, nbatch, ap, in_buf, out_buf, key)) return;
    const int tb = ap.colmode ? 16 : 8;  // column mode: 16 adjacent columns = 128-byte runs
    Launch ln;
    ln.key = key;
    ln.radix = 16;
    ln.tc = true;
    ln.fn = mb::tc_kernel(fmt, tb);
    if (!ln.fn) {
      set_error(MINFFT_B200_EUNSUPPORTED, "the tensor-core pass needs the single-precision library");
      ok = false;
      return;
    }
    ln.smem = mb::tc_smem(fmt, tb);
    if (ln.smem > (size_t)dev_max_smem) {
      set_error(MINFFT_B200_EUNSUPPORTED, "shared memory %zu exceeds %d", ln.smem, dev_max_smem);
      ok = false;
      return;
    }
    if (!a->host_only && !ensure_smem_attr(ln.fn, ln.smem)) {
      ok = false;
      return;
    }
    if (a->host_only) {
      static uint4 dummy[1];
      ln.tcp.bmat = dummy;
      ln.tcp.status = nullptr;
    } else {
      if (!a->tc_mem) {
        set_error(MINFFT_B200_EINVAL, "tensor-core operands missing (set the precision first)");
        ok = false;
        return;
      }
      ln.tcp.bmat = static_cast<const char*>(a->tc_mem) + (fmt == mb::TC_F16 ? 0 : mb::tc_bmat_bytes(mb::TC_F16));
      ln.tcp.status = a->dev_status;
    }
    ap.cpb = tb;
    ap.nbatch = nbatch;
    ap.lp = 0;
    ap.ntiles = (nbatch + tb - 1) / tb;
    ln.block = unsigned(mb::tc_threads(tb));
    // persistent: one CTA per resident slot.  The occupancy calculator
    // reports one CTA per SM for kernels that allocate tensor memory, so the
    // slots are counted here from registers, shared memory, threads and the
    // 512 TMEM columns of an SM.
    int occ = 1;
    if (!a->host_only) {
      cudaFuncAttributes fa;
      int dev = 0, smem_sm = 0, regs_sm = 0;
      if (cudaFuncGetAttributes(&fa, ln.fn) == cudaSuccess && cudaGetDevice(&dev) == cudaSuccess &&
          cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) == cudaSuccess &&
          cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) == cudaSuccess) {
        const int warps = int(ln.block + 31) / 32;
        const int regs_cta = warps * ((fa.numRegs * 32 + 255) / 256 * 256);
        const size_t smem_cta = ln.smem + fa.sharedSizeBytes + 1024;  // + the per-CTA reservation
        occ = std::min({regs_sm / std::max(regs_cta, 1), int(size_t(smem_sm) / smem_cta), 2048 / int(ln.block),
                        512 / mb::tc_tmem_columns(tb)});
        occ = std::max(occ, 1);
      } else {
        cudaGetLastError();
      }
    }
    ln.grid = unsigned(std::min<int64_t>(ap.ntiles, int64_t(sms) * occ));
    ln.in_buf = in_buf;
    ln.out_buf = out_buf;
    ln.in_c = ln.out_c = true;
    ln.combo = mb::K_CPLX;
    ln.L = L;
    ln.ap = ap;
    ln.bytes = 2.0 * L * sizeof(cpx) * double(nbatch);
    char buf[160];
    snprintf(buf, sizeof(buf), "tc_pass<%s,L=%d,%s> batch=%lld", fmt == mb::TC_F16 ? "f16x3" : "bf16x6", L,
             ap.colmode ? "col" : "row", (long long)nbatch);
    ln.label = buf;
    prog->launches.push_back(ln);
  }

  void add_axis_kernel(int combo, int L, int64_t nbatch, AxisParams ap, int in_buf, int out_buf, bool vec_in,
                       bool vec_out) {
    const int lg = ilog2(L);
    const TuneKey key{combo, L, ap.colmode, ap.st_ns > 1 ? 1 : 0, (ap.flags & mb::F_STAGE_ROWS) ? 1 : 0,
                      nbatch, ap.d0, ap.in_n, ap.out_k};
    if (use_tc(combo, L, ap)) {
      add_tc_kernel(L, nbatch, ap, in_buf, out_buf, key);
      return;
    }
    TuneVal tv;
    int R = 16;  // per-thread radix of the one-tile-per-CTA form
    if (tune_lookup(key, &tv)) {
      if (tv.pipe == 2 && stream_fits(combo, L, nbatch, ap, tv.radix, tv.cpb)) {
        add_stream_kernel(L, nbatch, ap, in_buf, out_buf, tv.cpb, key, tv.radix);
        return;
      }
      if ((tv.pipe == 3 || tv.pipe == 4) && stream_rows_fits(combo, L, ap, tv.cpb, tv.pipe - 1)) {
        add_stream_rows_kernel(combo, L, nbatch, ap, in_buf, out_buf, tv.cpb, tv.pipe - 1, key, vec_in, vec_out);
        return;
      }
      if (tv.pipe == 1 && pipe_fits(combo, L, tv.cpb, ap.colmode, tv.radix)) {
        add_pipe_kernel(combo, L, nbatch, ap, in_buf, out_buf, tv.cpb, key, tv.radix);
        return;
      }
      if (!tv.pipe && plain_fits(combo, L, tv.cpb, ap.flags, ap.colmode, tv.radix)) {
        ap.cpb = tv.cpb;
        R = tv.radix;
      }
    } else {
      TuneVal ov;
      {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        ov = g_default_override;
      }
      const bool want_pipe = ov.pipe == 1 || (ov.pipe < 0 && pipe_default());
      const int st_stages = ov.cpb > 0 ? ov.cpb : 3;
      if (ov.pipe == 2 && stream_fits(combo, L, nbatch, ap, ov.radix, st_stages)) {
        add_stream_kernel(L, nbatch, ap, in_buf, out_buf, st_stages, key, ov.radix);
        return;
      }
      if ((ov.pipe == 3 || ov.pipe == 4) && L >= 64) {
        int c = four_rows(combo) ? 4 : (ov.cpb > 0 ? ov.cpb : std::max(1, 256 / (L / 16)));
        while (c > 1 && !stream_rows_fits(combo, L, ap, c, ov.pipe - 1) && !four_rows(combo)) c /= 2;
        if (stream_rows_fits(combo, L, ap, c, ov.pipe - 1)) {
          add_stream_rows_kernel(combo, L, nbatch, ap, in_buf, out_buf, c, ov.pipe - 1, key, vec_in, vec_out);
          return;
        }
      }
      if (want_pipe) {
        int pc = ov.cpb > 0 ? ov.cpb : choose_pipe_cpb(combo, L, ap.colmode != 0);
        const int rr = pipe_fits(combo, L, 1, ap.colmode, ov.radix) ? ov.radix : 16;
        while (pc > 1 && !pipe_fits(combo, L, pc, ap.colmode, rr)) pc /= 2;
        if (pipe_fits(combo, L, pc, ap.colmode, rr)) {
          add_pipe_kernel(combo, L, nbatch, ap, in_buf, out_buf, pc, key, rr);
          return;
        }
      } else if (ov.pipe == 0 && (ov.cpb > 0 || ov.radix != 16)) {
        const int rr = plain_fits(combo, L, 1, ap.flags, ap.colmode, ov.radix) ? ov.radix : 16;
        int c = ov.cpb > 0 ? ov.cpb : choose_cpb(L, ap.colmode != 0, rr);
        while (c > 1 && !plain_fits(combo, L, c, ap.flags, ap.colmode, rr)) c /= 2;
        ap.cpb = c;
        R = rr;
      }
    }
    if (four_rows(combo)) {
      ap.cpb = 4;
      if (!mb::axis_kernel(combo, lg, R)) R = (R == 16) ? 8 : 16;
    }
    if (mirror_pairs(combo)) {
      // an even tile that divides the M sub-DFTs of a line (mirror i and M-1-i)
      const int64_t M = ap.d0 * ap.d1;
      if (ap.cpb < 2) ap.cpb = 2;
      while (ap.cpb > 2 && M % ap.cpb) ap.cpb /= 2;
      if (M % ap.cpb || nbatch % M || ap.cpb * (L / std::min(R, L)) > 512) {
        set_error(MINFFT_B200_EUNSUPPORTED, "no mirror-pair tile for the type-4 pass (L=%d, %lld sub-DFTs per line)",
                  L, (long long)M);
        ok = false;
        return;
      }
    }
    Launch ln;
    ln.key = key;
    ln.radix = R;
    ln.fn = mb::axis_kernel(combo, lg, R);
    if (!ln.fn) {
      set_error(MINFFT_B200_EUNSUPPORTED, "no kernel for combo %d, L=%d", combo, L);
      ok = false;
      return;
    }
    const int Re = std::min(R, L);
    const int tpt = L / Re;
    const bool tile = (L > Re) || staged(combo) || (ap.flags & mb::F_STAGE_ROWS);
    ap.lp = mb::tile_pitch(L, Re, ap.cpb, ap.colmode);
    ln.smem = tile ? mb::axis_pass_smem(L, Re, ap.cpb, ap.colmode)
                   : size_t(16 * ((2 * ap.cpb * sizeof(int64_t) + 15) / 16));
    if (ln.smem > (size_t)dev_max_smem) {
      set_error(MINFFT_B200_EUNSUPPORTED, "shared memory %zu exceeds %d", ln.smem, dev_max_smem);
      ok = false;
      return;
    }
    if (!a->host_only && !ensure_smem_attr(ln.fn, ln.smem)) {
      ok = false;
      return;
    }
    ap.nbatch = nbatch;
    ln.block = unsigned(ap.cpb * tpt);
    ln.grid = unsigned((nbatch + ap.cpb - 1) / ap.cpb);
    ln.in_buf = in_buf;
    ln.out_buf = out_buf;
    ln.vec_in = vec_in;
    ln.vec_out = vec_out;
    ln.in_c = (combo == mb::K_CPLX || combo == mb::K_C2R || combo == mb::K_C2RQ || combo == mb::K_T4OUT);
    ln.out_c = (combo == mb::K_CPLX || combo == mb::K_R2C || combo == mb::K_R2CQ || combo == mb::K_T4IN);
    ln.combo = combo;
    ln.L = L;
    ln.ap = ap;
    {
      static const char* names[] = {"cplx", "r2c", "c2r", "dct2", "dct3", "t4", "r2c+col4", "col4+c2r",
                                    "t4pre+cplx", "cplx+t4post"};
      const double R = sizeof(real), C = sizeof(cpx);
      double per = 0;
      switch (combo) {
        case mb::K_CPLX: per = 2.0 * L * C; break;
        case mb::K_T4IN:
        case mb::K_T4OUT: per = 2.0 * L * R + L * C; break;
        case mb::K_R2C:
        case mb::K_R2CQ: per = 2.0 * L * R + (L + 1) * C; break;
        case mb::K_C2R:
        case mb::K_C2RQ: per = (L + 1) * C + 2.0 * L * R; break;
        default: per = 4.0 * L * R; break;
      }
      ln.bytes = per * double(nbatch);
      char buf[160];
      snprintf(buf, sizeof(buf), "axis_pass<%s,L=%d,%s%s> batch=%lld", names[combo], L, ap.colmode ? "col" : "row",
               ap.st_ns > 1 ? ",hbm" : "", (long long)nbatch);
      ln.label = buf;
    }
    prog->launches.push_back(ln);
  }

  // transforms per tile of the pipelined kernel: two stages must fit
  int choose_pipe_cpb(int combo, int L, bool colmode, int Rq = 16) {
    const int R = std::min(Rq, L);
    const int tpt = L / R;
    int cpb = std::max(1, 256 / tpt);
    if (colmode) {
      const int want = int(64 / mb::pipe_raw_size(combo));  // 64-byte runs of adjacent columns
      if (cpb < want) cpb = std::max(cpb, std::min(want, std::max(1, 512 / tpt)));
    }
    const int er = mb::pipe_raw_elems(combo, L);
    const size_t esz = mb::pipe_raw_size(combo);
    auto smem = [&](int c) { return mb::pipe_smem(L, R, c, colmode ? 1 : 0, er, esz); };
    while (cpb > 1 && smem(cpb) > (size_t)dev_max_smem) cpb /= 2;
    return cpb;
  }

  // The streamed column pass covers complex column-mode launches whose
  // adjacent transforms are adjacent in the input (the batch index of unit
  // input stride is the innermost one, possibly after dropping a unit d0),
  // lengths 16 .. 512 and `stages` tiles of shared memory in flight.  It
  // rewrites `ap` into that normalised form.
  bool stream_normalise(int combo, int L, int64_t nbatch, AxisParams& ap) const {
    if (combo != mb::K_CPLX || !ap.colmode || L < 16 || L > 512) return false;
    if (ap.d0 == 1 && ap.d1 > 1) {
      // b = b1 + d1*b2: the transforms of unit stride are the b1 ones
      const int64_t d1 = ap.d1;
      ap.d0 = d1;
      ap.is0 = ap.is1;
      ap.os0 = ap.os1;
      ap.d1 = (nbatch + d1 - 1) / d1;
      ap.is1 = ap.is2;
      ap.os1 = ap.os2;
      ap.is2 = 0;
      ap.os2 = 0;
    }
    if (ap.is0 != 1 || ap.d0 < 2 || nbatch % (ap.d0 * ap.d1) != 0) return false;
    return true;
  }

  bool stream_fits(int combo, int L, int64_t nbatch, const AxisParams& ap0, int R, int stages) const {
    AxisParams ap = ap0;
    if (!stream_normalise(combo, L, nbatch, ap)) return false;
    if (stages < 2 || stages > 8 || !mb::stream_kernel(ilog2(L), R)) return false;
    return mb::stream_smem(L, stages) <= (size_t)dev_max_smem;
  }

  void add_stream_kernel(int L, int64_t nbatch, AxisParams ap, int in_buf, int out_buf, int stages,
                         const TuneKey& key, int R) {
    stream_normalise(mb::K_CPLX, L, nbatch, ap);
    const int W = mb::stream_cols();
    Launch ln;
    ln.key = key;
    ln.radix = R;
    ln.fn = mb::stream_kernel(ilog2(L), R);
    ln.stream = true;
    ap.nbatch = nbatch;
    ap.cpb = stages;
    ap.stage_bytes = mb::stream_stage_bytes(L);
    ap.gpb = (ap.d0 + W - 1) / W;
    ln.st_d2 = nbatch / (ap.d0 * ap.d1);
    ap.ntiles = ap.gpb * ap.d1 * ln.st_d2;
    ap.lp = 0;
    ln.smem = mb::stream_smem(L, stages);
    if (!ln.fn || ln.smem > (size_t)dev_max_smem) {
      set_error(MINFFT_B200_EUNSUPPORTED, "no streamed pass for L=%d with %d stages", L, stages);
      ok = false;
      return;
    }
    if (!a->host_only && !ensure_smem_attr(ln.fn, ln.smem)) {
      ok = false;
      return;
    }
    ln.block = unsigned(W * (L / R));
    int occ = 1;
    if (!a->host_only) {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ln.fn, (int)ln.block, ln.smem) != cudaSuccess ||
          occ < 1) {
        cudaGetLastError();
        occ = 1;
      }
    }
    ln.grid = unsigned(std::min<int64_t>(ap.ntiles, int64_t(sms) * occ));
    ln.in_buf = in_buf;
    ln.out_buf = out_buf;
    ln.in_c = ln.out_c = true;
    ln.combo = mb::K_CPLX;
    ln.L = L;
    ln.ap = ap;
    ln.bytes = 2.0 * L * sizeof(cpx) * double(nbatch);
    char buf[160];
    snprintf(buf, sizeof(buf), "stream_pass<cplx,L=%d,col%s> batch=%lld", L, ap.st_ns > 1 ? ",hbm" : "",
             (long long)nbatch);
    ln.label = buf;
    prog->launches.push_back(ln);
  }

  // The streamed row pass: row-mode launches whose rows are contiguous,
  // lengths 64 .. 4096 (2048 for the split-column kinds), cpb rows per tile
  // and `stages` tiles in flight (tuning forms 3 and 4: two and three).
  static int raw_row_elems(int combo, int L) {
    switch (combo) {
      case mb::K_CPLX: return L;
      case mb::K_C2R:
      case mb::K_C2RQ: return L + 1;
      default: return 2 * L;
    }
  }
  static int raw_elem_size(int combo) {
    return (combo == mb::K_CPLX || combo == mb::K_C2R || combo == mb::K_C2RQ) ? int(sizeof(cpx)) : int(sizeof(real));
  }
  bool stream_rows_fits(int combo, int L, const AxisParams& ap, int cpb, int stages) const {
    if (L < 64 || ap.colmode || ap.in_n != 1 || cpb < 1 || stages < 2 || stages > 8) return false;
    if (four_rows(combo) && cpb != 4) return false;
    if (!mb::stream_rows_kernel_fn(combo, ilog2(L)) || cpb * (L / 16) > 512) return false;
    const int rb = raw_row_elems(combo, L) * raw_elem_size(combo);
    const int pitch = (rb + 15) / 16 * 16;
    return mb::stream_rows_smem(L, 16, cpb, stages, pitch) <= (size_t)dev_max_smem;
  }

  void add_stream_rows_kernel(int combo, int L, int64_t nbatch, AxisParams ap, int in_buf, int out_buf, int cpb,
                              int stages, const TuneKey& key, bool vec_in, bool vec_out) {
    Launch ln;
    ln.key = key;
    ln.radix = 16;
    ln.fn = mb::stream_rows_kernel_fn(combo, ilog2(L));
    ln.stream_rows = true;
    const int esz = raw_elem_size(combo);
    ap.cpb = cpb;
    ap.nbatch = nbatch;
    ap.nstages = stages;
    ap.row_bytes = raw_row_elems(combo, L) * esz;
    ap.row_pitch = (ap.row_bytes + 15) / 16 * 16;
    ap.ntiles = (nbatch + cpb - 1) / cpb;
    ap.lp = mb::tile_pitch(L, 16, cpb, 0);
    ln.ch_static = pow2_align({int64_t(ap.row_bytes), ap.is0 * esz, ap.is1 * esz, ap.is2 * esz});
    ln.smem = mb::stream_rows_smem(L, 16, cpb, stages, ap.row_pitch);
    if (!ln.fn || ln.smem > (size_t)dev_max_smem) {
      set_error(MINFFT_B200_EUNSUPPORTED, "no streamed row pass for combo %d, L=%d", combo, L);
      ok = false;
      return;
    }
    if (!a->host_only && !ensure_smem_attr(ln.fn, ln.smem)) {
      ok = false;
      return;
    }
    ln.block = unsigned(cpb * (L / 16));
    int occ = 1;
    if (!a->host_only) {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ln.fn, (int)ln.block, ln.smem) != cudaSuccess ||
          occ < 1) {
        cudaGetLastError();
        occ = 1;
      }
    }
    ln.grid = unsigned(std::min<int64_t>(ap.ntiles, int64_t(sms) * occ));
    ln.in_buf = in_buf;
    ln.out_buf = out_buf;
    ln.vec_in = vec_in;
    ln.vec_out = vec_out;
    ln.in_c = (combo == mb::K_CPLX || combo == mb::K_C2R || combo == mb::K_C2RQ);
    ln.out_c = (combo == mb::K_CPLX || combo == mb::K_R2C || combo == mb::K_R2CQ);
    ln.combo = combo;
    ln.L = L;
    ln.ap = ap;
    {
      static const char* names[] = {"cplx", "r2c", "c2r", "dct2", "dct3", "t4", "r2c+col4", "col4+c2r",
                                    "t4pre+cplx", "cplx+t4post"};
      const double Rb = sizeof(real), C = sizeof(cpx);
      double per = 0;
      switch (combo) {
        case mb::K_CPLX: per = 2.0 * L * C; break;
        case mb::K_R2C:
        case mb::K_R2CQ: per = 2.0 * L * Rb + (L + 1) * C; break;
        case mb::K_C2R:
        case mb::K_C2RQ: per = (L + 1) * C + 2.0 * L * Rb; break;
        default: per = 4.0 * L * Rb; break;
      }
      ln.bytes = per * double(nbatch);
      char buf[160];
      snprintf(buf, sizeof(buf), "stream_rows<%s,L=%d> batch=%lld", names[combo], L, (long long)nbatch);
      ln.label = buf;
    }
    prog->launches.push_back(ln);
  }

  void add_pipe_kernel(int combo, int L, int64_t nbatch, AxisParams ap, int in_buf, int out_buf, int cpb,
                       const TuneKey& key, int Rq = 16) {
    const int lg = ilog2(L);
    Launch ln;
    ln.key = key;
    ln.radix = Rq;
    ln.fn = mb::pipe_kernel(combo, lg, Rq);
    ln.pipe = true;
    const int R = std::min(Rq, L);
    const int tpt = L / R;
    const int esz = mb::pipe_raw_size(combo), er = mb::pipe_raw_elems(combo, L);
    ap.cpb = cpb;
    ap.nbatch = nbatch;
    if (ap.colmode) {
      ap.gpb = (ap.d0 + ap.cpb - 1) / ap.cpb;
      ap.ntiles = (nbatch / ap.d0) * ap.gpb;
      ln.ch_static = pow2_align({int64_t(ap.cpb) * esz, ap.in_n * esz, ap.is1 * esz, ap.is2 * esz});
    } else {
      ap.gpb = 0;
      ap.ntiles = (nbatch + ap.cpb - 1) / ap.cpb;
      const int64_t run = int64_t(er % 2 == 1 ? er - 1 : er) * esz;
      ln.ch_static = pow2_align({run, int64_t(er) * esz, ap.is1 * esz, ap.is2 * esz});
    }
    ap.lp = mb::tile_pitch(L, R, ap.cpb, ap.colmode);
    ap.stage_bytes = (int)mb::pipe_stage_bytes(L, R, ap.cpb, ap.colmode, er, esz);
    ln.smem = mb::pipe_smem(L, R, ap.cpb, ap.colmode, er, esz);
    if (ln.smem > (size_t)dev_max_smem) {
      set_error(MINFFT_B200_EUNSUPPORTED, "shared memory %zu exceeds %d", ln.smem, dev_max_smem);
      ok = false;
      return;
    }
    if (!a->host_only && !ensure_smem_attr(ln.fn, ln.smem)) {
      ok = false;
      return;
    }
    ln.block = unsigned(ap.cpb * tpt);
    int occ = 1;
    if (!a->host_only) {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ln.fn, (int)ln.block, ln.smem) != cudaSuccess ||
          occ < 1) {
        cudaGetLastError();
        occ = 1;
      }
    }
    ln.grid = unsigned(std::min<int64_t>(ap.ntiles, int64_t(sms) * occ));
    ln.in_buf = in_buf;
    ln.out_buf = out_buf;
    ln.vec_out = (combo == mb::K_C2R);
    ln.in_c = (combo == mb::K_CPLX || combo == mb::K_C2R || combo == mb::K_C2RQ || combo == mb::K_T4OUT);
    ln.out_c = (combo == mb::K_CPLX || combo == mb::K_R2C || combo == mb::K_R2CQ || combo == mb::K_T4IN);
    ln.combo = combo;
    ln.L = L;
    ln.ap = ap;
    {
      static const char* names[] = {"cplx", "r2c", "c2r", "dct2", "dct3", "t4", "r2c+col4", "col4+c2r",
                                    "t4pre+cplx", "cplx+t4post"};
      const double Rb = sizeof(real), C = sizeof(cpx);
      double per = 0;
      switch (combo) {
        case mb::K_CPLX: per = 2.0 * L * C; break;
        case mb::K_R2C: per = 2.0 * L * Rb + (L + 1) * C; break;
        case mb::K_C2R: per = (L + 1) * C + 2.0 * L * Rb; break;
        default: per = 4.0 * L * Rb; break;
      }
      ln.bytes = per * double(nbatch);
      char buf[160];
      snprintf(buf, sizeof(buf), "axis_pipe<%s,L=%d,%s%s> batch=%lld", names[combo], L, ap.colmode ? "col" : "row",
               ap.st_ns > 1 ? ",hbm" : "", (long long)nbatch);
      ln.label = buf;
    }
    prog->launches.push_back(ln);
  }

  void add_line_kernel(int which, LineParams lp, int64_t items, int in_buf, int out_buf) {
    Launch ln;
    ln.fn = mb::line_kernel(which);
    ln.is_line = true;
    ln.block = 256;
    const int64_t want = (items + 255) / 256;
    ln.grid = unsigned(std::max<int64_t>(1, std::min<int64_t>(want, int64_t(sms) * 32)));
    ln.in_buf = in_buf;
    ln.out_buf = out_buf;
    ln.combo = which;
    switch (which) {
      case mb::LK_C2R_PACK:
      case mb::LK_R2C_UNPACK: ln.in_c = ln.out_c = true; break;
      case mb::LK_DCT2_PRE:
      case mb::LK_T4_PRE:
      case mb::LK_DCT3_PACK: ln.out_c = true; break;
      case mb::LK_DCT2_POST:
      case mb::LK_DCT3_POST:
      case mb::LK_T4_POST: ln.in_c = true; break;
      default:
        ln.in_c = (lp.mode == mb::UNIT_CPLX_TO_REAL || lp.mode == mb::UNIT_COPY_CPLX);
        ln.out_c = (lp.mode == mb::UNIT_REAL_TO_CPLX || lp.mode == mb::UNIT_COPY_CPLX);
        break;
    }
    ln.lp = lp;
    {
      static const char* names[] = {"dct2_pre", "t4_pre", "c2r_pack", "dct3_pack", "r2c_unpack",
                                    "dct2_post", "dct3_post", "t4_post", "unit"};
      const double R = sizeof(real), C = sizeof(cpx);
      const double lines = double(lp.outer) * double(lp.inner), L = double(lp.L);
      switch (which) {
        case mb::LK_DCT2_PRE:
        case mb::LK_T4_PRE: ln.bytes = lines * (2 * L * R + L * C); break;
        case mb::LK_DCT3_PACK: ln.bytes = lines * (2 * L * R + L * C); break;
        case mb::LK_C2R_PACK: ln.bytes = lines * ((L + 1) * C + L * C); break;
        case mb::LK_R2C_UNPACK: ln.bytes = lines * (L * C + (L + 1) * C); break;
        case mb::LK_DCT2_POST:
        case mb::LK_DCT3_POST:
        case mb::LK_T4_POST: ln.bytes = lines * (L * C + 2 * L * R); break;
        default: {
          const double in_e = ln.in_c ? C : R, out_e = ln.out_c ? C : R;
          ln.bytes = L * (in_e + out_e);
        }
      }
      char buf[160];
      snprintf(buf, sizeof(buf), "line<%s> items=%lld", names[which], (long long)items);
      ln.label = buf;
    }
    prog->launches.push_back(ln);
  }

  void add_unit(int mode, int64_t count, real scale, int in_buf, int out_buf) {
    LineParams lp{};
    lp.L = count;
    lp.mode = mode;
    lp.scale = scale;
    add_line_kernel(mb::LK_UNIT, lp, count, in_buf, out_buf);
  }

  AxisParams base_params() {
    AxisParams ap;
    memset(&ap, 0, sizeof(ap));
    ap.d0 = ap.d1 = 1;
    ap.st_ns = 1;
    ap.st_div = 1;
    return ap;
  }

  void set_kind_tables(AxisParams& ap, int combo, int64_t N) {
    switch (combo) {
      case mb::K_R2C: ap.t1 = tab(TB_RFT, N); break;
      case mb::K_C2R: ap.t2 = tab(TB_RFT, N); break;
      case mb::K_DCT2:
      case mb::K_DCT3:
        ap.t1 = tab(TB_T23, N);
        ap.t2 = tab(TB_RFT, N);
        break;
      case mb::K_T4:
        ap.t1 = tab(TB_T4PRE, N);
        ap.t2 = tab(TB_T4POST, N);
        break;
      default: break;
    }
  }

  // roots w_M^(mul*i + add) of a long line's pre/post step as the product of
  // a coarse and a fine table (slot 1 replaces lp.t1, slot 2 lp.t2): two
  // tables of about sqrt(M) entries instead of one of the line's length
  void set_root_pair(LineParams& lp, int slot, int64_t M, int mul, int add) {
    const cpx* hi = tab(TB_STHI, M);
    const cpx* lo = tab(TB_STLO, M);
    const int bits = (int)st_lobits_for(M);
    if (slot == 1) {
      lp.hi1 = hi;
      lp.lo1 = lo;
      lp.bits1 = bits;
      lp.mul1 = mul;
      lp.add1 = add;
    } else {
      lp.hi2 = hi;
      lp.lo2 = lo;
      lp.bits2 = bits;
      lp.mul2 = mul;
      lp.add2 = add;
    }
  }

  int pick_temp(std::initializer_list<int> exclude) {
    for (int b : {BUF_T2, BUF_T3, BUF_T4}) {
      bool bad = false;
      for (int e : exclude) bad |= (e == b);
      if (!bad) return b;
    }
    return BUF_T4;
  }

  // 2-D real DFT of H arrays of Nr rows of N reals with a split column DFT:
  // Nr = 4Q, the column DFT of length Nr done as a radix-4 stage fused into
  // the row pass (four rows j + Q*m per CTA) and length-Q DFTs of the four
  // blocks, so the column passes work on short columns with wide tiles.  Taken
  // when the rows fit four to a CTA and Nr is at least MINFFT_B200_SPLIT2D
  // (default 1024; 0 turns it off).
  bool split_2d(int64_t Nr, int64_t N) const {
    static const int64_t min_rows = [] {
      const char* e = getenv("MINFFT_B200_SPLIT2D");
      if (!e) return int64_t(1024);
      const long long v = atoll(e);
      return v <= 0 ? std::numeric_limits<int64_t>::max() : int64_t(v);
    }();
    const int64_t L = N / 2;
    if (Nr < min_rows || Nr % 4 != 0 || L < 16 || L > 2048) return false;
    if (ilog2(Nr / 4) > kColCapLog2) return false;
    return mb::axis_pass_smem(int(L), int(std::min<int64_t>(16, L)), 4, 0) <= (size_t)dev_max_smem;
  }

  // Forward: rows X -> block layout in `mid` (row j of block q at (q*Q + j)*K),
  // then length-Q column DFTs mid -> Y (output p of block q at row q + 4p).
  // Split column DFT of the 2-D DCT-2/DST-2 and DCT-3/DST-3 (Nr rows of N
  // reals): Nr = 8Q with Q = 64 .. 512, N/2 = 64 .. 1024, from the same row
  // count as the split 2-D real DFT (MINFFT_B200_SPLIT2D), when enabled.
  int dctq_cols(int64_t Q) const {
    int W = int(128 / sizeof(cpx));
    while (W > 1 && 2 * W * (Q / 16) > 512) W /= 2;
    return W;
  }
  bool split_dct(int64_t Nr, int64_t N) const {
    // opt-in (MINFFT_B200_SPLITDCT=1): measured slower than the one-tile row
    // and column passes on 2048 x 2048 in both precisions
    const char* env = getenv("MINFFT_B200_SPLITDCT");  // read at each planning
    if (!(env && env[0] == '1') || !split_2d(Nr, N) || Nr % 8 != 0) return false;
    const int64_t Q = Nr / 8, L = N / 2;
    if (!mb::dctq_kernel(0, ilog2(L)) || !mb::dctq_kernel(1, ilog2(Q)) || !is_pow2(Q)) return false;
    const int W = dctq_cols(Q);
    if (N % W != 0) return false;
    return mb::dctq_row_smem(int(L)) <= (size_t)dev_max_smem && mb::dctq_col_smem(int(Q), W) <= (size_t)dev_max_smem;
  }

  void add_dctq(int which, int64_t H, int64_t Nr, int64_t N, int flags, int in_buf, int out_buf, int mid) {
    const int64_t Q = Nr / 8, L = N / 2, Lc = Nr / 2;
    const bool row = (which == 0 || which == 3);
    Launch ln;
    ln.dctq = which;
    ln.fn = mb::dctq_kernel(which, ilog2(row ? L : Q));
    ln.radix = 16;
    mb::DctqParams& d = ln.dq;
    d.H = H;
    d.Nr = Nr;
    d.N = N;
    d.Q = Q;
    d.flags = flags;
    d.W = dctq_cols(Q);
    d.lp = row ? mb::tile_pitch(int(L), 16, 8, 0) : mb::tile_pitch(int(Q), 16, 2 * d.W, 1);
    d.tw_row = tab(TB_TW, L);
    d.rft_row = tab(TB_RFT, N);
    d.t23_row = tab(TB_T23, N);
    d.tw_c = tab(TB_TW, Lc);
    d.tw_q = tab(TB_TW, Q);
    d.rft_c = tab(TB_RFT, Nr);
    d.t23_c = tab(TB_T23, Nr);
    ln.smem = row ? mb::dctq_row_smem(int(L)) : mb::dctq_col_smem(int(Q), d.W);
    if (!ln.fn || ln.smem > (size_t)dev_max_smem) {
      set_error(MINFFT_B200_EUNSUPPORTED, "no split DCT pass for %lld x %lld", (long long)Nr, (long long)N);
      ok = false;
      return;
    }
    if (!a->host_only && !ensure_smem_attr(ln.fn, ln.smem)) {
      ok = false;
      return;
    }
    ln.block = unsigned(row ? 8 * (L / 16) : 2 * d.W * (Q / 16));
    ln.grid = unsigned(row ? H * Q : H * 2 * (N / d.W));
    ln.in_buf = in_buf;
    ln.out_buf = out_buf;
    ln.mid_buf = mid;
    ln.in_c = (which == 1 || which == 3);
    ln.out_c = false;
    ln.L = int(row ? L : Q);
    const double R = sizeof(real), C = sizeof(cpx);
    ln.bytes = double(H) * Nr * N * R + double(H) * Lc * N * C;  // the real array and the blocks
    static const char* names[] = {"dct2 rows+col4", "col4 dct2 cols", "dct3 cols col4", "col4+dct3 rows"};
    char buf[160];
    snprintf(buf, sizeof(buf), "dct_split<%s,%s=%lld> %lldx%lld", names[which], row ? "L" : "Q",
             (long long)(row ? L : Q), (long long)Nr, (long long)N);
    ln.label = buf;
    prog->launches.push_back(ln);
  }

  // Row pitch of the intermediate of a split 2-D real DFT: K complex values
  // rounded up to whole 16-byte units, so that its columns can be fetched
  // with tensor copies (the extra column is never read).
  static int64_t split_pitch(int64_t K) {
    const int64_t per16 = int64_t(16 / sizeof(cpx));
    return (K + per16 - 1) / per16 * per16;
  }

  void plan_realdft_split(int64_t H, int64_t Nr, int64_t N, int in_buf, int mid, int out_buf) {
    const int64_t K = N / 2 + 1, Q = Nr / 4, L = N / 2, Kp = split_pitch(K);
    need(mid, size_t(H * Nr * Kp) * sizeof(cpx));
    AxisParams ap = base_params();
    ap.d0 = 4;
    ap.d1 = Q;
    ap.is0 = Q * N;
    ap.is1 = N;
    ap.is2 = Nr * N;
    ap.in_n = 1;
    ap.os0 = Q * Kp;
    ap.os1 = Kp;
    ap.os2 = Nr * Kp;
    ap.out_k = 1;
    ap.cpb = 4;
    ap.tw = tab(TB_TW, L);
    ap.t1 = tab(TB_RFT, N);
    ap.t2 = tab(TB_TW, Nr);
    add_axis_kernel(mb::K_R2CQ, int(L), H * Nr, ap, in_buf, mid, true, false);
    AxisParams cp = base_params();
    cp.d0 = K;
    cp.d1 = 4;
    cp.is0 = 1;
    cp.is1 = Q * Kp;
    cp.is2 = Nr * Kp;
    cp.in_n = Kp;
    cp.os0 = 1;
    cp.os1 = K;
    cp.os2 = Nr * K;
    cp.out_k = 4 * K;
    cp.colmode = 1;
    cp.cpb = choose_cpb(int(Q), true);
    cp.tw = tab(TB_TW, Q);
    add_axis_kernel(mb::K_CPLX, int(Q), H * 4 * K, cp, mid, out_buf, false, false);
  }

  // Inverse: length-Q inverse column DFTs of rows q + 4p, X -> block layout in
  // `mid`, then the fused radix-4 stage and the inverse real DFTs of the rows,
  // mid -> Y.
  void plan_invrealdft_split(int64_t H, int64_t Nr, int64_t N, int in_buf, int mid, int out_buf) {
    const int64_t K = N / 2 + 1, Q = Nr / 4, L = N / 2, Kp = split_pitch(K);
    need(mid, size_t(H * Nr * Kp) * sizeof(cpx));
    AxisParams cp = base_params();
    cp.d0 = K;
    cp.d1 = 4;
    cp.is0 = 1;
    cp.is1 = K;
    cp.is2 = Nr * K;
    cp.in_n = 4 * K;
    cp.os0 = 1;
    cp.os1 = Q * Kp;
    cp.os2 = Nr * Kp;
    cp.out_k = Kp;
    cp.colmode = 1;
    cp.flags = mb::F_CONJ_IN | mb::F_CONJ_OUT;
    cp.cpb = choose_cpb(int(Q), true);
    cp.tw = tab(TB_TW, Q);
    add_axis_kernel(mb::K_CPLX, int(Q), H * 4 * K, cp, in_buf, mid, false, false);
    AxisParams ap = base_params();
    ap.d0 = 4;
    ap.d1 = Q;
    ap.is0 = Q * Kp;
    ap.is1 = Kp;
    ap.is2 = Nr * Kp;
    ap.in_n = 1;
    ap.os0 = Q * N;
    ap.os1 = N;
    ap.os2 = Nr * N;
    ap.out_k = 1;
    ap.cpb = 4;
    ap.tw = tab(TB_TW, L);
    ap.t1 = tab(TB_TW, Nr);
    ap.t2 = tab(TB_RFT, N);
    add_axis_kernel(mb::K_C2RQ, int(L), H * Nr, ap, mid, out_buf, false, true);
  }

  void plan_axis(const AxisStep& s) {
    const size_t R_ = sizeof(real), C_ = sizeof(cpx);
    if (s.N == 1) {
      const int64_t cnt = s.outer * s.inner;
      const real r2 = real(1.414213562373095048801688724209698079);
      switch (s.combo) {
        case mb::K_CPLX:
          if (s.in_buf != s.out_buf) add_unit(mb::UNIT_COPY_CPLX, cnt, 1, s.in_buf, s.out_buf);
          break;
        case mb::K_R2C: add_unit(mb::UNIT_REAL_TO_CPLX, cnt, 1, s.in_buf, s.out_buf); break;
        case mb::K_C2R: add_unit(mb::UNIT_CPLX_TO_REAL, cnt, 1, s.in_buf, s.out_buf); break;
        case mb::K_DCT2: add_unit(mb::UNIT_SCALE_REAL, cnt, 2, s.in_buf, s.out_buf); break;
        case mb::K_DCT3:
          if (s.in_buf != s.out_buf) add_unit(mb::UNIT_SCALE_REAL, cnt, 1, s.in_buf, s.out_buf);
          break;
        case mb::K_T4: add_unit(mb::UNIT_SCALE_REAL, cnt, r2, s.in_buf, s.out_buf); break;
      }
      (void)R_;
      (void)C_;
      return;
    }
    const int64_t L = (s.combo == mb::K_CPLX) ? s.N : s.N / 2;
    const bool colmode = s.inner > 1;
    const int cap = colmode ? kColCapLog2 : kRowCapLog2;
    if (ilog2(L) <= cap) {
      AxisParams ap = base_params();
      ap.d0 = s.inner;
      ap.d1 = s.outer;
      ap.is0 = 1;
      ap.is1 = s.in_row;
      ap.in_n = s.inner;
      ap.os0 = 1;
      ap.os1 = s.out_row;
      ap.out_k = s.inner;
      ap.colmode = colmode ? 1 : 0;
      ap.cpb = choose_cpb((int)L, colmode);
      ap.flags = s.flags;
      ap.tw = tab(TB_TW, L);
      set_kind_tables(ap, s.combo, s.N);
      add_axis_kernel(s.combo, (int)L, s.outer * s.inner, ap, s.in_buf, s.out_buf, s.combo == mb::K_R2C,
                      s.combo == mb::K_C2R);
      return;
    }
    plan_multipass(s, L);
  }

  // Stockham FFT over HBM for a long axis (see the file comment).
  void plan_multipass(const AxisStep& s, int64_t Lt) {
    const int bits = ilog2(Lt);
    const int cap = pass_cap_log2(a->precision);
    int P = (bits + cap - 1) / cap;
    std::vector<int> pb = pass_bits(bits, P);
    // a tensor-core mode whose chain has no 256-point pass at the FP32 pass
    // count (2^17 .. 2^24 points in two passes) takes one more pass so that
    // its radix-16 stages run on the tensor cores
    if (a->precision != MINFFT_B200_PREC_FP32 && bits >= 2 * ilog2(mb::kTcLength) &&
        std::find(pb.begin(), pb.end(), ilog2(mb::kTcLength)) == pb.end()) {
      std::vector<int> more = pass_bits(bits, P + 1);
      if (std::find(more.begin(), more.end(), ilog2(mb::kTcLength)) != more.end()) {
        pb = more;
        P = P + 1;
      }
    }
    const int64_t inner = s.inner, outer = s.outer;
    const int64_t Lp = Lt * inner;
    const size_t work_bytes = size_t(outer) * size_t(Lp) * sizeof(cpx);
    const bool inverse_cplx = (s.combo == mb::K_CPLX) && (s.flags & mb::F_CONJ_IN);
    const bool conj_chain = inverse_cplx || s.combo == mb::K_C2R || s.combo == mb::K_DCT3;

    // --- pre-processing: chain source
    int cs = s.in_buf;
    auto line = [&](int64_t in_so, int64_t in_sn, int64_t out_so, int64_t out_sn) {
      LineParams lp{};
      lp.outer = outer;
      lp.inner = inner;
      lp.L = Lt;
      lp.in_so = in_so;
      lp.in_sn = in_sn;
      lp.out_so = out_so;
      lp.out_sn = out_sn;
      lp.flags = s.flags;
      return lp;
    };
    // A 1-D type-4 chain of two or more passes fuses its pre-rotation into
    // the first pass's load and its post-rotation into the last pass's store
    // (LoadT4Chain, StoreT4Chain): two passes over HBM instead of four.  In a
    // tensor-core mode only an end pass on the CUDA cores of 128 to 1024
    // points (the lengths the FP32 and FP64 type-4 chains take) fuses its
    // rotation: the 256-point tensor-core passes take plain complex input and
    // output.  The other rotation stays a separate element-wise step.
    // (the fused passes form their roots from 32-bit exponents into the tables of 8N)
    const bool t4_chain =
        s.combo == mb::K_T4 && inner == 1 && P >= 2 && s.N <= (int64_t(1) << 28) && t4_fuse_enabled();
    auto cuda_core_pass = [&](int p) {
      return a->precision == MINFFT_B200_PREC_FP32 ||
             ((int64_t(1) << pb[p]) != mb::kTcLength && pb[p] >= 7 && pb[p] <= kPassCapLog2Cc);
    };
    const bool t4_fused_in = t4_chain && cuda_core_pass(0);
    const bool t4_fused_out = t4_chain && cuda_core_pass(P - 1);
    if (!t4_fused_in &&
        (s.combo == mb::K_DCT2 || s.combo == mb::K_T4 || s.combo == mb::K_C2R || s.combo == mb::K_DCT3)) {
      cs = BUF_T2;
      need(cs, work_bytes);
      LineParams lp = line(s.in_row, inner, Lp, inner);
      int which = 0;
      int64_t items = outer * inner * Lt;
      if (s.combo == mb::K_DCT2) {
        which = mb::LK_DCT2_PRE;
      } else if (s.combo == mb::K_T4) {
        which = mb::LK_T4_PRE;
        set_root_pair(lp, 1, 2 * s.N, 1, 0);  // w_2N^n
        items = outer * inner * (Lt / 2);      // points n and Lt-1-n per item
      } else if (s.combo == mb::K_C2R) {
        which = mb::LK_C2R_PACK;
        set_root_pair(lp, 2, s.N, 1, 0);  // w_N^k
        items = outer * inner * (Lt / 2 + 1);
      } else {
        which = mb::LK_DCT3_PACK;
        set_root_pair(lp, 1, 4 * s.N, 1, 0);  // w_4N^n
        set_root_pair(lp, 2, s.N, 1, 0);      // w_N^k
        items = outer * inner * (Lt / 2 + 1);
      }
      add_line_kernel(which, lp, items, s.in_buf, cs);
    }
    const bool post = !t4_fused_out &&
                      (s.combo == mb::K_R2C || s.combo == mb::K_DCT2 || s.combo == mb::K_DCT3 || s.combo == mb::K_T4);

    // --- the HBM passes
    int prev = cs;
    int64_t Ns = 1;
    int cd = s.out_buf;
    for (int p = 0; p < P; ++p) {
      const int64_t Rp = int64_t(1) << pb[p];
      const bool last = (p == P - 1);
      int dst;
      if (!last) {
        dst = pick_temp({prev});
        need(dst, work_bytes);
      } else if (post) {
        dst = pick_temp({prev});
        need(dst, work_bytes);
        cd = dst;
      } else {
        dst = s.out_buf;
      }
      const bool fuse_in = t4_fused_in && p == 0, fuse_out = t4_fused_out && last;
      const int64_t Nsp = Ns * inner;
      AxisParams ap = base_params();
      ap.d0 = Nsp;
      ap.d1 = Lt / (Ns * Rp);
      ap.is0 = 1;
      ap.is1 = Nsp;
      ap.is2 = Lp;
      ap.in_n = Lp / Rp;
      ap.os0 = 1;
      ap.os1 = Nsp * Rp;
      ap.os2 = Lp;
      ap.out_k = Nsp;
      ap.st_ns = Ns;
      ap.st_div = inner;
      ap.st_shift = ilog2(Lt / (Ns * Rp));
      ap.st_lobits = (int)st_lobits_for(Lt);
      if (Ns > 1) {
        ap.st_hi = tab(TB_STHI, Lt);
        ap.st_lo = tab(TB_STLO, Lt);
      }
      ap.colmode = 1;
      ap.cpb = choose_cpb((int)Rp, true);
      ap.flags = 0;
      if (Nsp == 1) ap.flags |= mb::F_STAGE_ROWS;
      if (p == 0 && inverse_cplx) ap.flags |= mb::F_CONJ_IN;
      if (last && conj_chain && s.combo != mb::K_DCT3) ap.flags |= mb::F_CONJ_OUT;
      ap.tw = tab(TB_TW, Rp);
      int combo = mb::K_CPLX;
      if (fuse_in) {
        combo = mb::K_T4IN;
        ap.flags |= (s.flags & mb::F_DST);
        ap.st_hi = tab(TB_STHI, 2 * s.N);  // w_2N^g, coarse x fine
        ap.st_lo = tab(TB_STLO, 2 * s.N);
        ap.st_lobits = (int)st_lobits_for(2 * s.N);
        ap.is2 = 0;
        ap.kn = s.N;
        ap.k_in_line = s.in_row;
      }
      if (fuse_out) {
        combo = mb::K_T4OUT;
        ap.flags |= (s.flags & mb::F_DST);
        ap.t1 = tab(TB_STHI, 8 * s.N);  // w_8N^(2q+1), coarse x fine
        ap.t2 = tab(TB_STLO, 8 * s.N);
        ap.kbits = (int)st_lobits_for(8 * s.N);
        ap.os2 = 0;
        ap.kn = s.N;
        ap.k_out_line = s.out_row;
      }
      add_axis_kernel(combo, (int)Rp, outer * (Lp / Rp), ap, prev, dst, false, false);
      if (ok) prog->launches.back().hbm_pass = true;
      prev = dst;
      Ns *= Rp;
    }

    // --- post-processing
    if (post) {
      LineParams lp = line(Lp, inner, s.out_row, inner);
      int which = 0;
      int64_t items = outer * inner * (Lt / 2 + 1);
      if (s.combo == mb::K_R2C) {
        which = mb::LK_R2C_UNPACK;
        set_root_pair(lp, 1, s.N, 1, 0);  // w_N^k
      } else if (s.combo == mb::K_DCT2) {
        which = mb::LK_DCT2_POST;
        set_root_pair(lp, 1, 4 * s.N, 1, 0);  // w_4N^n
        set_root_pair(lp, 2, s.N, 1, 0);      // w_N^k
      } else if (s.combo == mb::K_DCT3) {
        which = mb::LK_DCT3_POST;
        items = outer * inner * Lt;
      } else {
        which = mb::LK_T4_POST;
        set_root_pair(lp, 2, 8 * s.N, 2, 1);  // w_8N^(2q+1)
        items = outer * inner * (Lt / 2);      // points m and Lt-1-m per item
      }
      add_line_kernel(which, lp, items, cd, s.out_buf);
    }
  }
};

// ----------------------------------------------------- program building
struct Shape {
  std::vector<int64_t> d;  // dims with the batch count prepended
};

int64_t prod(const std::vector<int64_t>& v, size_t b, size_t e) {
  int64_t p = 1;
  for (size_t i = b; i < e; ++i) p *= v[i];
  return p;
}

bool build_program(minfft_aux* a, int op, int howmany, bool alias, Program* prog) {
  DeviceInfo di = device_info(a->device);
  Planner pl{a, prog, di.max_smem, di.sms};
  // full shape with the batch count as a leading, untransformed axis
  std::vector<int64_t> D;
  D.push_back(howmany);
  for (int n : a->dims) D.push_back(n);
  const size_t nd = D.size();  // >= 2
  const bool multi = (nd > 2) || howmany > 1;

  auto complex_axes = [&](std::vector<int64_t> shape, size_t first, size_t last_excl, int flags, int in_buf,
                          int out_buf, bool reverse) {
    // complex DFT along axes [first, last_excl) of `shape`
    int cur = in_buf;
    std::vector<size_t> order;
    for (size_t ax = first; ax < last_excl; ++ax) order.push_back(ax);
    if (reverse) std::reverse(order.begin(), order.end());
    for (size_t ax : order) {
      AxisStep s{};
      s.combo = mb::K_CPLX;
      s.N = shape[ax];
      s.outer = prod(shape, 0, ax);
      s.inner = prod(shape, ax + 1, shape.size());
      s.in_row = s.N * s.inner;
      s.out_row = s.in_row;
      s.flags = flags;
      s.in_buf = cur;
      s.out_buf = out_buf;
      pl.plan_axis(s);
      if (!(s.N == 1 && cur == out_buf)) cur = out_buf;
    }
    return cur;
  };

  switch (op) {
    case MINFFT_B200_DFT:
    case MINFFT_B200_INVDFT: {
      const int fl = (op == MINFFT_B200_INVDFT) ? (mb::F_CONJ_IN | mb::F_CONJ_OUT) : 0;
      int cur = complex_axes(D, 1, nd, fl, BUF_X, BUF_Y, true);
      if (cur != BUF_Y) pl.add_unit(mb::UNIT_COPY_CPLX, prod(D, 0, nd), 1, cur, BUF_Y);
      break;
    }
    case MINFFT_B200_REALDFT: {
      const int64_t N = D[nd - 1], K = N / 2 + 1;
      const bool via_t1 = alias && multi;
      std::vector<int64_t> H(D);
      H[nd - 1] = K;
      const size_t spec_bytes = size_t(prod(H, 0, nd)) * sizeof(cpx);
      if (nd == 3 && pl.split_2d(D[1], N)) {
        pl.need(BUF_T1, spec_bytes);
        pl.plan_realdft_split(D[0], D[1], N, BUF_X, BUF_T1, BUF_Y);
        break;
      }
      AxisStep s{};
      s.combo = mb::K_R2C;
      s.N = N;
      s.outer = prod(D, 0, nd - 1);
      s.inner = 1;
      s.in_row = N;
      s.out_row = K;
      s.in_buf = BUF_X;
      s.out_buf = via_t1 ? BUF_T1 : BUF_Y;
      if (via_t1) pl.need(BUF_T1, spec_bytes);
      pl.plan_axis(s);
      int cur = complex_axes(H, 1, nd - 1, 0, s.out_buf, BUF_Y, true);
      if (cur != BUF_Y) pl.add_unit(mb::UNIT_COPY_CPLX, prod(H, 0, nd), 1, cur, BUF_Y);
      break;
    }
    case MINFFT_B200_INVREALDFT: {
      const int64_t N = D[nd - 1], K = N / 2 + 1;
      std::vector<int64_t> H(D);
      H[nd - 1] = K;
      const size_t spec_bytes = size_t(prod(H, 0, nd)) * sizeof(cpx);
      if (nd == 3 && pl.split_2d(D[1], N)) {
        pl.need(BUF_T1, spec_bytes);
        pl.plan_invrealdft_split(D[0], D[1], N, BUF_X, BUF_T1, BUF_Y);
        break;
      }
      int src = BUF_X;
      if (nd > 2) {
        pl.need(BUF_T1, spec_bytes);
        src = complex_axes(H, 1, nd - 1, mb::F_CONJ_IN | mb::F_CONJ_OUT, BUF_X, BUF_T1, false);
      }
      const bool via_t1 = alias && howmany > 1 && nd == 2;
      AxisStep s{};
      s.combo = mb::K_C2R;
      s.N = N;
      s.outer = prod(D, 0, nd - 1);
      s.inner = 1;
      s.in_row = K;
      s.out_row = N;
      s.in_buf = src;
      s.out_buf = via_t1 ? BUF_T1 : BUF_Y;
      if (via_t1) pl.need(BUF_T1, size_t(prod(D, 0, nd)) * sizeof(real));
      pl.plan_axis(s);
      if (via_t1) pl.add_unit(mb::UNIT_SCALE_REAL, prod(D, 0, nd), 1, BUF_T1, BUF_Y);
      break;
    }
    default: {
      int combo = mb::K_T4, fl = 0;
      if (op == MINFFT_B200_DCT2 || op == MINFFT_B200_DST2) combo = mb::K_DCT2;
      if (op == MINFFT_B200_DCT3 || op == MINFFT_B200_DST3) combo = mb::K_DCT3;
      if (op == MINFFT_B200_DST2 || op == MINFFT_B200_DST3 || op == MINFFT_B200_DST4) fl = mb::F_DST;
      if (nd == 3 && combo != mb::K_T4 && pl.split_dct(D[1], D[2])) {
        // the 2-D split column DFT: blocks of the column DFT in T1
        const size_t blocks = size_t(D[0] * D[1] * D[2]) * sizeof(real);
        pl.need(BUF_T1, blocks);
        if (combo == mb::K_DCT2) {
          pl.add_dctq(0, D[0], D[1], D[2], fl, BUF_X, BUF_T1, BUF_T1);
          pl.add_dctq(1, D[0], D[1], D[2], fl, BUF_T1, BUF_Y, BUF_T1);
        } else {
          pl.add_dctq(2, D[0], D[1], D[2], fl, BUF_X, BUF_T1, BUF_T1);
          pl.add_dctq(3, D[0], D[1], D[2], fl, BUF_T1, BUF_Y, BUF_T1);
        }
        break;
      }
      int cur = BUF_X;
      for (size_t ax = nd - 1; ax >= 1; --ax) {
        AxisStep s{};
        s.combo = combo;
        s.N = D[ax];
        s.outer = prod(D, 0, ax);
        s.inner = prod(D, ax + 1, nd);
        s.in_row = s.N * s.inner;
        s.out_row = s.in_row;
        s.flags = fl;
        s.in_buf = cur;
        s.out_buf = BUF_Y;
        pl.plan_axis(s);
        if (!(s.N == 1 && combo == mb::K_DCT3 && cur == BUF_Y)) cur = BUF_Y;
      }
      if (cur != BUF_Y) pl.add_unit(mb::UNIT_SCALE_REAL, prod(D, 0, nd), 1, cur, BUF_Y);
      break;
    }
  }
  return pl.ok;
}

// bytes of one input / output array of op for plan a
int64_t io_bytes(const minfft_aux* a, int op, bool output) {
  const int64_t p = a->total;
  const int64_t N = a->dims.back();
  const int64_t spec = (p / N) * (N / 2 + 1);
  switch (op) {
    case MINFFT_B200_DFT:
    case MINFFT_B200_INVDFT: return p * (int64_t)sizeof(cpx);
    case MINFFT_B200_REALDFT: return output ? spec * (int64_t)sizeof(cpx) : p * (int64_t)sizeof(real);
    case MINFFT_B200_INVREALDFT: return output ? p * (int64_t)sizeof(real) : spec * (int64_t)sizeof(cpx);
    default: return p * (int64_t)sizeof(real);
  }
}

bool ensure_buffer(minfft_aux* a, int buf, size_t bytes) {
  if (bytes == 0 || a->buf_bytes[buf] >= bytes) return true;
  if (a->bufs[buf]) cudaFree(a->bufs[buf]);
  a->bufs[buf] = nullptr;
  a->buf_bytes[buf] = 0;
  void* p = nullptr;
  if (!cuda_ok(mb::dev_malloc(&p, bytes), "cudaMalloc(scratch)")) return false;
  a->bufs[buf] = p;
  a->buf_bytes[buf] = bytes;
  return true;
}

Program* get_program(minfft_aux* a, int op, int howmany, bool alias) {
  auto key = std::make_tuple(op, howmany, alias ? 1 : 0);
  auto it = a->programs.find(key);
  if (it != a->programs.end()) return &it->second;
  Program prog;
  if (!build_program(a, op, howmany, alias, &prog)) return nullptr;
  if (!a->host_only)
    for (int b = BUF_T1; b < BUF_COUNT; ++b)
      if (!ensure_buffer(a, b, prog.tbytes[b])) return nullptr;
  return &(a->programs[key] = std::move(prog));
}

enum PtrKind { PTR_PAGEABLE = 0, PTR_PINNED, PTR_DEVICE };

PtrKind pointer_kind(const void* p) {
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return PTR_PAGEABLE;
  }
  if (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) return PTR_DEVICE;
  return attr.type == cudaMemoryTypeHost ? PTR_PINNED : PTR_PAGEABLE;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// Programmatic dependent launch for the planner's kernels (every one of them
// starts with pdl_release / pdl_wait): consecutive launches of a program
// overlap the next kernel's scheduling with the previous one's drain.
// MINFFT_B200_PDL=0 turns it off.
bool pdl_enabled() {
  static const bool on = [] {
    const char* e = getenv("MINFFT_B200_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}

bool enqueue(minfft_aux* a, const Launch& ln, void** args, size_t smem, const char* what) {
  if (!pdl_enabled()) return cuda_ok(cudaLaunchKernel(ln.fn, dim3(ln.grid), dim3(ln.block), args, smem, a->stream), what);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ln.grid);
  cfg.blockDim = dim3(ln.block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = a->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cuda_ok(cudaLaunchKernelExC(&cfg, ln.fn, args), what);
}

// Enqueue one planned launch with its buffers resolved.
// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links only the runtime).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return EncodeTiledFn(nullptr);
    }
    return reinterpret_cast<EncodeTiledFn>(f);
  }();
  return fn;
}

// Tensor map of a streamed pass's input: dims (2*d0 reals, L elements, d1,
// d2), box (2W reals, min(L, 256) elements, 1, 1).  False where the address
// or a stride breaks the 16-byte rules of tensor copies; the kernel then
// copies with cp.async.
bool stream_map(CUtensorMap* m, const Launch& ln, const AxisParams& ap) {
  const uint64_t C = sizeof(cpx);
  const uint64_t s1 = uint64_t(ap.in_n) * C, s2 = uint64_t(ap.is1) * C, s3 = uint64_t(ap.is2) * C;
  const uint64_t d2 = uint64_t(ln.st_d2);
  if ((reinterpret_cast<uintptr_t>(ap.in) & 15) || (s1 & 15) || (ap.d1 > 1 && (s2 & 15)) || (d2 > 1 && (s3 & 15)))
    return false;
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  const cuuint64_t dims[4] = {cuuint64_t(2 * ap.d0), cuuint64_t(ln.L), cuuint64_t(ap.d1), cuuint64_t(d2)};
  // unit extents get a harmless stride (the coordinate is always 0)
  const uint64_t span1 = s1 * uint64_t(ln.L);
  const uint64_t st1 = ap.d1 > 1 ? s2 : (span1 + 15) / 16 * 16;
  const uint64_t st2 = d2 > 1 ? s3 : (st1 * uint64_t(ap.d1) + 15) / 16 * 16;
  const cuuint64_t strides[3] = {cuuint64_t(s1), cuuint64_t(st1), cuuint64_t(st2)};
  const cuuint32_t box[4] = {cuuint32_t(2 * mb::stream_cols()), cuuint32_t(ln.L < 256 ? ln.L : 256), 1, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  for (int i = 0; i < 3; ++i)
    if (strides[i] >= (uint64_t(1) << 40)) return false;
  const CUtensorMapDataType dt = sizeof(real) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  return fn(m, dt, 4, const_cast<void*>(ap.in), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor map of a streamed tensor-core pass's input (complex single
// precision): column tiles dims (2*d0 reals, 256 points, d1, d2), box (32
// reals, 128 points); row tiles dims (512 reals, d0 transforms, d1, d2), box
// (256 reals, 16 transforms).
bool tc_stream_map(CUtensorMap* m, const Launch& ln, const AxisParams& ap) {
  const uint64_t C = sizeof(cpx);
  const uint64_t d2 = uint64_t(ln.st_d2);
  const bool rows = ln.tcs == 2;
  const uint64_t s1 = rows ? uint64_t(ap.is0) * C : uint64_t(ap.in_n) * C;
  const uint64_t s2 = uint64_t(ap.is1) * C, s3 = uint64_t(ap.is2) * C;
  if ((reinterpret_cast<uintptr_t>(ap.in) & 15) || (s1 & 15) || (ap.d1 > 1 && (s2 & 15)) || (d2 > 1 && (s3 & 15)))
    return false;
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  const uint64_t n1 = rows ? uint64_t(ap.d0) : uint64_t(ln.L);
  const cuuint64_t dims[4] = {cuuint64_t(rows ? 2 * ln.L : 2 * ap.d0), cuuint64_t(n1), cuuint64_t(ap.d1),
                              cuuint64_t(d2)};
  const uint64_t st1 = ap.d1 > 1 ? s2 : (s1 * n1 + 15) / 16 * 16;
  const uint64_t st2 = d2 > 1 ? s3 : (st1 * uint64_t(ap.d1) + 15) / 16 * 16;
  const cuuint64_t strides[3] = {cuuint64_t(s1), cuuint64_t(st1), cuuint64_t(st2)};
  for (int i = 0; i < 3; ++i)
    if (strides[i] >= (uint64_t(1) << 40)) return false;
  const cuuint32_t box[4] = {cuuint32_t(rows ? 256 : 2 * mb::kTcStreamTile), cuuint32_t(rows ? mb::kTcStreamTile : 128),
                              1, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<void*>(ap.in), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool launch_one(minfft_aux* a, const Launch& ln, void* const* bufs) {
  void* args[1];
  if (ln.is_line) {
    LineParams lp = ln.lp;
    lp.in = bufs[ln.in_buf];
    lp.out = bufs[ln.out_buf];
    args[0] = &lp;
    return enqueue(a, ln, args, 0, "launch(line)");
  }
  AxisParams ap = ln.ap;
  ap.in = bufs[ln.in_buf];
  ap.out = bufs[ln.out_buf];
  ap.status = a->dev_status;
  if (ln.vec_in && (reinterpret_cast<uintptr_t>(ap.in) % sizeof(cpx)) == 0) ap.flags |= mb::F_VEC;
  if (ln.vec_out && (reinterpret_cast<uintptr_t>(ap.out) % sizeof(cpx)) == 0) ap.flags |= mb::F_VEC;
  if (ln.pipe) {
    int ch = ln.ch_static;
    while (ch > 4 && (reinterpret_cast<uintptr_t>(ap.in) % ch) != 0) ch /= 2;
    ap.chunk = ch;
  }
  if (ln.dctq >= 0) {
    mb::DctqParams d = ln.dq;
    d.in = bufs[ln.in_buf];
    d.out = bufs[ln.out_buf];
    d.mid = static_cast<cpx*>(bufs[ln.mid_buf]);
    void* dargs[1] = {&d};
    return enqueue(a, ln, dargs, ln.smem, "launch(dct split)");
  }
  if (ln.dctq >= 0) {
    mb::DctqParams d = ln.dq;
    d.in = bufs[ln.in_buf];
    d.out = bufs[ln.out_buf];
    d.mid = static_cast<cpx*>(bufs[ln.mid_buf]);
    void* dargs[1] = {&d};
    return enqueue(a, ln, dargs, ln.smem, "launch(dct split)");
  }
  if (ln.stream_rows) {
    // one bulk copy per row where the rows start on 16-byte boundaries,
    // else per-thread cp.async in the largest chunk the addresses allow
    const uintptr_t base = reinterpret_cast<uintptr_t>(ap.in);
    if ((base & 15) == 0 && ln.ch_static == 16)
      ap.flags |= mb::F_STREAM_TMA;
    int ch = ln.ch_static;
    while (ch > 4 && (base % ch) != 0) ch /= 2;
    ap.chunk = ch;
    args[0] = &ap;
    return enqueue(a, ln, args, ln.smem, "launch(stream rows)");
  }
  if (ln.stream) {
    alignas(64) CUtensorMap map;
    memset(&map, 0, sizeof(map));
    if (stream_map(&map, ln, ap))
      ap.flags |= mb::F_STREAM_TMA;
    else if (reinterpret_cast<uintptr_t>(ap.in) % sizeof(cpx)) {
      set_error(MINFFT_B200_EINVAL, "complex input not aligned to its size");
      return false;
    }
    void* sargs[2] = {&ap, &map};
    return enqueue(a, ln, sargs, ln.smem, "launch(stream)");
  }
  if (ln.tc) {
    mb::TcParams tcp = ln.tcp;
    const long long withhold = g_tc_withhold.load();
    if (withhold > 0) {
      tcp.withhold = 1;
      tcp.wait_polls = withhold;
    }
    if (ln.tcs) {
      alignas(64) CUtensorMap map;
      memset(&map, 0, sizeof(map));
      if (tc_stream_map(&map, ln, ap)) ap.flags |= mb::F_STREAM_TMA;
      void* sargs[3] = {&ap, &tcp, &map};
      return enqueue(a, ln, sargs, ln.smem, "launch(tc stream)");
    }
    void* targs[2] = {&ap, &tcp};
    return enqueue(a, ln, targs, ln.smem, "launch(tc)");
  }
  args[0] = &ap;
  return enqueue(a, ln, args, ln.smem, "launch(axis)");
}

bool run_program(minfft_aux* a, Program* prog, void* x, void* y) {
  void* bufs[BUF_COUNT];
  bufs[BUF_X] = x;
  bufs[BUF_Y] = y;
  for (int b = BUF_T1; b < BUF_COUNT; ++b) bufs[b] = a->bufs[b];
  // complex data is accessed as aligned float2/double2: reject user buffers
  // that are not, before anything is launched
  for (const Launch& ln : prog->launches) {
    const bool bad_in = ln.in_c && (reinterpret_cast<uintptr_t>(bufs[ln.in_buf]) % sizeof(cpx)) != 0;
    const bool bad_out = ln.out_c && (reinterpret_cast<uintptr_t>(bufs[ln.out_buf]) % sizeof(cpx)) != 0;
    if (bad_in || bad_out) {
      set_error(MINFFT_B200_EINVAL, "complex data must be aligned to %zu bytes", sizeof(cpx));
      return false;
    }
  }
  for (Launch& ln : prog->launches) {
    size_t ev0 = 0;
    if (a->prof) {
      while (a->ev_pool.size() < a->ev_used + 2) {
        cudaEvent_t e;
        if (!cuda_ok(cudaEventCreate(&e), "cudaEventCreate")) return false;
        a->ev_pool.push_back(e);
      }
      ev0 = a->ev_used;
      a->ev_used += 2;
      if (!cuda_ok(cudaEventRecord(a->ev_pool[ev0], a->stream), "cudaEventRecord")) return false;
    }
    if (!launch_one(a, ln, bufs)) return false;
    if (a->prof) {
      if (!cuda_ok(cudaEventRecord(a->ev_pool[ev0 + 1], a->stream), "cudaEventRecord")) return false;
      a->pending.push_back({&ln, ev0, ev0 + 1});
    }
  }
  return true;
}

// Fold recorded launch timings into the per-label statistics.
bool harvest(minfft_aux* a) {
  if (a->pending.empty()) return true;
  if (!cuda_ok(cudaEventSynchronize(a->ev_pool[a->pending.back().e1]), "cudaEventSynchronize")) return false;
  for (const auto& pe : a->pending) {
    float ms = 0;
    if (!cuda_ok(cudaEventElapsedTime(&ms, a->ev_pool[pe.e0], a->ev_pool[pe.e1]), "cudaEventElapsedTime"))
      return false;
    auto it = std::find_if(a->stats.begin(), a->stats.end(),
                           [&](const minfft_aux::Stat& st) { return st.label == pe.ln->label; });
    if (it == a->stats.end()) {
      a->stats.push_back(minfft_aux::Stat());
      it = a->stats.end() - 1;
      it->label = pe.ln->label;
      it->bytes = pe.ln->bytes;
    }
    it->launches += 1;
    it->ms += ms;
  }
  a->pending.clear();
  a->ev_used = 0;
  return true;
}

bool grow(void** p, size_t* have, size_t want) {
  if (*have >= want) return true;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  if (!cuda_ok(mb::dev_malloc(p, want), "cudaMalloc(staging)")) return false;
  *have = want;
  return true;
}

int execute(int op, void* x, void* y, int howmany, const minfft_aux* ca) {
  minfft_aux* a = const_cast<minfft_aux*>(ca);
  if (!a) {
    set_error(MINFFT_B200_EINVAL, "NULL plan");
    return MINFFT_B200_EINVAL;
  }
  if (op_family(op) != a->family) {
    set_error(MINFFT_B200_EINVAL, "transform %d does not match the plan kind %d", op, a->family);
    return MINFFT_B200_EINVAL;
  }
  if (!x || !y || howmany < 1) {
    set_error(MINFFT_B200_EINVAL, "NULL data pointer or howmany < 1");
    return MINFFT_B200_EINVAL;
  }
  DeviceGuard guard(a->device);
  const size_t in_b = size_t(io_bytes(a, op, false)) * howmany;
  const size_t out_b = size_t(io_bytes(a, op, true)) * howmany;
  const PtrKind xk = pointer_kind(x), yk = pointer_kind(y);
  const bool x_dev = xk == PTR_DEVICE, y_dev = yk == PTR_DEVICE;
  // host arrays are staged through device buffers; the call waits for its
  // result unless the plan is in host-async mode and both arrays are
  // page-locked (then everything stays ordered on the plan's stream)
  const bool wait_host = !(a->host_async && xk != PTR_PAGEABLE && yk != PTR_PAGEABLE);
  void* dx = x;
  void* dy = y;
  const bool same = (x == y);
  if (!x_dev) {
    if (!grow(&a->stage_in, &a->stage_in_bytes, std::max(in_b, same ? out_b : 0))) return g_err;
    dx = a->stage_in;
    if (!cuda_ok(cudaMemcpyAsync(dx, x, in_b, cudaMemcpyHostToDevice, a->stream), "cudaMemcpyAsync(H2D)"))
      return g_err;
  }
  if (!y_dev) {
    if (same) {
      dy = dx;
    } else {
      if (!grow(&a->stage_out, &a->stage_out_bytes, out_b)) return g_err;
      dy = a->stage_out;
    }
  }
  const uintptr_t xs = reinterpret_cast<uintptr_t>(dx), ys = reinterpret_cast<uintptr_t>(dy);
  const bool alias = (xs < ys + out_b) && (ys < xs + in_b);
  Program* prog = get_program(a, op, howmany, alias);
  if (!prog) return g_err ? g_err : MINFFT_B200_ECUDA;
  if (!run_program(a, prog, dx, dy)) return g_err;
  if (!y_dev) {
    if (!cuda_ok(cudaMemcpyAsync(y, dy, out_b, cudaMemcpyDeviceToHost, a->stream), "cudaMemcpyAsync(D2H)"))
      return g_err;
    if (wait_host && !cuda_ok(cudaStreamSynchronize(a->stream), "cudaStreamSynchronize")) return g_err;
  }
  return MINFFT_B200_OK;
}

// ---------------------------------------------------------------- makers
minfft_aux* make_plan(int family, int d, const int* Ns) {
  if (d < 1 || Ns == nullptr) {
    set_error(MINFFT_B200_EINVAL, "dimension count must be >= 1");
    return nullptr;
  }
  int64_t total = 1;
  for (int i = 0; i < d; ++i) {
    if (!is_pow2(Ns[i])) {
      set_error(MINFFT_B200_EINVAL, "length %d is not a positive power of two", Ns[i]);
      return nullptr;
    }
    total *= Ns[i];
  }
  if (total > (int64_t(1) << 31)) {
    set_error(MINFFT_B200_EINVAL, "transform size exceeds 2^31 elements");
    return nullptr;
  }
  minfft_aux* a = new (std::nothrow) minfft_aux();
  if (!a) {
    set_error(MINFFT_B200_ENOMEM, "host allocation failed");
    return nullptr;
  }
  a->family = family;
  a->dims.assign(Ns, Ns + d);
  a->total = total;
  if (!cuda_ok(cudaGetDevice(&a->device), "cudaGetDevice")) {
    delete a;
    return nullptr;
  }
  {
    void* st = nullptr;
    if (!cuda_ok(mb::dev_malloc(&st, 16), "cudaMalloc(status)") || !cuda_ok(cudaMemset(st, 0, 16), "cudaMemset(status)")) {
      if (st) cudaFree(st);
      delete a;
      return nullptr;
    }
    a->dev_status = static_cast<int*>(st);
  }
  // plan every transform of the family (out of place, one array) now, so
  // tables and scratch are allocated up front as the reference's makers do
  static const int fam_ops[4][4] = {{MINFFT_B200_DFT, MINFFT_B200_INVDFT, -1, -1},
                                    {MINFFT_B200_REALDFT, MINFFT_B200_INVREALDFT, -1, -1},
                                    {MINFFT_B200_DCT2, MINFFT_B200_DST2, MINFFT_B200_DCT3, MINFFT_B200_DST3},
                                    {MINFFT_B200_DCT4, MINFFT_B200_DST4, -1, -1}};
  for (int k = 0; k < 4; ++k) {
    const int op = fam_ops[family][k];
    if (op < 0) continue;
    if (!get_program(a, op, 1, false)) {
      minfft_free_aux(a);
      return nullptr;
    }
  }
  return a;
}

}  // namespace

// ===================================================================== ABI
MB_EXPORT void minfft_free_aux(minfft_aux* a) {
  if (!a) return;
  {
    DeviceGuard guard(a->device);
    for (auto& kv : a->tables) cudaFree(kv.second);
    for (int b = 0; b < BUF_COUNT; ++b)
      if (a->bufs[b]) cudaFree(a->bufs[b]);
    if (a->stage_in) cudaFree(a->stage_in);
    if (a->stage_out) cudaFree(a->stage_out);
    if (a->tc_mem) cudaFree(a->tc_mem);
    if (a->dev_status) cudaFree(a->dev_status);
    for (cudaEvent_t e : a->ev_pool) cudaEventDestroy(e);
  }
  delete a;
}

#define MB_TRANSFORM(name, code, TI, TO)                                   \
  MB_EXPORT void minfft_##name(TI* x, TO* y, const minfft_aux* a) {       \
    execute(code, static_cast<void*>(x), static_cast<void*>(y), 1, a);    \
  }

MB_TRANSFORM(dft, MINFFT_B200_DFT, minfft_cmpl, minfft_cmpl)
MB_TRANSFORM(invdft, MINFFT_B200_INVDFT, minfft_cmpl, minfft_cmpl)
MB_TRANSFORM(realdft, MINFFT_B200_REALDFT, minfft_real, minfft_cmpl)
MB_TRANSFORM(invrealdft, MINFFT_B200_INVREALDFT, minfft_cmpl, minfft_real)
MB_TRANSFORM(dct2, MINFFT_B200_DCT2, minfft_real, minfft_real)
MB_TRANSFORM(dst2, MINFFT_B200_DST2, minfft_real, minfft_real)
MB_TRANSFORM(dct3, MINFFT_B200_DCT3, minfft_real, minfft_real)
MB_TRANSFORM(dst3, MINFFT_B200_DST3, minfft_real, minfft_real)
MB_TRANSFORM(dct4, MINFFT_B200_DCT4, minfft_real, minfft_real)
MB_TRANSFORM(dst4, MINFFT_B200_DST4, minfft_real, minfft_real)

#define MB_MAKERS(fam, code)                                                                      \
  MB_EXPORT minfft_aux* minfft_mkaux_##fam(int d, int* Ns) { return make_plan(code, d, Ns); }    \
  MB_EXPORT minfft_aux* minfft_mkaux_##fam##_1d(int N) { return make_plan(code, 1, &N); }        \
  MB_EXPORT minfft_aux* minfft_mkaux_##fam##_2d(int N1, int N2) {                                 \
    int Ns[2] = {N1, N2};                                                                         \
    return make_plan(code, 2, Ns);                                                                \
  }                                                                                               \
  MB_EXPORT minfft_aux* minfft_mkaux_##fam##_3d(int N1, int N2, int N3) {                         \
    int Ns[3] = {N1, N2, N3};                                                                     \
    return make_plan(code, 3, Ns);                                                                \
  }

MB_MAKERS(dft, FAM_DFT)
MB_MAKERS(realdft, FAM_REALDFT)
MB_MAKERS(t2t3, FAM_T2T3)
MB_MAKERS(t4, FAM_T4)

// ------------------------------------------------------------ extensions
MB_EXPORT int minfft_b200_last_error(void) {
  const int e = g_err;
  g_err = 0;
  return e;
}

MB_EXPORT const char* minfft_b200_last_error_message(void) { return g_msg; }

MB_EXPORT int minfft_b200_set_stream(minfft_aux* a, void* stream) {
  if (!a) {
    set_error(MINFFT_B200_EINVAL, "NULL plan");
    return MINFFT_B200_EINVAL;
  }
  a->stream = static_cast<cudaStream_t>(stream);
  return MINFFT_B200_OK;
}

MB_EXPORT void* minfft_b200_get_stream(const minfft_aux* a) { return a ? static_cast<void*>(a->stream) : nullptr; }

MB_EXPORT int minfft_b200_synchronize(const minfft_aux* a) {
  if (!a) {
    set_error(MINFFT_B200_EINVAL, "NULL plan");
    return MINFFT_B200_EINVAL;
  }
  DeviceGuard guard(a->device);
  return cuda_ok(cudaStreamSynchronize(a->stream), "cudaStreamSynchronize") ? MINFFT_B200_OK : g_err;
}

MB_EXPORT int minfft_b200_execute_batch(int op, void* x, void* y, int howmany, const minfft_aux* a) {
  return execute(op, x, y, howmany, a);
}

MB_EXPORT long long minfft_b200_input_bytes(int op, const minfft_aux* a) {
  if (!a || op_family(op) != a->family) return -1;
  return io_bytes(a, op, false);
}

MB_EXPORT long long minfft_b200_output_bytes(int op, const minfft_aux* a) {
  if (!a || op_family(op) != a->family) return -1;
  return io_bytes(a, op, true);
}

MB_EXPORT long long minfft_b200_plan_bytes(const minfft_aux* a) {
  if (!a) return -1;
  long long b = (long long)a->table_bytes;
  for (int i = 0; i < BUF_COUNT; ++i) b += (long long)a->buf_bytes[i];
  return b;
}

MB_EXPORT int minfft_b200_launch_count(int op, const minfft_aux* ca) {
  minfft_aux* a = const_cast<minfft_aux*>(ca);
  if (!a || op_family(op) != a->family) return -1;
  DeviceGuard guard(a->device);
  Program* p = get_program(a, op, 1, false);
  return p ? (int)p->launches.size() : -1;
}

MB_EXPORT int minfft_b200_set_precision(minfft_aux* a, int mode) {
  if (!a || mode < MINFFT_B200_PREC_FP32 || mode > MINFFT_B200_PREC_TC_BF16) {
    set_error(MINFFT_B200_EINVAL, "bad precision arguments");
    return MINFFT_B200_EINVAL;
  }
  if (mode != MINFFT_B200_PREC_FP32 && sizeof(real) != 4) {
    set_error(MINFFT_B200_EUNSUPPORTED, "tensor-core passes exist in the single-precision library only");
    return MINFFT_B200_EUNSUPPORTED;
  }
  if (mode != MINFFT_B200_PREC_FP32 && !a->tc_mem) {
    // both formats' B operands, then the status word
    DeviceGuard guard(a->device);
    const size_t b16 = mb::tc_bmat_bytes(mb::TC_F16), bb = mb::tc_bmat_bytes(mb::TC_BF16);
    std::vector<uint16_t> img, img2;
    mb::tc_bmat_host(mb::TC_F16, img);
    mb::tc_bmat_host(mb::TC_BF16, img2);
    img.insert(img.end(), img2.begin(), img2.end());
    img.resize(img.size() + 8, 0);
    void* d = nullptr;
    if (!cuda_ok(mb::dev_malloc(&d, b16 + bb + 16), "cudaMalloc(tc operands)")) return g_err;
    if (!cuda_ok(cudaMemcpy(d, img.data(), b16 + bb + 16, cudaMemcpyHostToDevice), "cudaMemcpy(tc operands)")) {
      cudaFree(d);
      return g_err;
    }
    a->tc_mem = d;
    a->table_bytes += b16 + bb + 16;
  }
  if (a->precision != mode) {
    a->precision = mode;
    a->programs.clear();
  }
  return MINFFT_B200_OK;
}

MB_EXPORT int minfft_b200_get_precision(const minfft_aux* a) { return a ? a->precision : -1; }

MB_EXPORT int minfft_b200_set_host_async(minfft_aux* a, int enable) {
  if (!a) {
    set_error(MINFFT_B200_EINVAL, "NULL plan");
    return MINFFT_B200_EINVAL;
  }
  a->host_async = enable != 0;
  return MINFFT_B200_OK;
}

MB_EXPORT int minfft_b200_device_status(const minfft_aux* ca) {
  if (!ca) {
    set_error(MINFFT_B200_EINVAL, "NULL plan");
    return MINFFT_B200_EINVAL;
  }
  if (!ca->dev_status) return MINFFT_B200_OK;
  DeviceGuard guard(ca->device);
  if (!cuda_ok(cudaStreamSynchronize(ca->stream), "cudaStreamSynchronize")) return g_err;
  int v = 0;
  if (!cuda_ok(cudaMemcpy(&v, ca->dev_status, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy(status)"))
    return g_err;
  if (v) {
    const int zero = 0;
    cudaMemcpy(ca->dev_status, &zero, sizeof(int), cudaMemcpyHostToDevice);
    set_error(MINFFT_B200_ETIMEOUT, "a kernel gave up waiting on a device-side barrier");
    return MINFFT_B200_ETIMEOUT;
  }
  return MINFFT_B200_OK;
}

MB_EXPORT int minfft_b200_tc_status(const minfft_aux* ca) { return minfft_b200_device_status(ca); }

MB_EXPORT int minfft_b200_profile(minfft_aux* a, int enable) {
  if (!a) {
    set_error(MINFFT_B200_EINVAL, "NULL plan");
    return MINFFT_B200_EINVAL;
  }
  DeviceGuard guard(a->device);
  if (!harvest(a)) return g_err;
  a->prof = enable != 0;
  a->stats.clear();
  // enable > 1 reserves events for that many launches up front, so event
  // creation stays out of a timed region
  while (enable > 1 && a->ev_pool.size() < size_t(2) * size_t(enable)) {
    cudaEvent_t e;
    if (!cuda_ok(cudaEventCreate(&e), "cudaEventCreate")) return g_err;
    a->ev_pool.push_back(e);
  }
  return MINFFT_B200_OK;
}

MB_EXPORT int minfft_b200_profile_count(minfft_aux* a) {
  if (!a) return -1;
  DeviceGuard guard(a->device);
  if (!harvest(a)) return -1;
  return (int)a->stats.size();
}

MB_EXPORT int minfft_b200_profile_entry(minfft_aux* a, int i, const char** label, long long* launches,
                                        double* total_ms, double* bytes_per_launch) {
  if (!a) return MINFFT_B200_EINVAL;
  DeviceGuard guard(a->device);
  if (!harvest(a)) return g_err;
  if (i < 0 || i >= (int)a->stats.size()) return MINFFT_B200_EINVAL;
  const auto& st = a->stats[i];
  if (label) *label = st.label.c_str();
  if (launches) *launches = st.launches;
  if (total_ms) *total_ms = st.ms;
  if (bytes_per_launch) *bytes_per_launch = st.bytes;
  return MINFFT_B200_OK;
}

// ---------------------------------------------------------------- self-check
namespace {

struct Extent {
  int64_t in_max, out_max;  // largest element index touched, in the buffer's element type
};

// Largest batch offset of an axis launch (all strides are non-negative).
void axis_batch_max(const AxisParams& ap, int64_t& oi, int64_t& oo) {
  const int64_t nb = ap.nbatch;
  const int64_t b0 = std::min<int64_t>(ap.d0, nb) - 1;
  const int64_t b1 = std::min<int64_t>(ap.d1, (nb + ap.d0 - 1) / ap.d0) - 1;
  const int64_t b2 = (nb - 1) / (ap.d0 * ap.d1);
  oi = b0 * ap.is0 + b1 * ap.is1 + b2 * ap.is2;
  oo = b0 * ap.os0 + b1 * ap.os1 + b2 * ap.os2;
}

Extent launch_extent(const Launch& ln) {
  Extent e{0, 0};
  if (ln.dctq >= 0) {  // the whole real array and the whole block array
    const int64_t reals = ln.dq.H * ln.dq.Nr * ln.dq.N, blocks = ln.dq.H * (ln.dq.Nr / 2) * ln.dq.N;
    e.in_max = (ln.in_c ? blocks : reals) - 1;
    e.out_max = (ln.in_c ? reals : blocks) - 1;
    return e;
  }
  if (!ln.is_line) {
    const AxisParams& ap = ln.ap;
    const int64_t L = ln.L;
    int64_t oi, oo;
    axis_batch_max(ap, oi, oo);
    switch (ln.combo) {
      case mb::K_CPLX:
        e.in_max = oi + (L - 1) * ap.in_n;
        e.out_max = oo + (L - 1) * ap.out_k;
        break;
      case mb::K_R2C:
      case mb::K_R2CQ:  // d0 = 4: the largest batch offset is block 3's row
        e.in_max = oi + 2 * L - 1;
        e.out_max = oo + L * ap.out_k;
        break;
      case mb::K_C2R:
      case mb::K_C2RQ:
        e.in_max = oi + L * ap.in_n;
        e.out_max = oo + 2 * L - 1;
        break;
      case mb::K_T4IN: {  // the real lines of the input (the pass's is2 is 0)
        const int64_t lines = ap.nbatch / (ap.d0 * ap.d1);
        e.in_max = (lines - 1) * ap.k_in_line + ap.kn - 1;
        e.out_max = oo + (L - 1) * ap.out_k;
        break;
      }
      case mb::K_T4OUT: {  // the real lines of the output (the pass's os2 is 0)
        const int64_t lines = ap.nbatch / (ap.d0 * ap.d1);
        e.in_max = oi + (L - 1) * ap.in_n;
        e.out_max = (lines - 1) * ap.k_out_line + ap.kn - 1;
        break;
      }
      default:
        e.in_max = oi + (2 * L - 1) * ap.in_n;
        e.out_max = oo + (2 * L - 1) * ap.out_k;
        break;
    }
    return e;
  }
  const LineParams& lp = ln.lp;
  const int64_t L = lp.L;
  if (ln.combo == mb::LK_UNIT) {
    e.in_max = e.out_max = L - 1;
    return e;
  }
  int64_t in_n = 0, out_n = 0;
  switch (ln.combo) {
    case mb::LK_DCT2_PRE:
    case mb::LK_T4_PRE:
    case mb::LK_DCT3_PACK: in_n = 2 * L - 1; out_n = L - 1; break;
    case mb::LK_C2R_PACK: in_n = L; out_n = L - 1; break;
    case mb::LK_R2C_UNPACK: in_n = L - 1; out_n = L; break;
    default: in_n = L - 1; out_n = 2 * L - 1; break;
  }
  e.in_max = (lp.outer - 1) * lp.in_so + in_n * lp.in_sn + (lp.inner - 1);
  e.out_max = (lp.outer - 1) * lp.out_so + out_n * lp.out_sn + (lp.inner - 1);
  return e;
}

}  // namespace

// Plan `op` for the given shape without touching a device and check every
// launch: element ranges inside their buffers, complex/real views of the
// user buffers, launch shapes, and no in-place use of the passes that
// cannot run in place.  Returns the number of violations (0 = plan is
// sound); a description of the first ones goes to `report`, or, for a
// sound plan, the launches' labels in launch order, one per line.
MB_EXPORT int minfft_b200_plan_selfcheck_precision(int op, int d, const int* Ns, int howmany, int alias,
                                                   int precision, char* report, int report_len, int* launches) {
  const int fam = op_family(op);
  std::string rep;
  if (fam < 0 || d < 1 || !Ns || howmany < 1) return -1;
  if (precision < MINFFT_B200_PREC_FP32 || precision > MINFFT_B200_PREC_TC_BF16) return -1;
  if (precision != MINFFT_B200_PREC_FP32 && sizeof(real) != 4) return -1;
  for (int i = 0; i < d; ++i)
    if (!is_pow2(Ns[i])) return -1;
  minfft_aux a;
  a.family = fam;
  a.dims.assign(Ns, Ns + d);
  a.total = 1;
  for (int i = 0; i < d; ++i) a.total *= Ns[i];
  a.device = -1;
  a.host_only = true;
  a.precision = precision;
  Program prog;
  if (!build_program(&a, op, howmany, alias != 0, &prog)) {
    if (report && report_len > 0) snprintf(report, report_len, "planning failed: %s", g_msg);
    return 1;
  }
  int bad = 0;
  auto fail = [&](const char* fmt, auto... args) {
    ++bad;
    char buf[256];
    snprintf(buf, sizeof(buf), fmt, args...);
    if (rep.size() < 2000) rep += std::string(buf) + "\n";
  };
  size_t cap[BUF_COUNT];
  cap[BUF_X] = size_t(io_bytes(&a, op, false)) * howmany;
  cap[BUF_Y] = size_t(io_bytes(&a, op, true)) * howmany;
  if (alias) cap[BUF_X] = cap[BUF_Y] = std::max(cap[BUF_X], cap[BUF_Y]);
  for (int b = BUF_T1; b < BUF_COUNT; ++b) cap[b] = prog.tbytes[b];
  const DeviceInfo di = device_info(-1);
  for (size_t i = 0; i < prog.launches.size(); ++i) {
    const Launch& ln = prog.launches[i];
    const Extent e = launch_extent(ln);
    const size_t ie = ln.in_c ? sizeof(cpx) : sizeof(real), oe = ln.out_c ? sizeof(cpx) : sizeof(real);
    if (size_t(e.in_max + 1) * ie > cap[ln.in_buf])
      fail("launch %zu (%s): input reaches byte %lld of buffer %d (%zu bytes)", i, ln.label.c_str(),
           (long long)((e.in_max + 1) * ie), ln.in_buf, cap[ln.in_buf]);
    if (size_t(e.out_max + 1) * oe > cap[ln.out_buf])
      fail("launch %zu (%s): output reaches byte %lld of buffer %d (%zu bytes)", i, ln.label.c_str(),
           (long long)((e.out_max + 1) * oe), ln.out_buf, cap[ln.out_buf]);
    if (ln.block < 1 || ln.block > 1024 || ln.grid < 1) fail("launch %zu: bad shape %u x %u", i, ln.grid, ln.block);
    if (!ln.is_line && ln.block > 512) fail("launch %zu: block %u above launch bounds", i, ln.block);
    if (!ln.is_line && !ln.stream && !ln.tcs && ln.dctq < 0 &&
        ln.block != unsigned(ln.ap.cpb * (ln.L / std::min(ln.radix, std::max(ln.L, 1)))))
      fail("launch %zu: block %u is not cpb x L/R", i, ln.block);
    if (ln.smem > size_t(di.max_smem)) fail("launch %zu: %zu bytes of shared memory", i, ln.smem);
    const bool alias_io = (ln.in_buf == ln.out_buf) || (alias && ((ln.in_buf == BUF_X && ln.out_buf == BUF_Y) ||
                                                                 (ln.in_buf == BUF_Y && ln.out_buf == BUF_X)));
    if (alias_io && (ln.hbm_pass || (ln.is_line && ln.combo != mb::LK_UNIT)))
      fail("launch %zu (%s): runs in place but cannot", i, ln.label.c_str());
    if (!ln.is_line && !ln.pipe && !ln.tc && !ln.stream && !ln.stream_rows && ln.dctq < 0 && ln.grid > 0 &&
        int64_t(ln.grid) * ln.ap.cpb < ln.ap.nbatch)
      fail("launch %zu: grid does not cover the batch", i);
    if (ln.stream_rows) {
      const AxisParams& ap = ln.ap;
      if (ap.colmode || ap.in_n != 1) fail("launch %zu (%s): streamed rows need contiguous rows", i, ln.label.c_str());
      if (ap.ntiles * ap.cpb < ap.nbatch || ln.grid < 1 || int64_t(ln.grid) > ap.ntiles)
        fail("launch %zu (%s): streamed row tiles do not cover the batch", i, ln.label.c_str());
      if (ap.row_pitch < ap.row_bytes || ap.row_pitch % 16 || ap.nstages < 2 || ap.nstages > 8)
        fail("launch %zu: streamed row stages", i);
      if (ln.ch_static < 4 || ap.row_bytes % ln.ch_static)
        fail("launch %zu: streamed row copy chunk %d", i, ln.ch_static);
    }
    if (ln.stream) {
      const AxisParams& ap = ln.ap;
      const int W = mb::stream_cols();
      if (ap.is0 != 1 || !ap.colmode || ln.combo != mb::K_CPLX)
        fail("launch %zu (%s): streamed pass needs adjacent unit-stride columns", i, ln.label.c_str());
      if (ap.d0 * ap.d1 * ln.st_d2 != ap.nbatch || ap.gpb * W < ap.d0 || ap.ntiles != ap.gpb * ap.d1 * ln.st_d2)
        fail("launch %zu (%s): streamed tiles do not cover the batch", i, ln.label.c_str());
      if (ln.block != unsigned(W * (ln.L / ln.radix)) || ap.cpb < 2 || ap.cpb > 8)
        fail("launch %zu: streamed shape %u threads, %d stages", i, ln.block, ap.cpb);
      if (size_t(ap.stage_bytes) < size_t(W) * (ln.L + 1) * sizeof(cpx) || ap.stage_bytes % 128)
        fail("launch %zu: stage of %d bytes", i, ap.stage_bytes);
      if (ln.grid < 1 || int64_t(ln.grid) > ap.ntiles) fail("launch %zu: persistent grid %u", i, ln.grid);
    }
    if (ln.pipe) {
      const AxisParams& ap = ln.ap;
      if (ap.colmode) {
        if (ap.nbatch % ap.d0 != 0) fail("launch %zu: column tiles would straddle d0 blocks", i);
        if ((ap.nbatch / ap.d0) * ap.gpb != ap.ntiles || ap.gpb * ap.cpb < ap.d0)
          fail("launch %zu: column tiles do not cover the batch", i);
      } else {
        if (ap.ntiles * ap.cpb < ap.nbatch) fail("launch %zu: row tiles do not cover the batch", i);
        if (ap.in_n != 1 && ln.combo != mb::K_R2C) fail("launch %zu: row-mode copy needs contiguous rows", i);
      }
      if (ln.grid < 1 || int64_t(ln.grid) > ap.ntiles) fail("launch %zu: persistent grid %u", i, ln.grid);
      const int esz = mb::pipe_raw_size(ln.combo);
      if (ln.ch_static < esz && ln.ch_static < 16 && esz <= 16 && ln.ch_static % 4 != 0)
        fail("launch %zu: copy chunk %d", i, ln.ch_static);
      if (size_t(ap.stage_bytes) < size_t(ap.cpb) * mb::pipe_raw_elems(ln.combo, ln.L) * esz ||
          size_t(ap.stage_bytes) <
              size_t(ap.cpb) * mb::tile_pitch(ln.L, std::min(ln.radix, ln.L), ap.cpb, ap.colmode) * sizeof(cpx))
        fail("launch %zu: stage of %d bytes too small", i, ap.stage_bytes);
    }
    if (!ln.is_line && (ln.combo == mb::K_R2CQ || ln.combo == mb::K_C2RQ) &&
        (ln.ap.cpb != 4 || ln.ap.d0 != 4 || ln.ap.nbatch % 4 != 0 || ln.ap.colmode || ln.pipe))
      fail("launch %zu (%s): split-column pass needs four rows j + Q*m per CTA", i, ln.label.c_str());
    if (ln.tc) {
      if (ln.L != mb::kTcLength || ln.combo != mb::K_CPLX)
        fail("launch %zu (%s): tensor-core pass on an unsupported axis", i, ln.label.c_str());
      if (ln.tcs) {
        const AxisParams& ap = ln.ap;
        const int W = mb::kTcStreamTile;
        if ((ln.tcs == 1) != (ap.colmode != 0) || (ap.colmode ? ap.is0 != 1 : ap.in_n != 1))
          fail("launch %zu (%s): streamed tensor-core tile layout", i, ln.label.c_str());
        if (ap.d0 * ap.d1 * ln.st_d2 != ap.nbatch || ap.gpb * W < ap.d0 || ap.ntiles != ap.gpb * ap.d1 * ln.st_d2)
          fail("launch %zu (%s): streamed tensor-core tiles do not cover the batch", i, ln.label.c_str());
        if (ln.block != unsigned(mb::kTcStreamThreads) || ap.cpb < 2 || ap.cpb > 8 || ln.grid < 1 ||
            int64_t(ln.grid) > ap.ntiles)
          fail("launch %zu: streamed tensor-core shape", i);
      } else {
        if (ln.ap.cpb != 8 && ln.ap.cpb != 16) fail("launch %zu: tensor-core tile of %d transforms", i, ln.ap.cpb);
        if (ln.ap.ntiles * ln.ap.cpb < ln.ap.nbatch || ln.grid < 1 || int64_t(ln.grid) > ln.ap.ntiles)
          fail("launch %zu: tensor-core tiles do not cover the batch", i);
      }
    }
  }
  if (launches) *launches = (int)prog.launches.size();
  if (bad == 0)
    for (const Launch& ln : prog.launches) rep += ln.label + "\n";
  if (report && report_len > 0) snprintf(report, report_len, "%s", rep.c_str());
  return bad;
}

MB_EXPORT int minfft_b200_plan_selfcheck(int op, int d, const int* Ns, int howmany, int alias, char* report,
                                         int report_len, int* launches) {
  return minfft_b200_plan_selfcheck_precision(op, d, Ns, howmany, alias, MINFFT_B200_PREC_FP32, report, report_len,
                                              launches);
}

// ------------------------------------------------------------- autotuner
namespace {

// Mean milliseconds of `reps` back-to-back runs of one launch (after one
// untimed run), or a negative value on error.
float time_launch(minfft_aux* a, const Launch& ln, void* const* bufs, int reps) {
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return -1;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return -1;
  }
  float ms = -1;
  if (launch_one(a, ln, bufs) && cudaEventRecord(e0, a->stream) == cudaSuccess) {
    bool ok = true;
    for (int r = 0; r < reps && ok; ++r) ok = launch_one(a, ln, bufs);
    if (ok && cudaEventRecord(e1, a->stream) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
        cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
      ms /= float(reps);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms;
}

}  // namespace

// Time every candidate configuration (kernel form x transforms per CTA) of
// each axis launch of transform `op` on `howmany` arrays, on scratch
// buffers, and record the fastest in the process-wide tuning table; the
// plan's launch lists are then rebuilt with the winners.  Returns 0 or an
// error code.
MB_EXPORT int minfft_b200_autotune(minfft_aux* a, int op, int howmany, int reps) {
  if (!a || op_family(op) != a->family || howmany < 1) {
    set_error(MINFFT_B200_EINVAL, "bad autotune arguments");
    return MINFFT_B200_EINVAL;
  }
  if (reps < 1) reps = 5;
  DeviceGuard guard(a->device);
  if (!harvest(a)) return g_err;
  Program* p0 = get_program(a, op, howmany, false);
  if (!p0) return g_err ? g_err : MINFFT_B200_ECUDA;
  std::vector<TuneKey> keys;
  for (const Launch& ln : p0->launches)
    if (!ln.is_line && !ln.tc && ln.dctq < 0) keys.push_back(ln.key);
  const size_t in_b = size_t(io_bytes(a, op, false)) * howmany, out_b = size_t(io_bytes(a, op, true)) * howmany;
  void *x = nullptr, *y = nullptr;
  if (!cuda_ok(cudaMalloc(&x, in_b), "cudaMalloc(autotune)")) return g_err;
  if (!cuda_ok(cudaMalloc(&y, out_b), "cudaMalloc(autotune)")) {
    cudaFree(x);
    return g_err;
  }
  cudaMemsetAsync(x, 0, in_b, a->stream);
  cudaMemsetAsync(y, 0, out_b, a->stream);
  DeviceInfo di = device_info(a->device);
  std::map<TuneKey, TuneVal> force, best;
  t_force = &force;
  int rc = MINFFT_B200_OK;
  for (const TuneKey& key : keys) {
    if (best.count(key)) continue;
    Planner probe{a, nullptr, di.max_smem, di.sms};
    float best_ms = 1e30f;
    TuneVal best_v{0, 0, 16};
    // the launch's own parameters (for the streamed form's applicability)
    const Launch* base = nullptr;
    for (const Launch& ln : p0->launches)
      if (!ln.is_line && !ln.tc && ln.dctq < 0 && !(ln.key < key) && !(key < ln.key)) base = &ln;
    for (int cand = 0; cand < 8; ++cand) {
      const int pipe = cand < 4 ? (cand & 1) : (cand < 6 ? 2 : cand - 3), radix = (cand < 6 && (cand & 2)) ? 8 : 16;
      if (radix == 8 && key.L <= 8) continue;
      const int top = pipe == 2 ? 4 : probe.max_threads_cpb(key.L, radix);
      for (int cpb = pipe == 2 ? 2 : 1; cpb <= top; cpb = pipe == 2 ? cpb + 1 : 2 * cpb) {
        if (Planner::four_rows(key.combo) && ((pipe != 3 && pipe != 4 && pipe) || cpb != 4)) continue;
        bool fits;
        if (pipe == 3 || pipe == 4)
          fits = base && probe.stream_rows_fits(key.combo, key.L, base->ap, cpb, pipe - 1);
        else if (pipe == 2)
          fits = base && probe.stream_fits(key.combo, key.L, base->ap.nbatch, base->ap, radix, cpb);
        else if (pipe == 1)
          fits = probe.pipe_fits(key.combo, key.L, cpb, key.colmode, radix);
        else
          fits = probe.plain_fits(key.combo, key.L, cpb, key.staged ? mb::F_STAGE_ROWS : 0, key.colmode, radix);
        if (!fits) continue;
        force[key] = TuneVal{pipe, cpb, radix};
        Program P;
        if (!build_program(a, op, howmany, false, &P)) continue;
        bool bufs_ok = true;
        for (int b = BUF_T1; b < BUF_COUNT; ++b) bufs_ok &= ensure_buffer(a, b, P.tbytes[b]);
        if (!bufs_ok) {
          rc = g_err;
          break;
        }
        void* bufs[BUF_COUNT] = {x, y, a->bufs[BUF_T1], a->bufs[BUF_T2], a->bufs[BUF_T3], a->bufs[BUF_T4]};
        for (const Launch& ln : P.launches) {
          if (ln.is_line || ln.key < key || key < ln.key) continue;
          const float ms = time_launch(a, ln, bufs, reps);
          if (ms > 0 && ms < best_ms) {
            best_ms = ms;
            best_v = TuneVal{pipe, cpb, radix};
          }
          break;
        }
      }
    }
    force.erase(key);
    if (best_ms < 1e29f) best[key] = best_v;
  }
  t_force = nullptr;
  cudaStreamSynchronize(a->stream);
  cudaGetLastError();
  cudaFree(x);
  cudaFree(y);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (auto& kv : best) g_tune[kv.first] = kv.second;
  }
  a->programs.clear();
  return rc;
}

// Save / load / clear the process-wide tuning table (text, one entry per line).
MB_EXPORT int minfft_b200_tune_save(const char* path) {
  if (!path) return MINFFT_B200_EINVAL;
  FILE* f = fopen(path, "w");
  if (!f) {
    set_error(MINFFT_B200_EINVAL, "cannot write %s", path);
    return MINFFT_B200_EINVAL;
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  fprintf(f, "# minfft_b200 tuning table (%s): combo L colmode hbm staged nbatch d0 in_n out_k pipe cpb radix\n",
          sizeof(real) == 8 ? "double" : "single");
  for (auto& kv : g_tune) {
    const TuneKey& k = kv.first;
    fprintf(f, "%d %d %d %d %d %lld %lld %lld %lld %d %d %d\n", k.combo, k.L, k.colmode, k.hbm, k.staged,
            (long long)k.nbatch, (long long)k.d0, (long long)k.in_n, (long long)k.out_k, kv.second.pipe,
            kv.second.cpb, kv.second.radix);
  }
  fclose(f);
  return MINFFT_B200_OK;
}

MB_EXPORT int minfft_b200_tune_load(const char* path) {
  if (!path) return MINFFT_B200_EINVAL;
  FILE* f = fopen(path, "r");
  if (!f) {
    set_error(MINFFT_B200_EINVAL, "cannot read %s", path);
    return MINFFT_B200_EINVAL;
  }
  char line[512];
  std::lock_guard<std::mutex> lk(g_tune_mu);
  while (fgets(line, sizeof(line), f)) {
    if (line[0] == '#') continue;
    TuneKey k{};
    TuneVal v{};
    long long nb, d0, in_n, out_k;
    if (sscanf(line, "%d %d %d %d %d %lld %lld %lld %lld %d %d %d", &k.combo, &k.L, &k.colmode, &k.hbm, &k.staged,
               &nb, &d0, &in_n, &out_k, &v.pipe, &v.cpb, &v.radix) == 12 &&
        (v.radix == 8 || v.radix == 16) && v.pipe >= 0 && v.pipe <= 4) {
      k.nbatch = nb;
      k.d0 = d0;
      k.in_n = in_n;
      k.out_k = out_k;
      g_tune[k] = v;
    }
  }
  fclose(f);
  return MINFFT_B200_OK;
}

MB_EXPORT int minfft_b200_tune_clear(void) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune.clear();
  return MINFFT_B200_OK;
}

MB_EXPORT int minfft_b200_tune_size(void) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  return (int)g_tune.size();
}

// Launch configuration used where the tuning table has no entry: pipe = 1
// persistent pipelined kernels, 0 one tile per CTA, -1 the planner's choice;
// cpb > 0 sets transforms per CTA (reduced until it fits), 0 the heuristic;
// radix 8 or 16 registers per thread (16 where 8 does not exist).  Plans
// built afterwards use it.
MB_EXPORT int minfft_b200_tune_set_default(int pipe, int cpb, int radix) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_default_override = TuneVal{pipe < 0 ? -1 : std::min(pipe, 4), cpb < 0 ? 0 : cpb, radix == 8 ? 8 : 16};
  return MINFFT_B200_OK;
}

// ------------------------------------------------------------ test hooks
MB_EXPORT int minfft_b200_test_fail_device_alloc(long long k) {
  if (k < 0) {
    set_error(MINFFT_B200_EINVAL, "allocation index must be >= 0");
    return MINFFT_B200_EINVAL;
  }
  g_fail_at.store(0);
  g_alloc_count.store(0);
  g_fail_at.store(k);
  return MINFFT_B200_OK;
}

MB_EXPORT long long minfft_b200_test_device_alloc_count(void) { return g_alloc_count.load(); }

MB_EXPORT int minfft_b200_test_tc_withhold(long long polls) {
  if (polls < 0) {
    set_error(MINFFT_B200_EINVAL, "poll count must be >= 0");
    return MINFFT_B200_EINVAL;
  }
  g_tc_withhold.store(polls);
  return MINFFT_B200_OK;
}
