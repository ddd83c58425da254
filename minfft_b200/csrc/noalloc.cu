// minfft_b200_dft_noalloc: a complex DFT that allocates no memory.
//
// Who needs it.  Some callers cannot call cudaMalloc (or have us call it on
// their behalf): code whose device memory is entirely owned by another
// allocator -- a framework's caching pool that has reserved the GPU's memory,
// or an embedded runtime with a fixed memory budget -- and latency-bound loops
// where an allocation (and the device-wide synchronisation that cudaFree
// implies) is not acceptable.  The planned path (minfft_mkaux_dft_1d +
// minfft_dft) allocates its root tables and, for lengths beyond one thread
// block, the scratch array between its passes; this entry point needs
// neither.
//
// How.  It runs the same two-pass Stockham FFT over HBM that the planner
// uses for long lengths (the existing axis-pass kernel, twice), but the
// intermediate array and the passes' root tables live in the file-scope
// static device arrays below, of a fixed maximum size.  Every GPU that loads
// this library holds them until the process exits: 4 MiB of scratch in the
// double build and 2 MiB in the single build, plus 32 KiB / 16 KiB of roots.
//
// Sharing.  All calls on a device share the arrays, which keep the last
// call's contents.  Nothing has to start at zero: each call first rewrites
// the root tables, and its first pass writes every scratch element its second
// pass reads.  Calls that overlap on the GPU (on different streams, or from
// different threads without ordering) race on the arrays; a caller must order
// them, e.g. by using one stream.
//
// Set-up.  The first call on each device looks up the arrays' device
// addresses (cudaGetSymbolAddress, once per device, with that device
// current); issue that first call before any stream capture.  The lookup is
// tied to the device's context: after cudaDeviceReset the module is loaded
// again (its arrays may move), so the next call on that device, which sees a
// new context, repeats the set-up.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "axis_pass.cuh"
#include "kernel_registry.h"
#include "minfft_b200.h"

#define MB_EXPORT extern "C" __attribute__((visibility("default")))

namespace mb {
void set_last_error(int code, const char* msg);
}

namespace {

using mb::cpx;

constexpr int kMaxLog2 = 18;                   // longest transform: 2^18 points
constexpr int kMinLog2 = 2;                    // shortest: 4 points (two passes of >= 2)
constexpr int kRootSlot = 1 << ((kMaxLog2 + 1) / 2);  // 512 roots per table

// The scratch between the two passes, and the four root tables of a call:
// in-CTA roots of pass 1 and pass 2, coarse and fine roots of length n.
static __device__ __align__(256) cpx g_noalloc_scratch[1 << kMaxLog2];
static __device__ __align__(256) cpx g_noalloc_roots[4 * kRootSlot];

struct DeviceArrays {
  cpx* scratch = nullptr;
  cpx* roots = nullptr;
  unsigned long long ctx_id = 0;  // the context the addresses belong to
};

std::mutex g_mu;
DeviceArrays g_arrays[128];

// Unique id of the calling thread's current context (the device's primary
// context once the runtime has set it up); a reset device gets a new one.
// The driver functions come through the runtime, so the library does not
// link libcuda itself.
bool current_context_id(unsigned long long* id) {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    return cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
                   q == cudaDriverEntryPointSuccess
               ? reinterpret_cast<GetCurrent>(f)
               : nullptr;
  }();
  static GetId get_id = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    return cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
                   q == cudaDriverEntryPointSuccess
               ? reinterpret_cast<GetId>(f)
               : nullptr;
  }();
  CUcontext ctx = nullptr;
  return get_current && get_id && get_current(&ctx) == CUDA_SUCCESS && ctx && get_id(ctx, id) == CUDA_SUCCESS;
}

// Device addresses of the static arrays on `dev`, looked up once per device
// (again after the device's context changed, e.g. after cudaDeviceReset).
// The caller has already made a runtime call on `dev` (the pointer checks),
// so its primary context is current.
bool device_arrays(int dev, DeviceArrays* out) {
  if (dev < 0 || dev >= 128) return false;
  unsigned long long id = 0;
  if (!current_context_id(&id)) return false;
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceArrays& a = g_arrays[dev];
  if (!a.scratch || a.ctx_id != id) {
    cpx* s = nullptr;
    cpx* r = nullptr;
    if (cudaGetSymbolAddress((void**)&s, g_noalloc_scratch) != cudaSuccess) return false;
    if (cudaGetSymbolAddress((void**)&r, g_noalloc_roots) != cudaSuccess) return false;
    a.scratch = s;
    a.roots = r;
    a.ctx_id = id;
  }
  *out = a;
  return true;
}

// w_N^m = exp(-2*pi*i*m/N) for the four tables of a call, evaluated in double.
__global__ void fill_roots(int n, int r1, int r2, int lobits) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 4 * kRootSlot) return;
  const int table = t / kRootSlot, m = t % kRootSlot;
  int N = 0, e = 0, count = 0;
  switch (table) {
    case 0: N = r1; e = m; count = r1; break;
    case 1: N = r2; e = m; count = r2; break;
    case 2: N = n; e = m << lobits; count = n >> lobits; break;
    default: N = n; e = m; count = 1 << lobits; break;
  }
  if (m >= count) return;
  double s, c;
  sincospi(-2.0 * double(e) / double(N), &s, &c);
  g_noalloc_roots[t] = mb::cmk(mb::real(c), mb::real(s));
}

// transforms per CTA: 128-byte runs of adjacent columns where possible
int pick_cpb(int L) {
  const int tpt = L / std::min(L, 16);
  int cpb = std::max(1, 256 / tpt);
  const int want = int(128 / sizeof(cpx));
  if (cpb < want) cpb = std::max(cpb, std::min(want, std::max(1, 512 / tpt)));
  // stay within the default 48 KiB of dynamic shared memory
  while (cpb > 1 && mb::axis_pass_smem(L, std::min(L, 16), cpb, 1) > 48 * 1024) cpb /= 2;
  return cpb;
}

int fail(int code, const char* msg) {
  mb::set_last_error(code, msg);
  return code;
}

}  // namespace

MB_EXPORT int minfft_b200_dft_noalloc(const void* x, void* y, int n, int inverse, void* stream) {
  if (n < (1 << kMinLog2) || n > (1 << kMaxLog2) || (n & (n - 1)) != 0)
    return fail(MINFFT_B200_EINVAL, "minfft_b200_dft_noalloc: length must be a power of two in [4, 262144]");
  if (!x || !y) return fail(MINFFT_B200_EINVAL, "minfft_b200_dft_noalloc: NULL data pointer");
  if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) % sizeof(cpx) != 0)
    return fail(MINFFT_B200_EINVAL, "minfft_b200_dft_noalloc: complex data must be aligned to its size");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(MINFFT_B200_ECUDA, "minfft_b200_dft_noalloc: no device");
  for (const void* p : {x, static_cast<const void*>(y)}) {
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess ||
        (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)) {
      cudaGetLastError();
      return fail(MINFFT_B200_EINVAL, "minfft_b200_dft_noalloc: x and y must be device memory");
    }
    if (attr.type == cudaMemoryTypeDevice && attr.device != dev)
      return fail(MINFFT_B200_EINVAL, "minfft_b200_dft_noalloc: x and y must be on the current device");
  }
  DeviceArrays arr;
  if (!device_arrays(dev, &arr))
    return fail(MINFFT_B200_ECUDA, "minfft_b200_dft_noalloc: cudaGetSymbolAddress failed");

  int b = 0;
  while ((1 << b) < n) ++b;
  const int b1 = (b + 1) / 2, b2 = b - b1;  // both in [1, 9]
  const int r1 = 1 << b1, r2 = 1 << b2;
  const int lobits = (b + 1) / 2;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  fill_roots<<<(4 * kRootSlot + 255) / 256, 256, 0, st>>>(n, r1, r2, lobits);
  if (cudaGetLastError() != cudaSuccess) return fail(MINFFT_B200_ECUDA, "minfft_b200_dft_noalloc: launch failed");

  // pass 1: n/r1 sub-DFTs of length r1 (stride n/r1), rows of r1 into scratch
  mb::AxisParams p1;
  memset(&p1, 0, sizeof(p1));
  p1.in = x;
  p1.out = arr.scratch;
  p1.nbatch = n / r1;
  p1.d0 = 1;
  p1.d1 = n / r1;
  p1.is0 = 1;
  p1.is1 = 1;
  p1.is2 = n;
  p1.in_n = n / r1;
  p1.os0 = 1;
  p1.os1 = r1;
  p1.os2 = n;
  p1.out_k = 1;
  p1.tw = arr.roots;
  p1.st_ns = 1;
  p1.st_div = 1;
  p1.colmode = 1;
  p1.cpb = pick_cpb(r1);
  p1.lp = mb::tile_pitch(r1, 16, p1.cpb, 1);
  p1.flags = mb::F_STAGE_ROWS | (inverse ? mb::F_CONJ_IN : 0);

  // pass 2: n/r2 sub-DFTs of length r2 pre-multiplied by w_n^((j mod r1) r)
  mb::AxisParams p2;
  memset(&p2, 0, sizeof(p2));
  p2.in = arr.scratch;
  p2.out = y;
  p2.nbatch = n / r2;
  p2.d0 = r1;
  p2.d1 = 1;
  p2.is0 = 1;
  p2.is1 = r1;
  p2.is2 = n;
  p2.in_n = n / r2;
  p2.os0 = 1;
  p2.os1 = n;
  p2.os2 = n;
  p2.out_k = r1;
  p2.tw = arr.roots + kRootSlot;
  p2.st_hi = arr.roots + 2 * kRootSlot;
  p2.st_lo = arr.roots + 3 * kRootSlot;
  p2.st_ns = r1;
  p2.st_div = 1;
  p2.st_shift = 0;
  p2.st_lobits = lobits;
  p2.colmode = 1;
  p2.cpb = pick_cpb(r2);
  p2.lp = mb::tile_pitch(r2, 16, p2.cpb, 1);
  p2.flags = inverse ? mb::F_CONJ_OUT : 0;

  for (const mb::AxisParams* p : {&p1, &p2}) {
    const int L = (p == &p1) ? r1 : r2;
    const void* fn = mb::axis_kernel(mb::K_CPLX, (p == &p1) ? b1 : b2);
    const int R = L < 16 ? L : 16;
    const unsigned block = unsigned(p->cpb * (L / R));
    const unsigned grid = unsigned((p->nbatch + p->cpb - 1) / p->cpb);
    void* args[1] = {const_cast<mb::AxisParams*>(p)};
    if (cudaLaunchKernel(fn, dim3(grid), dim3(block), args, mb::axis_pass_smem(L, 16, p->cpb, 1), st) !=
        cudaSuccess)
      return fail(MINFFT_B200_ECUDA, "minfft_b200_dft_noalloc: launch failed");
  }
  return MINFFT_B200_OK;
}
