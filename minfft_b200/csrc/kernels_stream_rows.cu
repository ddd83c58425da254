// Instantiations of the streamed row pass (stream_pass.cuh) for every row
// kind: in-CTA lengths 2^6 .. 2^12, radix 16.
#include "kernel_registry.h"
#include "stream_pass.cuh"

namespace mb {

namespace {
template <class Ld, class St>
const void* rows_kernel(int log2L) {
  static const void* const table[13] = {nullptr,
                                        nullptr,
                                        nullptr,
                                        nullptr,
                                        nullptr,
                                        nullptr,
                                        (const void*)stream_rows_kernel<64, 16, Ld, St>,
                                        (const void*)stream_rows_kernel<128, 16, Ld, St>,
                                        (const void*)stream_rows_kernel<256, 16, Ld, St>,
                                        (const void*)stream_rows_kernel<512, 16, Ld, St>,
                                        (const void*)stream_rows_kernel<1024, 16, Ld, St>,
                                        (const void*)stream_rows_kernel<2048, 16, Ld, St>,
                                        (const void*)stream_rows_kernel<4096, 16, Ld, St>};
  return (log2L >= 0 && log2L <= 12) ? table[log2L] : nullptr;
}
}  // namespace

const void* stream_rows_kernel_fn(int combo, int log2L) {
  switch (combo) {
    case K_CPLX: return rows_kernel<LoadCplx, StoreCplx>(log2L);
    case K_R2C: return rows_kernel<LoadR2C, StoreR2C>(log2L);
    case K_C2R: return rows_kernel<LoadC2R, StoreC2R>(log2L);
    case K_DCT2: return rows_kernel<LoadDCT2, StoreDCT2>(log2L);
    case K_DCT3: return rows_kernel<LoadDCT3, StoreDCT3>(log2L);
    case K_T4: return rows_kernel<LoadT4, StoreT4>(log2L);
    case K_R2CQ: return log2L <= 11 ? rows_kernel<LoadR2C, StoreR2CQ>(log2L) : nullptr;
    case K_C2RQ: return log2L <= 11 ? rows_kernel<LoadC2RQ, StoreC2R>(log2L) : nullptr;
    default: return nullptr;
  }
}

}  // namespace mb
