// Instantiations of the streamed (persistent, TMA-fed) complex column pass:
// in-CTA lengths 2^4 .. 2^9 (a tile of W columns x L elements is at most
// 64 KiB), radix 16 and, where the CTA stays within 512 threads, radix 8.
#include "kernel_registry.h"
#include "stream_pass.cuh"

namespace mb {

const void* stream_kernel(int log2L, int R) {
  static const void* const r16[10] = {nullptr,
                                      nullptr,
                                      nullptr,
                                      nullptr,
                                      (const void*)stream_pass_kernel<16, 16>,
                                      (const void*)stream_pass_kernel<32, 16>,
                                      (const void*)stream_pass_kernel<64, 16>,
                                      (const void*)stream_pass_kernel<128, 16>,
                                      (const void*)stream_pass_kernel<256, 16>,
                                      (const void*)stream_pass_kernel<512, 16>};
  static const void* const r8[10] = {nullptr,
                                     nullptr,
                                     nullptr,
                                     nullptr,
                                     (const void*)stream_pass_kernel<16, 8>,
                                     (const void*)stream_pass_kernel<32, 8>,
                                     (const void*)stream_pass_kernel<64, 8>,
                                     (const void*)stream_pass_kernel<128, 8>,
                                     (const void*)stream_pass_kernel<256, 8>,
                                     sizeof(cpx) == 16 ? (const void*)stream_pass_kernel<512, 8> : nullptr};
  if (log2L < 4 || log2L > 9) return nullptr;
  return R == 8 ? r8[log2L] : r16[log2L];
}

}  // namespace mb
