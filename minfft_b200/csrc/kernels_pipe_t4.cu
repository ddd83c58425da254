// Instantiations of the pipelined axis-pass kernel for PT4 / StoreT4, one per
// in-CTA DFT length 2^1 .. 2^13 (index 0 is unused).
#include "pipe_pass.cuh"

namespace mb {

const void* pipe_kernel_t4(int log2L) {
  static const void* const table[] = {
      nullptr,                                           (const void*)axis_pipe_kernel<2, PT4, StoreT4>,
      (const void*)axis_pipe_kernel<4, PT4, StoreT4>,    (const void*)axis_pipe_kernel<8, PT4, StoreT4>,
      (const void*)axis_pipe_kernel<16, PT4, StoreT4>,   (const void*)axis_pipe_kernel<32, PT4, StoreT4>,
      (const void*)axis_pipe_kernel<64, PT4, StoreT4>,   (const void*)axis_pipe_kernel<128, PT4, StoreT4>,
      (const void*)axis_pipe_kernel<256, PT4, StoreT4>,  (const void*)axis_pipe_kernel<512, PT4, StoreT4>,
      (const void*)axis_pipe_kernel<1024, PT4, StoreT4>, (const void*)axis_pipe_kernel<2048, PT4, StoreT4>,
      (const void*)axis_pipe_kernel<4096, PT4, StoreT4>, (const void*)axis_pipe_kernel<8192, PT4, StoreT4>,
  };
  return (log2L >= 1 && log2L <= 13) ? table[log2L] : nullptr;
}

}  // namespace mb
