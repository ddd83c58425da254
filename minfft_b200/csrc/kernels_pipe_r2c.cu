// Instantiations of the pipelined axis-pass kernel for PR2C / StoreR2C, one per
// in-CTA DFT length 2^1 .. 2^13 (index 0 is unused).
#include "pipe_pass.cuh"

namespace mb {

const void* pipe_kernel_r2c(int log2L) {
  static const void* const table[] = {
      nullptr,                                           (const void*)axis_pipe_kernel<2, PR2C, StoreR2C>,
      (const void*)axis_pipe_kernel<4, PR2C, StoreR2C>,    (const void*)axis_pipe_kernel<8, PR2C, StoreR2C>,
      (const void*)axis_pipe_kernel<16, PR2C, StoreR2C>,   (const void*)axis_pipe_kernel<32, PR2C, StoreR2C>,
      (const void*)axis_pipe_kernel<64, PR2C, StoreR2C>,   (const void*)axis_pipe_kernel<128, PR2C, StoreR2C>,
      (const void*)axis_pipe_kernel<256, PR2C, StoreR2C>,  (const void*)axis_pipe_kernel<512, PR2C, StoreR2C>,
      (const void*)axis_pipe_kernel<1024, PR2C, StoreR2C>, (const void*)axis_pipe_kernel<2048, PR2C, StoreR2C>,
      (const void*)axis_pipe_kernel<4096, PR2C, StoreR2C>, (const void*)axis_pipe_kernel<8192, PR2C, StoreR2C>,
  };
  return (log2L >= 1 && log2L <= 13) ? table[log2L] : nullptr;
}

}  // namespace mb
