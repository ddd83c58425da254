// Instantiations of the pipelined axis-pass kernel for PDCT3 / StoreDCT3:
// in-CTA DFT lengths 2^0 .. 2^13, radix 8 and 16 per thread (lengths below 16
// use their own length as the radix; configurations above 512 threads per
// transform do not exist).
#include "pipe_pass.cuh"

namespace mb {

const void* pipe_kernel_dct3(int log2L, int radix16) {
  static const void* const table[14][2] = {
      {nullptr, nullptr},
      {(const void*)axis_pipe_kernel<2, 2, PDCT3, StoreDCT3>, (const void*)axis_pipe_kernel<2, 2, PDCT3, StoreDCT3>},
      {(const void*)axis_pipe_kernel<4, 4, PDCT3, StoreDCT3>, (const void*)axis_pipe_kernel<4, 4, PDCT3, StoreDCT3>},
      {(const void*)axis_pipe_kernel<8, 8, PDCT3, StoreDCT3>, (const void*)axis_pipe_kernel<8, 8, PDCT3, StoreDCT3>},
      {(const void*)axis_pipe_kernel<16, 8, PDCT3, StoreDCT3>, (const void*)axis_pipe_kernel<16, 16, PDCT3, StoreDCT3>},
      {(const void*)axis_pipe_kernel<32, 8, PDCT3, StoreDCT3>, (const void*)axis_pipe_kernel<32, 16, PDCT3, StoreDCT3>},
      {(const void*)axis_pipe_kernel<64, 8, PDCT3, StoreDCT3>, (const void*)axis_pipe_kernel<64, 16, PDCT3, StoreDCT3>},
      {(const void*)axis_pipe_kernel<128, 8, PDCT3, StoreDCT3>, (const void*)axis_pipe_kernel<128, 16, PDCT3, StoreDCT3>},
      {(const void*)axis_pipe_kernel<256, 8, PDCT3, StoreDCT3>, (const void*)axis_pipe_kernel<256, 16, PDCT3, StoreDCT3>},
      {(const void*)axis_pipe_kernel<512, 8, PDCT3, StoreDCT3>, (const void*)axis_pipe_kernel<512, 16, PDCT3, StoreDCT3>},
      {(const void*)axis_pipe_kernel<1024, 8, PDCT3, StoreDCT3>, (const void*)axis_pipe_kernel<1024, 16, PDCT3, StoreDCT3>},
      {(const void*)axis_pipe_kernel<2048, 8, PDCT3, StoreDCT3>, (const void*)axis_pipe_kernel<2048, 16, PDCT3, StoreDCT3>},
      {(const void*)axis_pipe_kernel<4096, 8, PDCT3, StoreDCT3>, (const void*)axis_pipe_kernel<4096, 16, PDCT3, StoreDCT3>},
      {nullptr, (const void*)axis_pipe_kernel<8192, 16, PDCT3, StoreDCT3>},
  };
  return (log2L >= 0 && log2L <= 13) ? table[log2L][radix16 ? 1 : 0] : nullptr;
}

}  // namespace mb
