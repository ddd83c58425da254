// Instantiations of the axis-pass kernel for the LoadCplx / StoreCplx combination,
// one per in-CTA DFT length 2^0 .. 2^13.
#include "axis_pass.cuh"

namespace mb {

const void* axis_kernel_cplx(int log2L) {
  static const void* const table[] = {
      (const void*)axis_pass_kernel<1, LoadCplx, StoreCplx>,    (const void*)axis_pass_kernel<2, LoadCplx, StoreCplx>,
      (const void*)axis_pass_kernel<4, LoadCplx, StoreCplx>,    (const void*)axis_pass_kernel<8, LoadCplx, StoreCplx>,
      (const void*)axis_pass_kernel<16, LoadCplx, StoreCplx>,   (const void*)axis_pass_kernel<32, LoadCplx, StoreCplx>,
      (const void*)axis_pass_kernel<64, LoadCplx, StoreCplx>,   (const void*)axis_pass_kernel<128, LoadCplx, StoreCplx>,
      (const void*)axis_pass_kernel<256, LoadCplx, StoreCplx>,  (const void*)axis_pass_kernel<512, LoadCplx, StoreCplx>,
      (const void*)axis_pass_kernel<1024, LoadCplx, StoreCplx>, (const void*)axis_pass_kernel<2048, LoadCplx, StoreCplx>,
      (const void*)axis_pass_kernel<4096, LoadCplx, StoreCplx>, (const void*)axis_pass_kernel<8192, LoadCplx, StoreCplx>,
  };
  return (log2L >= 0 && log2L <= 13) ? table[log2L] : nullptr;
}

}  // namespace mb
