// f64 instances of the fixed-length power-of-two kernels.
#include "pow2_fixed_launch.cuh"

namespace b2f {

cudaError_t launch_pow2_fixed_f64(int lg, bool colmajor, const LinesParams& prm, unsigned grid,
                                  unsigned threads, size_t smem, cudaStream_t st) {
  return colmajor ? fx_launch_wide<double, true>(lg, prm, grid, threads, smem, st)
                  : fx_launch_wide<double, false>(lg, prm, grid, threads, smem, st);
}

cudaError_t launch_real_fixed_f64(int lg, bool r2c, const RealParams& prm, unsigned grid,
                                  unsigned threads, size_t smem, cudaStream_t st) {
  return r2c ? fx_real_any<double, true>(lg, prm, grid, threads, smem, st)
             : fx_real_any<double, false>(lg, prm, grid, threads, smem, st);
}

}  // namespace b2f
