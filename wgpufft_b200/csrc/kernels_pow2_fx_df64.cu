// df64 instances of the fixed-length power-of-two kernels.
#include "pow2_fixed_launch.cuh"

namespace b2f {

cudaError_t launch_pow2_fixed_df64(int lg, bool colmajor, const LinesParams& prm, unsigned grid,
                                   unsigned threads, size_t smem, cudaStream_t st) {
  return colmajor ? fx_launch_wide<df, true>(lg, prm, grid, threads, smem, st)
                  : fx_launch_wide<df, false>(lg, prm, grid, threads, smem, st);
}

}  // namespace b2f
