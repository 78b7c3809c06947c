// Power-of-two register kernels with the line length fixed at compile time
// (regfft_fixed.cuh).  f32: contiguous lines of 16..8192 points (16 values a
// thread) and column tiles of 16..512 (16 values) and 1024..8192 points
// (32 values); the f64 and df64 instances sit in kernels_pow2_fx_f64.cu and
// kernels_pow2_fx_df64.cu (one translation unit each, compiled in parallel).
#include "pow2_fixed_launch.cuh"

namespace b2f {

// The compile-time kernel for (E, layout, N), or cudaErrorInvalidValue when
// there is none (the caller uses the generic kernel).
cudaError_t launch_pow2_fixed(Prec prec, int E, bool colmajor, const LinesParams& prm,
                              unsigned grid, unsigned threads, size_t smem, cudaStream_t st) {
  const uint32_t N = prm.N;
  if (N < 16 || N > 8192 || (N & (N - 1))) return cudaErrorInvalidValue;
  const int lg = 31 - __builtin_clz(N);
  if (prec == PREC_F64 || prec == PREC_DF64) {
    if (E != 16) return cudaErrorInvalidValue;
    return prec == PREC_F64 ? launch_pow2_fixed_f64(lg, colmajor, prm, grid, threads, smem, st)
                            : launch_pow2_fixed_df64(lg, colmajor, prm, grid, threads, smem, st);
  }
  if (prec != PREC_F32) return cudaErrorInvalidValue;
  if (!colmajor && E == 16) {
    switch (lg) {
      case 4: return fx_launch<float, 16, false, 4>(prm, grid, threads, smem, st);
      case 5: return fx_launch<float, 16, false, 5>(prm, grid, threads, smem, st);
      case 6: return fx_launch<float, 16, false, 6>(prm, grid, threads, smem, st);
      case 7: return fx_launch<float, 16, false, 7>(prm, grid, threads, smem, st);
      case 8: return fx_launch<float, 16, false, 8>(prm, grid, threads, smem, st);
      case 9: return fx_launch<float, 16, false, 9>(prm, grid, threads, smem, st);
      case 10: return fx_launch<float, 16, false, 10>(prm, grid, threads, smem, st);
      case 11: return fx_launch<float, 16, false, 11>(prm, grid, threads, smem, st);
      case 12: return fx_launch<float, 16, false, 12>(prm, grid, threads, smem, st);
      case 13: return fx_launch<float, 16, false, 13>(prm, grid, threads, smem, st);
      default: break;
    }
  } else if (colmajor && E == 16) {
    switch (lg) {
      case 4: return fx_launch<float, 16, true, 4>(prm, grid, threads, smem, st);
      case 5: return fx_launch<float, 16, true, 5>(prm, grid, threads, smem, st);
      case 6: return fx_launch<float, 16, true, 6>(prm, grid, threads, smem, st);
      case 7: return fx_launch<float, 16, true, 7>(prm, grid, threads, smem, st);
      case 8: return fx_launch<float, 16, true, 8>(prm, grid, threads, smem, st);
      case 9: return fx_launch<float, 16, true, 9>(prm, grid, threads, smem, st);
      default: break;
    }
  } else if (colmajor && E == 32) {
    switch (lg) {
      case 10: return fx_launch<float, 32, true, 10>(prm, grid, threads, smem, st);
      case 11: return fx_launch<float, 32, true, 11>(prm, grid, threads, smem, st);
      case 12: return fx_launch<float, 32, true, 12>(prm, grid, threads, smem, st);
      case 13: return fx_launch<float, 32, true, 13>(prm, grid, threads, smem, st);
      default: break;
    }
  }
  return cudaErrorInvalidValue;
}

}  // namespace b2f

namespace b2f {

cudaError_t launch_real_fixed(Prec p, bool r2c, const RealParams& prm, unsigned grid,
                              unsigned threads, size_t smem, cudaStream_t st) {
  const uint32_t h = prm.h;
  if (prm.N0 != 2 * h || h < 16 || h > 4096 || (h & (h - 1))) return cudaErrorInvalidValue;
  const int lg = 31 - __builtin_clz(h);
  if (p == PREC_F32)
    return r2c ? fx_real_any<float, true>(lg, prm, grid, threads, smem, st)
               : fx_real_any<float, false>(lg, prm, grid, threads, smem, st);
  if (p == PREC_F64) return launch_real_fixed_f64(lg, r2c, prm, grid, threads, smem, st);
  return cudaErrorInvalidValue;
}

}  // namespace b2f
