// Launch helpers of the fixed-length power-of-two kernels
// (regfft_fixed.cuh), shared by the per-precision translation units.
#pragma once
#include "regfft_fixed.cuh"

namespace b2f {

template <class S, int E, bool COLMAJOR, int LOGN>
inline cudaError_t fx_launch(const LinesParams& prm, unsigned grid, unsigned threads, size_t smem,
                             cudaStream_t st) {
  return launch(k_pow2_fx<S, E, COLMAJOR, LOGN>, prm, grid, threads, smem, st);
}

// f64 and df64 (16 values a thread, lines of up to 4096 points)
template <class S, bool COLMAJOR>
inline cudaError_t fx_launch_wide(int lg, const LinesParams& prm, unsigned grid, unsigned threads,
                                  size_t smem, cudaStream_t st) {
  switch (lg) {
    case 4: return fx_launch<S, 16, COLMAJOR, 4>(prm, grid, threads, smem, st);
    case 5: return fx_launch<S, 16, COLMAJOR, 5>(prm, grid, threads, smem, st);
    case 6: return fx_launch<S, 16, COLMAJOR, 6>(prm, grid, threads, smem, st);
    case 7: return fx_launch<S, 16, COLMAJOR, 7>(prm, grid, threads, smem, st);
    case 8: return fx_launch<S, 16, COLMAJOR, 8>(prm, grid, threads, smem, st);
    case 9: return fx_launch<S, 16, COLMAJOR, 9>(prm, grid, threads, smem, st);
    case 10: return fx_launch<S, 16, COLMAJOR, 10>(prm, grid, threads, smem, st);
    case 11: return fx_launch<S, 16, COLMAJOR, 11>(prm, grid, threads, smem, st);
    case 12: return fx_launch<S, 16, COLMAJOR, 12>(prm, grid, threads, smem, st);
    default: return cudaErrorInvalidValue;
  }
}

template <class S, bool R2C, int LOGH>
inline cudaError_t fx_real(const RealParams& prm, unsigned grid, unsigned threads, size_t smem,
                           cudaStream_t st) {
  if (R2C) return launch(k_r2c_fx<S, LOGH>, prm, grid, threads, smem, st);
  return launch(k_c2r_fx<S, LOGH>, prm, grid, threads, smem, st);
}

template <class S, bool R2C>
inline cudaError_t fx_real_any(int lg, const RealParams& prm, unsigned grid, unsigned threads,
                               size_t smem, cudaStream_t st) {
  switch (lg) {
    case 4: return fx_real<S, R2C, 4>(prm, grid, threads, smem, st);
    case 5: return fx_real<S, R2C, 5>(prm, grid, threads, smem, st);
    case 6: return fx_real<S, R2C, 6>(prm, grid, threads, smem, st);
    case 7: return fx_real<S, R2C, 7>(prm, grid, threads, smem, st);
    case 8: return fx_real<S, R2C, 8>(prm, grid, threads, smem, st);
    case 9: return fx_real<S, R2C, 9>(prm, grid, threads, smem, st);
    case 10: return fx_real<S, R2C, 10>(prm, grid, threads, smem, st);
    case 11: return fx_real<S, R2C, 11>(prm, grid, threads, smem, st);
    case 12: return fx_real<S, R2C, 12>(prm, grid, threads, smem, st);
    default: return cudaErrorInvalidValue;
  }
}

// per-precision instances (kernels_pow2_fx_f64.cu, kernels_pow2_fx_df64.cu)
cudaError_t launch_pow2_fixed_f64(int lg, bool colmajor, const LinesParams& prm, unsigned grid,
                                  unsigned threads, size_t smem, cudaStream_t st);
cudaError_t launch_pow2_fixed_df64(int lg, bool colmajor, const LinesParams& prm, unsigned grid,
                                   unsigned threads, size_t smem, cudaStream_t st);
cudaError_t launch_real_fixed_f64(int lg, bool r2c, const RealParams& prm, unsigned grid,
                                  unsigned threads, size_t smem, cudaStream_t st);

}  // namespace b2f
