// Power-of-two register kernels with the line length fixed at compile time
// (regfft_fixed.cuh).  f32: contiguous lines of 16..8192 points (16 values a
// thread) and column tiles of 16..512 (16 values) and 1024..8192 points
// (32 values); f64: lines and column tiles of 16..4096 points (16 values).
#include "regfft_fixed.cuh"

namespace b2f {

template <class S, int E, bool COLMAJOR, int LOGN>
static cudaError_t fx_launch(const LinesParams& prm, unsigned grid, unsigned threads, size_t smem,
                             cudaStream_t st) {
  return launch(k_pow2_fx<S, E, COLMAJOR, LOGN>, prm, grid, threads, smem, st);
}

template <bool COLMAJOR>
static cudaError_t fx_launch_f64(int lg, const LinesParams& prm, unsigned grid, unsigned threads,
                                 size_t smem, cudaStream_t st) {
  switch (lg) {
    case 4: return fx_launch<double, 16, COLMAJOR, 4>(prm, grid, threads, smem, st);
    case 5: return fx_launch<double, 16, COLMAJOR, 5>(prm, grid, threads, smem, st);
    case 6: return fx_launch<double, 16, COLMAJOR, 6>(prm, grid, threads, smem, st);
    case 7: return fx_launch<double, 16, COLMAJOR, 7>(prm, grid, threads, smem, st);
    case 8: return fx_launch<double, 16, COLMAJOR, 8>(prm, grid, threads, smem, st);
    case 9: return fx_launch<double, 16, COLMAJOR, 9>(prm, grid, threads, smem, st);
    case 10: return fx_launch<double, 16, COLMAJOR, 10>(prm, grid, threads, smem, st);
    case 11: return fx_launch<double, 16, COLMAJOR, 11>(prm, grid, threads, smem, st);
    case 12: return fx_launch<double, 16, COLMAJOR, 12>(prm, grid, threads, smem, st);
    default: return cudaErrorInvalidValue;
  }
}

// The compile-time kernel for (E, layout, N), or cudaErrorInvalidValue when
// there is none (the caller uses the generic kernel).
cudaError_t launch_pow2_fixed(Prec prec, int E, bool colmajor, const LinesParams& prm,
                              unsigned grid, unsigned threads, size_t smem, cudaStream_t st) {
  const uint32_t N = prm.N;
  if (N < 16 || N > 8192 || (N & (N - 1))) return cudaErrorInvalidValue;
  const int lg = 31 - __builtin_clz(N);
  if (prec == PREC_F64) {
    if (E != 16) return cudaErrorInvalidValue;
    return colmajor ? fx_launch_f64<true>(lg, prm, grid, threads, smem, st)
                    : fx_launch_f64<false>(lg, prm, grid, threads, smem, st);
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

template <class S, bool R2C, int LOGH>
static cudaError_t fx_real(const RealParams& prm, unsigned grid, unsigned threads, size_t smem,
                           cudaStream_t st) {
  if (R2C) return launch(k_r2c_fx<S, LOGH>, prm, grid, threads, smem, st);
  return launch(k_c2r_fx<S, LOGH>, prm, grid, threads, smem, st);
}

template <class S, bool R2C>
static cudaError_t fx_real_any(int lg, const RealParams& prm, unsigned grid, unsigned threads,
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

cudaError_t launch_real_fixed(Prec p, bool r2c, const RealParams& prm, unsigned grid,
                              unsigned threads, size_t smem, cudaStream_t st) {
  const uint32_t h = prm.h;
  if (prm.N0 != 2 * h || h < 16 || h > 4096 || (h & (h - 1))) return cudaErrorInvalidValue;
  const int lg = 31 - __builtin_clz(h);
  if (p == PREC_F32)
    return r2c ? fx_real_any<float, true>(lg, prm, grid, threads, smem, st)
               : fx_real_any<float, false>(lg, prm, grid, threads, smem, st);
  if (p == PREC_F64)
    return r2c ? fx_real_any<double, true>(lg, prm, grid, threads, smem, st)
               : fx_real_any<double, false>(lg, prm, grid, threads, smem, st);
  return cudaErrorInvalidValue;
}

}  // namespace b2f
