// f32 power-of-two register kernels with the line length fixed at compile
// time (regfft_fixed.cuh): contiguous lines of 16..8192 points (16 values a
// thread) and column tiles of 16..512 (16 values) and 1024..8192 points
// (32 values).
#include "regfft_fixed.cuh"

namespace b2f {

template <int E, bool COLMAJOR, int LOGN>
static cudaError_t fx_launch(const LinesParams& prm, unsigned grid, unsigned threads, size_t smem,
                             cudaStream_t st) {
  return launch(k_pow2_fx<E, COLMAJOR, LOGN>, prm, grid, threads, smem, st);
}

// The compile-time kernel for (E, layout, N), or cudaErrorInvalidValue when
// there is none (the caller uses the generic kernel).
cudaError_t launch_pow2_fixed(int E, bool colmajor, const LinesParams& prm, unsigned grid,
                              unsigned threads, size_t smem, cudaStream_t st) {
  const uint32_t N = prm.N;
  if (N < 16 || N > 8192 || (N & (N - 1))) return cudaErrorInvalidValue;
  const int lg = 31 - __builtin_clz(N);
  if (!colmajor && E == 16) {
    switch (lg) {
      case 4: return fx_launch<16, false, 4>(prm, grid, threads, smem, st);
      case 5: return fx_launch<16, false, 5>(prm, grid, threads, smem, st);
      case 6: return fx_launch<16, false, 6>(prm, grid, threads, smem, st);
      case 7: return fx_launch<16, false, 7>(prm, grid, threads, smem, st);
      case 8: return fx_launch<16, false, 8>(prm, grid, threads, smem, st);
      case 9: return fx_launch<16, false, 9>(prm, grid, threads, smem, st);
      case 10: return fx_launch<16, false, 10>(prm, grid, threads, smem, st);
      case 11: return fx_launch<16, false, 11>(prm, grid, threads, smem, st);
      case 12: return fx_launch<16, false, 12>(prm, grid, threads, smem, st);
      case 13: return fx_launch<16, false, 13>(prm, grid, threads, smem, st);
      default: break;
    }
  } else if (colmajor && E == 16) {
    switch (lg) {
      case 4: return fx_launch<16, true, 4>(prm, grid, threads, smem, st);
      case 5: return fx_launch<16, true, 5>(prm, grid, threads, smem, st);
      case 6: return fx_launch<16, true, 6>(prm, grid, threads, smem, st);
      case 7: return fx_launch<16, true, 7>(prm, grid, threads, smem, st);
      case 8: return fx_launch<16, true, 8>(prm, grid, threads, smem, st);
      case 9: return fx_launch<16, true, 9>(prm, grid, threads, smem, st);
      default: break;
    }
  } else if (colmajor && E == 32) {
    switch (lg) {
      case 10: return fx_launch<32, true, 10>(prm, grid, threads, smem, st);
      case 11: return fx_launch<32, true, 11>(prm, grid, threads, smem, st);
      case 12: return fx_launch<32, true, 12>(prm, grid, threads, smem, st);
      case 13: return fx_launch<32, true, 13>(prm, grid, threads, smem, st);
      default: break;
    }
  }
  return cudaErrorInvalidValue;
}

}  // namespace b2f
