// Precision dispatch of the kernel launchers; the kernels themselves are
// instantiated once per precision in kernels_f32.cu, kernels_f64.cu and
// kernels_df64.cu (compiled in parallel).
#include <mutex>

#include "kernels.h"

namespace b2f {

template <class S>
cudaError_t launch_lines_t(const LinesParams&, unsigned, unsigned, size_t, cudaStream_t);
template <class S>
cudaError_t launch_rader_t(const RaderParams&, unsigned, unsigned, size_t, cudaStream_t);
template <class S>
cudaError_t launch_bluestein_t(const BluesteinParams&, unsigned, unsigned, size_t, cudaStream_t);
template <class S>
cudaError_t launch_r2c_t(const RealParams&, unsigned, unsigned, size_t, cudaStream_t);
template <class S>
cudaError_t launch_c2r_t(const RealParams&, unsigned, unsigned, size_t, cudaStream_t);
template <class S>
cudaError_t launch_scale_copy_t(const void*, void*, uint64_t, double, bool, cudaStream_t);
template <class S>
cudaError_t launch_blue_elem_t(const BlueElemParams&, cudaStream_t);

template <class S>
cudaError_t launch_real_elem_t(const RealElemParams&, cudaStream_t);
template <class S>
cudaError_t launch_small_volume_t(const SmallVolumeParams&, unsigned, size_t, cudaStream_t);

cudaError_t launch_small_volume(Prec p, const SmallVolumeParams& prm, unsigned threads,
                                size_t smem, cudaStream_t st) {
  if (p != PREC_F32) return cudaErrorInvalidValue;
  return launch_small_volume_t<float>(prm, threads, smem, st);
}

cudaError_t launch_real_elem(Prec p, const RealElemParams& prm, cudaStream_t st) {
  switch (p) {
    case PREC_F32: return launch_real_elem_t<float>(prm, st);
    case PREC_F64: return launch_real_elem_t<double>(prm, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_blue_elem(Prec p, const BlueElemParams& prm, cudaStream_t st) {
  switch (p) {
    case PREC_F32: return launch_blue_elem_t<float>(prm, st);
    case PREC_F64: return launch_blue_elem_t<double>(prm, st);
    case PREC_DF64: return launch_blue_elem_t<df>(prm, st);
  }
  return cudaErrorInvalidValue;
}

static size_t g_max_smem = 0;

size_t max_smem_per_block() {
  static std::once_flag once;
  std::call_once(once, [] {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
      v = 48 * 1024;
    g_max_smem = (size_t)v;
  });
  return g_max_smem;
}

template <class S, int E, bool COLMAJOR>
cudaError_t launch_pow2_t(const LinesParams&, unsigned, unsigned, size_t, cudaStream_t);

cudaError_t launch_pow2_fixed(Prec prec, int E, bool colmajor, const LinesParams& prm,
                              unsigned grid, unsigned threads, size_t smem, cudaStream_t st);

// The schedule the compile-time kernels assume for N = 2^m: radix-16
// stages, then one radix 2^(m mod 4) stage, stage twiddle tables in order.
static bool pow2_schedule_is_default(const LinesParams& prm) {
  const uint32_t N = prm.N;
  if (N < 16 || (N & (N - 1)) || prm.sch.N != N) return false;
  const int lg = 31 - __builtin_clz(N);
  const uint32_t nst = (uint32_t)(lg + 3) / 4;
  if (prm.sch.nst != nst) return false;
  uint32_t ns = 1, tw = 0;
  for (uint32_t s = 0; s < nst; ++s) {
    const uint32_t R = (int)s < lg / 4 ? 16u : (1u << (lg % 4));
    const StageDesc& d = prm.sch.st[s];
    if (d.R != R || d.Ns != ns || d.tw_off != tw) return false;
    tw += ns * (R - 1);
    ns *= R;
  }
  return true;
}

cudaError_t launch_pow2(Prec p, int E, bool colmajor, const LinesParams& prm, unsigned grid,
                        unsigned threads, size_t smem, cudaStream_t st) {
  // the compile-time kernel of this length when the schedule is the one it
  // assumes; the generic one otherwise
  if (pow2_schedule_is_default(prm)) {
    const cudaError_t e = launch_pow2_fixed(p, E, colmajor, prm, grid, threads, smem, st);
    if (e != cudaErrorInvalidValue) return e;
  }
  switch (p) {
    case PREC_F32:
      if (E == 32)  // column tiles only
        return colmajor ? launch_pow2_t<float, 32, true>(prm, grid, threads, smem, st)
                        : cudaErrorInvalidValue;
      return colmajor ? launch_pow2_t<float, 16, true>(prm, grid, threads, smem, st)
                      : launch_pow2_t<float, 16, false>(prm, grid, threads, smem, st);
    case PREC_F64:
      return colmajor ? launch_pow2_t<double, 16, true>(prm, grid, threads, smem, st)
                      : launch_pow2_t<double, 16, false>(prm, grid, threads, smem, st);
    case PREC_DF64:
      return colmajor ? launch_pow2_t<df, 16, true>(prm, grid, threads, smem, st)
                      : launch_pow2_t<df, 16, false>(prm, grid, threads, smem, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_lines(Prec p, const LinesParams& prm, unsigned grid, unsigned threads,
                         size_t smem, cudaStream_t st) {
  switch (p) {
    case PREC_F32: return launch_lines_t<float>(prm, grid, threads, smem, st);
    case PREC_F64: return launch_lines_t<double>(prm, grid, threads, smem, st);
    case PREC_DF64: return launch_lines_t<df>(prm, grid, threads, smem, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_rader(Prec p, const RaderParams& prm, unsigned grid, unsigned threads,
                         size_t smem, cudaStream_t st) {
  switch (p) {
    case PREC_F32: return launch_rader_t<float>(prm, grid, threads, smem, st);
    case PREC_F64: return launch_rader_t<double>(prm, grid, threads, smem, st);
    case PREC_DF64: return launch_rader_t<df>(prm, grid, threads, smem, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_bluestein(Prec p, const BluesteinParams& prm, unsigned grid,
                             unsigned threads, size_t smem, cudaStream_t st) {
  switch (p) {
    case PREC_F32: return launch_bluestein_t<float>(prm, grid, threads, smem, st);
    case PREC_F64: return launch_bluestein_t<double>(prm, grid, threads, smem, st);
    case PREC_DF64: return launch_bluestein_t<df>(prm, grid, threads, smem, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_r2c(Prec p, const RealParams& prm, unsigned grid, unsigned threads,
                       size_t smem, cudaStream_t st) {
  switch (p) {
    case PREC_F32: return launch_r2c_t<float>(prm, grid, threads, smem, st);
    case PREC_F64: return launch_r2c_t<double>(prm, grid, threads, smem, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_c2r(Prec p, const RealParams& prm, unsigned grid, unsigned threads,
                       size_t smem, cudaStream_t st) {
  switch (p) {
    case PREC_F32: return launch_c2r_t<float>(prm, grid, threads, smem, st);
    case PREC_F64: return launch_c2r_t<double>(prm, grid, threads, smem, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_scale_copy(Prec p, const void* in, void* out, uint64_t n, double scale,
                              bool conj, cudaStream_t st) {
  switch (p) {
    case PREC_F32: return launch_scale_copy_t<float>(in, out, n, scale, conj, st);
    case PREC_F64: return launch_scale_copy_t<double>(in, out, n, scale, conj, st);
    case PREC_DF64: return launch_scale_copy_t<df>(in, out, n, scale, conj, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace b2f
