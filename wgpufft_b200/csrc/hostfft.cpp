// FP64 host FFT for table generation (see hostfft.h).
#include "hostfft.h"

namespace b2f {

static void fft_rec(const cd* in, size_t stride, cd* out, size_t n, const std::vector<cd>& roots,
                    size_t rstride);

static void bluestein(const cd* in, size_t stride, cd* out, size_t n) {
  size_t m = 1;
  while (m < 2 * n - 1) m <<= 1;
  std::vector<cd> a(m), b(m), c(n);
  for (size_t k = 0; k < n; ++k) {
    c[k] = chirp_fwd(k, n);
    a[k] = in[k * stride] * c[k];
    b[k] = std::conj(c[k]);
    if (k) b[m - k] = b[k];
  }
  host_fft_fwd(a);
  host_fft_fwd(b);
  for (size_t k = 0; k < m; ++k) a[k] = std::conj(a[k] * b[k]);
  host_fft_fwd(a);  // conj(FFT(conj(y))) = unnormalised inverse
  for (size_t k = 0; k < n; ++k) out[k] = std::conj(a[k]) * c[k] / (double)m;
}

static void fft_rec(const cd* in, size_t stride, cd* out, size_t n, const std::vector<cd>& roots,
                    size_t rstride) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  size_t p = n;
  for (size_t f = 2; f * f <= n; ++f)
    if (n % f == 0) {
      p = f;
      break;
    }
  if (p == n) {
    if (n > 64) {
      bluestein(in, stride, out, n);
      return;
    }
    for (size_t k = 0; k < n; ++k) {
      cd s = 0;
      for (size_t j = 0; j < n; ++j) s += in[j * stride] * roots[(j * k % n) * rstride];
      out[k] = s;
    }
    return;
  }
  const size_t m = n / p;
  for (size_t r = 0; r < p; ++r) fft_rec(in + r * stride, stride * p, out + r * m, m, roots, rstride * p);
  std::vector<cd> col(p);
  for (size_t k = 0; k < m; ++k) {
    for (size_t r = 0; r < p; ++r) col[r] = out[r * m + k] * roots[(r * k) * rstride];
    for (size_t s = 0; s < p; ++s) {
      cd acc = 0;
      for (size_t r = 0; r < p; ++r) acc += col[r] * roots[((r * s) % p) * m * rstride];
      out[k + m * s] = acc;
    }
  }
}

void host_fft_fwd(std::vector<cd>& x) {
  const size_t n = x.size();
  if (n <= 1) return;
  std::vector<cd> roots(n);
  for (size_t k = 0; k < n; ++k) roots[k] = root_fwd(k, n);
  std::vector<cd> out(n);
  fft_rec(x.data(), 1, out.data(), n, roots, 1);
  x.swap(out);
}

}  // namespace b2f
