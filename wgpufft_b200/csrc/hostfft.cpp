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

// Parallel top levels of fft_rec: the p sub-transforms of the first levels
// run on separate threads, and the combining loop over k is split too.
static void fft_rec_par(const cd* in, size_t stride, cd* out, size_t n, const std::vector<cd>& roots,
                        size_t rstride, int depth) {
  size_t p = n;
  for (size_t f = 2; f * f <= n; ++f)
    if (n % f == 0) {
      p = f;
      break;
    }
  if (depth >= 4 || n < (1u << 16) || p == n) {
    fft_rec(in, stride, out, n, roots, rstride);
    return;
  }
  const size_t m = n / p;
  {
    std::vector<std::thread> th;
    for (size_t r = 0; r < p; ++r)
      th.emplace_back([=, &roots] {
        fft_rec_par(in + r * stride, stride * p, out + r * m, m, roots, rstride * p, depth + 1);
      });
    for (auto& t : th) t.join();
  }
  parallel_ranges(m, [&](uint64_t k0, uint64_t k1) {
    std::vector<cd> col(p), res(p);
    for (size_t k = k0; k < k1; ++k) {
      for (size_t r = 0; r < p; ++r) col[r] = out[r * m + k] * roots[(r * k) * rstride];
      for (size_t s = 0; s < p; ++s) {
        cd acc = 0;
        for (size_t r = 0; r < p; ++r) acc += col[r] * roots[((r * s) % p) * m * rstride];
        res[s] = acc;
      }
      for (size_t s = 0; s < p; ++s) out[k + m * s] = res[s];
    }
  });
}

void fill_roots(std::vector<cd>& r, uint64_t M) {
  r.assign(M, cd(0, 0));
  if (M == 0) return;
  if (M % 8 != 0) {
    // half turn by conjugation: r[M - k] = conj(r[k])
    const uint64_t h = M / 2;
    parallel_ranges(h + 1, [&](uint64_t a, uint64_t b) {
      for (uint64_t k = a; k < b; ++k) r[k] = root_fwd(k, M);
    });
    for (uint64_t k = h + 1; k < M; ++k) r[k] = std::conj(r[M - k]);
    return;
  }
  // first octant directly; the quarter turn: r[M/4 - k] = (sin t, -cos t)
  // for r[k] = (cos t, -sin t)
  const uint64_t q = M / 4, o = M / 8;
  parallel_ranges(o + 1, [&](uint64_t a, uint64_t b) {
    for (uint64_t k = a; k < b; ++k) r[k] = root_fwd(k, M);
  });
  for (uint64_t k = 0; k < o; ++k) {
    const cd w = r[k];
    r[q - k] = cd(-w.imag(), -w.real());
  }
  // second quarter: r[q + k] = -i r[k]
  for (uint64_t k = 1; k < q; ++k) r[q + k] = cd(r[k].imag(), -r[k].real());
  r[q] = cd(0.0, -1.0);
  // second half: r[M/2 + k] = -r[k]
  for (uint64_t k = 0; k < 2 * q; ++k) r[2 * q + k] = -r[k];
}

void host_fft_fwd(std::vector<cd>& x) {
  const size_t n = x.size();
  if (n <= 1) return;
  std::vector<cd> roots;
  fill_roots(roots, n);
  std::vector<cd> out(n);
  fft_rec_par(x.data(), 1, out.data(), n, roots, 1, 0);
  x.swap(out);
}

std::vector<cd> chirp_spectrum(uint64_t N, uint64_t M) {
  std::vector<cd> b(M, cd(0, 0));
  parallel_ranges(N, [&](uint64_t a, uint64_t e) {
    for (uint64_t m = a; m < e; ++m) {
      const cd c = std::conj(chirp_fwd(m, N));
      b[m] = c;
      if (m) b[M - m] = c;
    }
  });
  host_fft_fwd(b);
  for (auto& x : b) x /= (double)M;
  return b;
}

}  // namespace b2f
