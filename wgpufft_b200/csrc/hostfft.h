// FP64 host FFT used only to build the plan tables that must be exact to the
// last bit of the working precision: stage twiddles, the Rader kernel
// spectrum and the Bluestein chirp spectrum (the reference builds the same
// tables in FP64 on the host: src/runtime/twiddle.rs:15-37,
// src/runtime/rader_axis.rs:1318-1336, src/runtime/bluestein_axis.rs:841-856).
// Roots come from long double sin/cos of the exactly reduced angle, so each
// table entry is rounded once.
#pragma once
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <thread>
#include <vector>

namespace b2f {

using cd = std::complex<double>;

// exp(-2 pi i m / M), m reduced modulo M first.
inline cd root_fwd(uint64_t m, uint64_t M) {
  m %= M;
  // reduce to [-M/2, M/2] so the long double angle is small and exact-ish
  long double num = (long double)m;
  if (2 * m > M) num -= (long double)M;
  const long double ang = -2.0L * 3.141592653589793238462643383279502884L * num / (long double)M;
  return cd((double)cosl(ang), (double)sinl(ang));
}

// exp(-i pi n^2 / N) with n^2 reduced modulo 2N in integers.
inline cd chirp_fwd(uint64_t n, uint64_t N) {
  const unsigned __int128 sq = (unsigned __int128)n * n % (2 * (unsigned __int128)N);
  return root_fwd((uint64_t)sq, 2 * N);
}

// Unnormalised forward DFT of any length: recursive decimation in time that
// splits off the smallest factor, plain DFT for prime lengths up to 64 and
// Bluestein over a power of two above.  Large transforms run their top
// levels on several host threads.
void host_fft_fwd(std::vector<cd>& x);

// r[k] = exp(-2 pi i k / M) for k < M (r is resized): each root is computed
// once per octant as root_fwd does and mirrored through the exact
// symmetries of the unit circle (conjugation, the quarter-turn swap), on
// several host threads for large M.
void fill_roots(std::vector<cd>& r, uint64_t M);

// The Bluestein spectrum of a length-N line over a length-M convolution:
// FFT_M of the conjugate chirp (b[m] = b[M-m] = conj(chirp(m)), zero in the
// middle), divided by M.
std::vector<cd> chirp_spectrum(uint64_t N, uint64_t M);

// Runs f(begin, end) over [0, n) split across host threads (one call when n
// is small).
template <class F>
void parallel_ranges(uint64_t n, F f);

template <class F>
void parallel_ranges(uint64_t n, F f) {
  const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  const uint64_t nt = n < (1u << 15) ? 1 : std::min<uint64_t>(hw, n >> 14);
  if (nt <= 1) {
    f(0, n);
    return;
  }
  std::vector<std::thread> th;
  for (uint64_t t = 0; t < nt; ++t)
    th.emplace_back([&, t] { f(n * t / nt, n * (t + 1) / nt); });
  for (auto& x : th) x.join();
}

// chirp_fwd(n, N) for n < N (the Bluestein pre- and post-multiplier), on
// several host threads for long lines.
inline std::vector<cd> chirp_table(uint64_t N) {
  std::vector<cd> c(N);
  parallel_ranges(N, [&](uint64_t a, uint64_t b) {
    for (uint64_t n = a; n < b; ++n) c[n] = chirp_fwd(n, N);
  });
  return c;
}

}  // namespace b2f
