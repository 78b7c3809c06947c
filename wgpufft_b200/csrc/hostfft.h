// FP64 host FFT used only to build the plan tables that must be exact to the
// last bit of the working precision: stage twiddles, the Rader kernel
// spectrum and the Bluestein chirp spectrum (the reference builds the same
// tables in FP64 on the host: src/runtime/twiddle.rs:15-37,
// src/runtime/rader_axis.rs:1318-1336, src/runtime/bluestein_axis.rs:841-856).
// Roots come from long double sin/cos of the exactly reduced angle, so each
// table entry is rounded once.
#pragma once
#include <cmath>
#include <complex>
#include <cstdint>
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
// Bluestein over a power of two above.
void host_fft_fwd(std::vector<cd>& x);

}  // namespace b2f
