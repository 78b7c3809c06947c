// Transform kernels for sm_100a.  Each kernel stages G lines of one pass in
// shared memory, runs the Stockham engine (engine.cuh) and writes the lines
// back, fusing everything a pass needs around the FFT into the same trip
// through HBM: conjugation for inverse transforms, the four-step twiddle,
// normalisation, the Rader permutations and kernel-spectrum product, the
// Bluestein chirps, and the real-to-complex packing.
#pragma once
#include <mutex>
#include <set>
#include <utility>

#include "kernels.h"

namespace b2f {

template <class S>
using C = cpx<S>;

struct Group {
  int64_t in0, out0, dl_in, dl_out;
  uint32_t nvalid;
  uint64_t c0;
};

FFT_D Group group_of(const LineIO& io, uint32_t G, uint64_t blk) {
  Group g;
  const uint64_t rest = blk / io.tiles;
  const uint64_t tile = blk - rest * io.tiles;
  const uint64_t outer = rest / io.mid_n;
  const uint64_t mid = rest - outer * io.mid_n;
  const uint64_t c0 = tile * G;
  const uint64_t left = io.inner_n - c0;
  g.nvalid = left < G ? (uint32_t)left : G;
  g.in0 = (int64_t)outer * io.in_outer + (int64_t)mid * io.in_mid + (int64_t)c0 * io.in_inner;
  g.out0 = (int64_t)outer * io.out_outer + (int64_t)mid * io.out_mid + (int64_t)c0 * io.out_inner;
  g.dl_in = io.in_inner;
  g.dl_out = io.out_inner;
  g.c0 = c0;
  return g;
}

// Visits the (line c, point n) pairs of a G x count block.  cfirst walks
// adjacent lines first (coalesced when lines are adjacent columns); else it
// walks each line's points first (coalesced when lines are contiguous).
template <class F>
FFT_D void for_each_elem(uint32_t count, const FastDiv& dcount, uint32_t G, const FastDiv& dG,
                         bool cfirst, uint32_t tid, uint32_t T, F f) {
  const uint32_t total = G * count;
  if (cfirst) {
    for (uint32_t e = tid; e < total; e += T) {
      const uint32_t n = fdiv(e, dG);
      f(e - n * G, n);
    }
  } else {
    for (uint32_t e = tid; e < total; e += T) {
      const uint32_t c = fdiv(e, dcount);
      f(c, e - c * count);
    }
  }
}

// Elements a thread takes at once in the batched loops: a loop that loads
// one element and consumes it before the next keeps one global load in
// flight per thread and waits out each one's latency.
template <class S>
struct BatchU {
  static constexpr int value = sizeof(C<S>) <= 8 ? 8 : 4;
};

// for_each_elem, U elements a thread at a time: f(c, n) for all U first
// (their global loads in flight together), then g(c, n, value) for each.
template <int U, class V, class F, class Gf>
FFT_D void for_each_elem_batched(uint32_t count, const FastDiv& dcount, uint32_t G,
                                 const FastDiv& dG, bool cfirst, uint32_t tid, uint32_t T, F f,
                                 Gf g) {
  const uint32_t total = G * count;
  auto split = [&](uint32_t e, uint32_t& c, uint32_t& n) {
    if (cfirst) {
      n = fdiv(e, dG);
      c = e - n * G;
    } else {
      c = fdiv(e, dcount);
      n = e - c * count;
    }
  };
  uint32_t e = tid;
  for (; e + (U - 1) * T < total; e += U * T) {
    V v[U];
    uint32_t cs[U], ns[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      split(e + u * T, cs[u], ns[u]);
      v[u] = f(cs[u], ns[u]);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) g(cs[u], ns[u], v[u]);
  }
  for (; e < total; e += T) {
    uint32_t c, n;
    split(e, c, n);
    g(c, n, f(c, n));
  }
}

template <class S>
struct CPair {
  C<S> a, b;
};

// Column tiles whose line count G is a power of two dividing the thread
// count: each thread keeps one line c = tid mod G and walks its points
// n = tid / G, + T / G, ... (no division per value, stepped addresses).
FFT_D bool fixed_line_walk(uint32_t G, uint32_t T) {
  return (G & (G - 1)) == 0 && (T & (G - 1)) == 0;
}

template <class S>
FFT_D void load_lines(C<S>* sm, const LinesParams& p, const Group& g, uint32_t tid, uint32_t T) {
  constexpr int PAD = PadOf<S>::value;
  const C<S>* __restrict__ in = (const C<S>*)p.in;
  const bool conj_in = p.flags & PF_CONJ_IN;
  if ((p.flags & PF_CFIRST_LOAD) && fixed_line_walk(p.G, T)) {
    const uint32_t lg = 31 - __clz(p.G), c = tid & (p.G - 1), dn = T >> lg;
    if (c < g.nvalid) {
      const int64_t es = p.io.in_es;
      const C<S>* src = in + g.in0 + (int64_t)c * g.dl_in;
      C<S>* line = sm + c * p.LD;
      constexpr int U = BatchU<S>::value;
      uint32_t n = tid >> lg;
      for (; n + (U - 1) * dn < p.N; n += U * dn) {
        C<S> v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) v[u] = src[(int64_t)(n + u * dn) * es];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (conj_in) v[u].im = -v[u].im;
          line[pidx<PAD>(n + u * dn)] = v[u];
        }
      }
      for (; n < p.N; n += dn) {
        C<S> v = src[(int64_t)n * es];
        if (conj_in) v.im = -v.im;
        line[pidx<PAD>(n)] = v;
      }
    }
    return;
  }
  for_each_elem_batched<BatchU<S>::value, C<S>>(
      p.N, p.dN, p.G, p.dG, p.flags & PF_CFIRST_LOAD, tid, T,
      [&](uint32_t c, uint32_t n) {
        return c < g.nvalid ? in[g.in0 + (int64_t)c * g.dl_in + (int64_t)n * p.io.in_es]
                            : czero<S>();
      },
      [&](uint32_t c, uint32_t n, C<S> v) {
        if (c < g.nvalid) {
          if (conj_in) v.im = -v.im;
          sm[c * p.LD + pidx<PAD>(n)] = v;
        }
      });
}

template <class S>
FFT_D void store_lines(const C<S>* sm, const LinesParams& p, const Group& g, uint32_t tid,
                       uint32_t T) {
  constexpr int PAD = PadOf<S>::value;
  C<S>* __restrict__ out = (C<S>*)p.out;
  const uint32_t fl = p.flags;
  const S sc = Scalar<S>::from_double(p.scale);
  if ((fl & PF_CFIRST_STORE) && fixed_line_walk(p.G, T)) {
    const uint32_t lg = 31 - __clz(p.G), c = tid & (p.G - 1), dn = T >> lg;
    if (c >= g.nvalid) return;
    const int64_t es = p.io.out_es;
    C<S>* dst = out + g.out0 + (int64_t)c * g.dl_out;
    const C<S>* line = sm + c * p.LD;
    const C<S>* __restrict__ ta = (const C<S>*)p.tws_a;
    const C<S>* __restrict__ tb = (const C<S>*)p.tws_b;
    const uint64_t row = (fl & PF_TW_STORE) ? fdiv((uint32_t)(g.c0 + c), p.d_tw) : 0;
    // W_M^{row n}: a 32-bit exponent stepped by row * dn through the
    // power-of-two-split tables when M < 2^32
    const bool step_tw = ta != nullptr && p.d_tws.mul == 0 && p.tw_store_M <= 0xFFFFFFFFull;
    const uint32_t sh = p.d_tws.shift, msk = (1u << sh) - 1;
    const uint32_t n0 = tid >> lg;
    uint32_t m32 = (uint32_t)row * n0;
    const uint32_t dm = (uint32_t)row * dn;
    // twiddle W_M^{row n} of point n (its table loads)
    auto tw_at = [&](uint32_t n, uint32_t m) -> C<S> {
      if (step_tw) return cmul(ta[m >> sh], tb[m & msk]);
      const uint64_t mm = row * (uint64_t)n;
      return ta ? tw_two_level(ta, tb, mm, p.d_tws) : twiddle<S>(mm % p.tw_store_M, p.tw_store_M);
    };
    auto put = [&](uint32_t n, C<S> v) {
      if (fl & PF_SCALE) v = cscale(v, sc);
      if (fl & PF_CONJ_OUT) v.im = -v.im;
      dst[(int64_t)n * es] = v;
    };
    uint32_t n = n0;
    if (fl & PF_TW_STORE) {
      // U points' table loads in flight together
      constexpr int U = BatchU<S>::value;
      for (; n + (U - 1) * dn < p.N; n += U * dn) {
        C<S> w[U];
#pragma unroll
        for (int u = 0; u < U; ++u) w[u] = tw_at(n + u * dn, m32 + u * dm);
#pragma unroll
        for (int u = 0; u < U; ++u) put(n + u * dn, cmul(line[pidx<PAD>(n + u * dn)], w[u]));
        m32 += U * dm;
      }
    }
    for (; n < p.N; n += dn) {
      C<S> v = line[pidx<PAD>(n)];
      if (fl & PF_TW_STORE) {
        v = cmul(v, tw_at(n, m32));
        m32 += dm;
      }
      put(n, v);
    }
    return;
  }
  if (fl & PF_TW_STORE) {
    // row < M / N and n < N: the exponent stays below M
    for_each_elem_batched<BatchU<S>::value, C<S>>(
        p.N, p.dN, p.G, p.dG, fl & PF_CFIRST_STORE, tid, T,
        [&](uint32_t c, uint32_t n) {
          if (c >= g.nvalid) return czero<S>();
          const uint64_t row = fdiv((uint32_t)(g.c0 + c), p.d_tw);
          const uint64_t m = row * (uint64_t)n;
          return p.tws_a ? tw_two_level((const C<S>*)p.tws_a, (const C<S>*)p.tws_b, m, p.d_tws)
                         : twiddle<S>(m % p.tw_store_M, p.tw_store_M);
        },
        [&](uint32_t c, uint32_t n, C<S> w) {
          if (c < g.nvalid) {
            C<S> v = cmul(sm[c * p.LD + pidx<PAD>(n)], w);
            if (fl & PF_SCALE) v = cscale(v, sc);
            if (fl & PF_CONJ_OUT) v.im = -v.im;
            out[g.out0 + (int64_t)c * g.dl_out + (int64_t)n * p.io.out_es] = v;
          }
        });
    return;
  }
  for_each_elem(p.N, p.dN, p.G, p.dG, fl & PF_CFIRST_STORE, tid, T, [&](uint32_t c, uint32_t n) {
    if (c < g.nvalid) {
      C<S> v = sm[c * p.LD + pidx<PAD>(n)];
      if (fl & PF_SCALE) v = cscale(v, sc);
      if (fl & PF_CONJ_OUT) v.im = -v.im;
      out[g.out0 + (int64_t)c * g.dl_out + (int64_t)n * p.io.out_es] = v;
    }
  });
}

template <class S>
FFT_D const C<S>* tw_of(const LinesParams& p) {
  return (p.flags & PF_TW_TABLE) ? (const C<S>*)p.tw : nullptr;
}

// ------------------------------------------------------------ mixed radix
// Shared memory: two line buffers of G*LD elements (ping-pong).
template <class S>
__global__ void __launch_bounds__(512) k_lines(const __grid_constant__ LinesParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C<S>* A = reinterpret_cast<C<S>*>(smem_raw);
  C<S>* B = A + p.G * p.LD;
  const uint32_t tid = threadIdx.x, T = blockDim.x;
  const Group g = group_of(p.io, p.G, blockIdx.x);
  load_lines<S>(A, p, g, tid, T);
  __syncthreads();
  const C<S>* res = fft_lines_smem<S>(A, B, p.sch, p.G, p.LD, tid, T, tw_of<S>(p));
  store_lines<S>(res, p, g, tid, T);
}

// ------------------------------------------------------------------ Rader
// X[0] = sum x; X[g^-r] = x[0] + (a (*) b)[r] with a[q] = x[g^q] and
// b[q] = W_p^{g^-q}, a cyclic convolution of length p-1 taken through
// FFT_{p-1}, the product with the precomputed spectrum of b, and the
// inverse FFT (src/runtime/rader_axis.rs:1228-1336 builds the same pieces).
// Shared memory: two buffers of G*LD, then x0[G] and X0[G].
template <class S>
__global__ void __launch_bounds__(512) k_rader(const __grid_constant__ RaderParams rp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int PAD = PadOf<S>::value;
  const LinesParams& p = rp.L;
  C<S>* A = reinterpret_cast<C<S>*>(smem_raw);
  C<S>* B = A + p.G * p.LD;
  C<S>* x0s = B + p.G * p.LD;
  C<S>* X0s = x0s + p.G;
  const uint32_t tid = threadIdx.x, T = blockDim.x;
  const uint32_t P = p.N, P1 = P - 1, G = p.G, LD = p.LD;
  const Group g = group_of(p.io, G, blockIdx.x);
  load_lines<S>(A, p, g, tid, T);
  __syncthreads();
  if (tid < G) x0s[tid] = A[tid * LD];
  for_each_elem_batched<8, uint32_t>(
      P1, rp.dP1, G, p.dG, false, tid, T, [&](uint32_t, uint32_t q) { return rp.perm_in[q]; },
      [&](uint32_t l, uint32_t q, uint32_t j) { B[l * LD + pidx<PAD>(q)] = A[l * LD + pidx<PAD>(j)]; });
  __syncthreads();
  C<S>* r1 = fft_lines_smem<S>(B, A, p.sch, G, LD, tid, T, tw_of<S>(p));
  C<S>* o1 = (r1 == A) ? B : A;
  if (tid < G) X0s[tid] = x0s[tid] + r1[tid * LD];
  __syncthreads();
  {
    const C<S>* __restrict__ bhat = (const C<S>*)rp.bhat;
    for_each_elem_batched<BatchU<S>::value, C<S>>(
        P1, rp.dP1, G, p.dG, false, tid, T, [&](uint32_t, uint32_t m) { return bhat[m]; },
        [&](uint32_t l, uint32_t m, C<S> b) {
          C<S> v = cmul(r1[l * LD + pidx<PAD>(m)], b);
          v.im = -v.im;
          r1[l * LD + pidx<PAD>(m)] = v;
        });
  }
  __syncthreads();
  const C<S>* r2 = fft_lines_smem<S>(r1, o1, p.sch, G, LD, tid, T, tw_of<S>(p));
  // X[n] = x0 + conv[r(n)], conv = conj(result)
  C<S>* __restrict__ out = (C<S>*)p.out;
  const uint32_t fl = p.flags;
  const S sc = Scalar<S>::from_double(p.scale);
  for_each_elem_batched<8, uint32_t>(
      P, p.dN, G, p.dG, fl & PF_CFIRST_STORE, tid, T,
      [&](uint32_t c, uint32_t n) { return c < g.nvalid && n > 0 ? rp.perm_out[n - 1] : 0u; },
      [&](uint32_t c, uint32_t n, uint32_t j) {
        if (c < g.nvalid) {
          C<S> v;
          if (n == 0) {
            v = X0s[c];
          } else {
            C<S> w = r2[c * LD + pidx<PAD>(j)];
            w.im = -w.im;
            v = x0s[c] + w;
          }
          if (fl & PF_SCALE) v = cscale(v, sc);
          if (fl & PF_CONJ_OUT) v.im = -v.im;
          out[g.out0 + (int64_t)c * g.dl_out + (int64_t)n * p.io.out_es] = v;
        }
      });
}

// -------------------------------------------------------------- Bluestein
// X[k] = c_k * sum_j (x_j c_j) conj(c_{k-j}) with the chirp
// c_n = exp(-i pi n^2 / N), n^2 reduced modulo 2N in integers
// (src/runtime/bluestein_axis.rs:825-867); the convolution runs over M >= 2N-1
// points against the precomputed spectrum of the conjugate chirp.
template <class S>
FFT_D C<S> chirp(uint64_t n, uint32_t N) {
  const uint64_t twoN = 2ull * N;
  return twiddle<S>((n * n) % twoN, twoN);
}

template <class S>
__global__ void __launch_bounds__(512) k_bluestein(const __grid_constant__ BluesteinParams bp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int PAD = PadOf<S>::value;
  const LinesParams& p = bp.L;
  C<S>* A = reinterpret_cast<C<S>*>(smem_raw);
  C<S>* B = A + p.G * p.LD;
  const uint32_t tid = threadIdx.x, T = blockDim.x;
  const uint32_t N = p.N, M = bp.M, G = p.G, LD = p.LD;
  const Group g = group_of(p.io, G, blockIdx.x);
  const C<S>* __restrict__ ctab = (const C<S>*)bp.chirp;
  {
    const C<S>* __restrict__ in = (const C<S>*)p.in;
    const bool conj_in = p.flags & PF_CONJ_IN;
    for_each_elem_batched<BatchU<S>::value, CPair<S>>(
        N, p.dN, G, p.dG, p.flags & PF_CFIRST_LOAD, tid, T,
        [&](uint32_t c, uint32_t n) {
          CPair<S> x{czero<S>(), czero<S>()};
          if (c < g.nvalid) {
            x.a = in[g.in0 + (int64_t)c * g.dl_in + (int64_t)n * p.io.in_es];
            x.b = ctab ? ctab[n] : chirp<S>(n, N);
          }
          return x;
        },
        [&](uint32_t c, uint32_t n, CPair<S> x) {
          if (c < g.nvalid) {
            if (conj_in) x.a.im = -x.a.im;
            A[c * LD + pidx<PAD>(n)] = cmul(x.a, x.b);
          }
        });
    const uint32_t pad = M - N;
    const uint32_t tot = G * pad;
    for (uint32_t e = tid; e < tot; e += T) {
      const uint32_t l = fdiv(e, bp.dMN), m = N + (e - l * pad);
      A[l * LD + pidx<PAD>(m)] = czero<S>();
    }
  }
  __syncthreads();
  C<S>* r1 = fft_lines_smem<S>(A, B, p.sch, G, LD, tid, T, tw_of<S>(p));
  C<S>* o1 = (r1 == A) ? B : A;
  {
    const C<S>* __restrict__ bhat = (const C<S>*)bp.bhat;
    for_each_elem_batched<BatchU<S>::value, C<S>>(
        M, bp.dM, G, p.dG, false, tid, T, [&](uint32_t, uint32_t m) { return bhat[m]; },
        [&](uint32_t l, uint32_t m, C<S> b) {
          C<S> v = cmul(r1[l * LD + pidx<PAD>(m)], b);
          v.im = -v.im;
          r1[l * LD + pidx<PAD>(m)] = v;
        });
  }
  __syncthreads();
  const C<S>* r2 = fft_lines_smem<S>(r1, o1, p.sch, G, LD, tid, T, tw_of<S>(p));
  C<S>* __restrict__ out = (C<S>*)p.out;
  const uint32_t fl = p.flags;
  const S sc = Scalar<S>::from_double(p.scale);
  for_each_elem_batched<BatchU<S>::value, C<S>>(
      N, p.dN, G, p.dG, fl & PF_CFIRST_STORE, tid, T,
      [&](uint32_t c, uint32_t k) {
        return c < g.nvalid ? (ctab ? ctab[k] : chirp<S>(k, N)) : czero<S>();
      },
      [&](uint32_t c, uint32_t k, C<S> ch) {
        if (c < g.nvalid) {
          C<S> w = r2[c * LD + pidx<PAD>(k)];
          w.im = -w.im;
          C<S> v = cmul(w, ch);
          if (fl & PF_SCALE) v = cscale(v, sc);
          if (fl & PF_CONJ_OUT) v.im = -v.im;
          out[g.out0 + (int64_t)c * g.dl_out + (int64_t)k * p.io.out_es] = v;
        }
      });
}

// ------------------------------------------------------------------ real
// R2C, even N0 = 2h: the real line read as h complex pairs z[n] = x[2n] +
// i x[2n+1], Z = FFT_h(z), then X[k] = E + W^k O and X[h-k] = conj(E - W^k O)
// with E = (Z[k] + conj Z[h-k]) / 2, O = -i (Z[k] - conj Z[h-k]) / 2, written
// straight to the packed layout [N0/2 + 1, ...] of the reference
// (src/math/mod.rs:444-448).
template <class S>
__global__ void __launch_bounds__(512) k_r2c_even(const __grid_constant__ RealParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int PAD = PadOf<S>::value;
  C<S>* A = reinterpret_cast<C<S>*>(smem_raw);
  C<S>* B = A + p.G * p.LD;
  const uint32_t tid = threadIdx.x, T = blockDim.x;
  const uint32_t h = p.h, G = p.G, LD = p.LD, P = h + 1;
  const uint64_t l0 = (uint64_t)blockIdx.x * G;
  const uint32_t nvalid = (p.nlines - l0) < G ? (uint32_t)(p.nlines - l0) : G;
  const C<S>* __restrict__ in = (const C<S>*)p.in;
  for_each_elem_batched<4, C<S>>(
      h, p.dh, G, p.dG, false, tid, T,
      [&](uint32_t c, uint32_t n) { return c < nvalid ? in[(l0 + c) * h + n] : czero<S>(); },
      [&](uint32_t c, uint32_t n, C<S> v) {
        if (c < nvalid) A[c * LD + pidx<PAD>(n)] = v;
      });
  __syncthreads();
  const C<S>* Z = fft_lines_smem<S>(A, B, p.sch, G, LD, tid, T,
                                     (p.flags & PF_TW_TABLE) ? (const C<S>*)p.tw : nullptr);
  C<S>* __restrict__ out = (C<S>*)p.out;
  const S half = Scalar<S>::from_double(0.5);
  const S sc = Scalar<S>::from_double(p.scale);
  const uint32_t K = h / 2 + 1;
  const uint32_t tot = G * K;
  for (uint32_t e = tid; e < tot; e += T) {
    const uint32_t c = e / K, k = e - c * K;
    if (c >= nvalid) continue;
    const C<S> a = Z[c * LD + pidx<PAD>(k)];
    const C<S> b = conj(Z[c * LD + pidx<PAD>(k == 0 ? 0 : h - k)]);
    const C<S> E = cscale(a + b, half);
    const C<S> O = cscale(mul_neg_i(a - b), half);
    const C<S> WO = cmul(O, twiddle<S>(k, p.N0));
    C<S> xk = E + WO;
    C<S> xh = conj(E - WO);
    if (p.flags & PF_SCALE) {
      xk = cscale(xk, sc);
      xh = cscale(xh, sc);
    }
    C<S>* line = out + (l0 + c) * P;
    line[k] = xk;
    if (h - k != k) line[h - k] = xh;
  }
}

// C2R, even N0 = 2h: Z[k] = (X[k] + conj X[h-k]) + i conj(W^k) (X[k] - conj
// X[h-k]) for k < h (imaginary parts of X[0] and X[h] ignored, as the
// reference's CPU and GPU routes do, src/cpu.rs:476-481), then an inverse
// FFT_h gives (x[2n], x[2n+1]) unnormalised.
template <class S>
__global__ void __launch_bounds__(512) k_c2r_even(const __grid_constant__ RealParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int PAD = PadOf<S>::value;
  C<S>* A = reinterpret_cast<C<S>*>(smem_raw);
  C<S>* B = A + p.G * p.LD;
  const uint32_t tid = threadIdx.x, T = blockDim.x;
  const uint32_t h = p.h, G = p.G, LD = p.LD, P = h + 1;
  const uint64_t l0 = (uint64_t)blockIdx.x * G;
  const uint32_t nvalid = (p.nlines - l0) < G ? (uint32_t)(p.nlines - l0) : G;
  const C<S>* __restrict__ in = (const C<S>*)p.in;
  for_each_elem_batched<4, C<S>>(
      P, p.dP, G, p.dG, false, tid, T,
      [&](uint32_t c, uint32_t k) { return c < nvalid ? in[(l0 + c) * P + k] : czero<S>(); },
      [&](uint32_t c, uint32_t k, C<S> v) {
        if (c < nvalid) A[c * LD + pidx<PAD>(k)] = v;
      });
  __syncthreads();
  {
    const uint32_t K = h / 2 + 1;
    const uint32_t tot = G * K;
    for (uint32_t e = tid; e < tot; e += T) {
      const uint32_t c = e / K, k = e - c * K;
      C<S> Xk = A[c * LD + pidx<PAD>(k)];
      C<S> Xh = A[c * LD + pidx<PAD>(h - k)];
      if (k == 0) {
        Xk.im = Scalar<S>::zero();
        Xh.im = Scalar<S>::zero();
      }
      const C<S> Pp = Xk + conj(Xh);
      const C<S> Q = Xk - conj(Xh);
      const C<S> iWQ = mul_i(cmulc(Q, twiddle<S>(k, p.N0)));  // i conj(W^k) Q
      // stored conjugated: the forward engine then computes the inverse
      B[c * LD + pidx<PAD>(k)] = conj(Pp + iWQ);
      if (k != 0 && h - k != k) B[c * LD + pidx<PAD>(h - k)] = Pp - iWQ;
    }
  }
  __syncthreads();
  const C<S>* y = fft_lines_smem<S>(B, A, p.sch, G, LD, tid, T,
                                     (p.flags & PF_TW_TABLE) ? (const C<S>*)p.tw : nullptr);
  C<S>* __restrict__ out = (C<S>*)p.out;
  const S sc = Scalar<S>::from_double(p.scale);
  for_each_elem(h, p.dh, G, p.dG, false, tid, T, [&](uint32_t c, uint32_t n) {
    if (c < nvalid) {
      C<S> v = conj(y[c * LD + pidx<PAD>(n)]);
      if (p.flags & PF_SCALE) v = cscale(v, sc);
      out[(l0 + c) * h + n] = v;
    }
  });
}

// R2C, odd N0: a complex FFT of the real line, first (N0+1)/2 outputs kept.
template <class S>
__global__ void __launch_bounds__(512) k_r2c_odd(const __grid_constant__ RealParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int PAD = PadOf<S>::value;
  C<S>* A = reinterpret_cast<C<S>*>(smem_raw);
  C<S>* B = A + p.G * p.LD;
  const uint32_t tid = threadIdx.x, T = blockDim.x;
  const uint32_t N0 = p.N0, G = p.G, LD = p.LD, P = N0 / 2 + 1;
  const uint64_t l0 = (uint64_t)blockIdx.x * G;
  const uint32_t nvalid = (p.nlines - l0) < G ? (uint32_t)(p.nlines - l0) : G;
  const S* __restrict__ in = (const S*)p.in;
  for_each_elem(N0, p.dN0, G, p.dG, false, tid, T, [&](uint32_t c, uint32_t n) {
    if (c < nvalid) A[c * LD + pidx<PAD>(n)] = {in[(l0 + c) * N0 + n], Scalar<S>::zero()};
  });
  __syncthreads();
  const C<S>* y = fft_lines_smem<S>(A, B, p.sch, G, LD, tid, T,
                                     (p.flags & PF_TW_TABLE) ? (const C<S>*)p.tw : nullptr);
  C<S>* __restrict__ out = (C<S>*)p.out;
  const S sc = Scalar<S>::from_double(p.scale);
  for_each_elem(P, p.dP, G, p.dG, false, tid, T, [&](uint32_t c, uint32_t k) {
    if (c < nvalid) {
      C<S> v = y[c * LD + pidx<PAD>(k)];
      if (p.flags & PF_SCALE) v = cscale(v, sc);
      out[(l0 + c) * P + k] = v;
    }
  });
}

// C2R, odd N0: the Hermitian line rebuilt in shared memory (imaginary part
// of X[0] ignored), an inverse complex FFT, the real part kept.
template <class S>
__global__ void __launch_bounds__(512) k_c2r_odd(const __grid_constant__ RealParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int PAD = PadOf<S>::value;
  C<S>* A = reinterpret_cast<C<S>*>(smem_raw);
  C<S>* B = A + p.G * p.LD;
  const uint32_t tid = threadIdx.x, T = blockDim.x;
  const uint32_t N0 = p.N0, G = p.G, LD = p.LD, P = N0 / 2 + 1;
  const uint64_t l0 = (uint64_t)blockIdx.x * G;
  const uint32_t nvalid = (p.nlines - l0) < G ? (uint32_t)(p.nlines - l0) : G;
  const C<S>* __restrict__ in = (const C<S>*)p.in;
  for_each_elem(P, p.dP, G, p.dG, false, tid, T, [&](uint32_t c, uint32_t k) {
    if (c < nvalid) {
      C<S> X = in[(l0 + c) * P + k];
      if (k == 0) X.im = Scalar<S>::zero();
      A[c * LD + pidx<PAD>(k)] = conj(X);  // conjugated input of the inverse
      if (k != 0) A[c * LD + pidx<PAD>(N0 - k)] = X;
    }
  });
  __syncthreads();
  const C<S>* y = fft_lines_smem<S>(A, B, p.sch, G, LD, tid, T,
                                     (p.flags & PF_TW_TABLE) ? (const C<S>*)p.tw : nullptr);
  S* __restrict__ out = (S*)p.out;
  const S sc = Scalar<S>::from_double(p.scale);
  for_each_elem(N0, p.dN0, G, p.dG, false, tid, T, [&](uint32_t c, uint32_t n) {
    if (c < nvalid) {
      S v = y[c * LD + pidx<PAD>(n)].re;
      if (p.flags & PF_SCALE) v = v * sc;
      out[(l0 + c) * N0 + n] = v;
    }
  });
}

// Elementwise passes walk (line, chunk) pairs: a block iteration covers
// kElemChunk consecutive points of one line, so one long line spreads over
// the whole grid and many short lines share it alike.
constexpr uint32_t kElemChunk = 2048;

template <class S>
__global__ void __launch_bounds__(256) k_blue_elem(const __grid_constant__ BlueElemParams p) {
  const uint32_t tid = threadIdx.x, T = blockDim.x;
  const uint32_t N = p.N, M = p.M;
  const S sc = Scalar<S>::from_double(p.scale);
  const C<S>* __restrict__ ctab = (const C<S>*)p.chirp;
  // points per line this pass writes
  const uint32_t L = (p.mode == BE_POST || p.mode == BE_RADER_POST) ? N : M;
  const uint64_t cpl = (L + kElemChunk - 1) / kElemChunk;
  for (uint64_t blk = blockIdx.x; blk < p.nlines * cpl; blk += gridDim.x) {
    const uint64_t l = blk / cpl;
    const uint32_t c0 = (uint32_t)(blk - l * cpl) * kElemChunk;
    const uint32_t c1 = c0 + kElemChunk < L ? c0 + kElemChunk : L;
    const uint64_t o = l / p.s, i = l - o * p.s;
    const int64_t base = (int64_t)(o * (uint64_t)N * p.s + i);
    if (p.mode == BE_PRE) {
      const C<S>* __restrict__ in = (const C<S>*)p.in;
      C<S>* __restrict__ ws = (C<S>*)p.out + l * M;
      for (uint32_t m = c0 + tid; m < c1; m += T) {
        C<S> v = czero<S>();
        if (m < N) {
          v = in[base + (int64_t)m * (int64_t)p.s];
          if (p.flags & PF_CONJ_IN) v.im = -v.im;
          v = cmul(v, ctab ? ctab[m] : chirp<S>(m, N));
        }
        ws[m] = v;
      }
    } else if (p.mode == BE_MID) {
      C<S>* ws = (C<S>*)p.out + l * M;
      const C<S>* __restrict__ bhat = (const C<S>*)p.bhat;
      for (uint32_t k = c0 + tid; k < c1; k += T) {
        C<S> v = cmul(ws[k], bhat[k]);
        v.im = -v.im;
        ws[k] = v;
      }
    } else if (p.mode == BE_RADER_PRE) {
      // a[q] = x[g^q] into the workspace line; x[0] kept
      const C<S>* __restrict__ in = (const C<S>*)p.in;
      C<S>* __restrict__ ws = (C<S>*)p.out + l * M;
      for (uint32_t q = c0 + tid; q < c1; q += T) {
        C<S> v = in[base + (int64_t)p.perm_in[q] * (int64_t)p.s];
        if (p.flags & PF_CONJ_IN) v.im = -v.im;
        ws[q] = v;
      }
      if (c0 == 0 && tid == 0) {
        C<S> v = in[base];
        if (p.flags & PF_CONJ_IN) v.im = -v.im;
        ((C<S>*)p.x0)[2 * l] = v;
      }
    } else if (p.mode == BE_RADER_MID) {
      // A = FFT(a): X[0] = x[0] + A[0] kept; then conj(A * bhat) in place
      // (the thread that reads A[0] is the one that overwrites it)
      C<S>* ws = (C<S>*)p.out + l * M;
      const C<S>* __restrict__ bhat = (const C<S>*)p.bhat;
      if (c0 == 0 && tid == 0) ((C<S>*)p.x0)[2 * l + 1] = ((C<S>*)p.x0)[2 * l] + ws[0];
      for (uint32_t m = c0 + tid; m < c1; m += T) {
        C<S> v = cmul(ws[m], bhat[m]);
        v.im = -v.im;
        ws[m] = v;
      }
    } else if (p.mode == BE_RADER_POST) {
      // X[n] = x[0] + conj(y[r(n)]) for n >= 1, X[0] kept
      const C<S>* __restrict__ ws = (const C<S>*)p.in + l * M;
      C<S>* __restrict__ out = (C<S>*)p.out;
      const C<S>* x0 = (const C<S>*)p.x0 + 2 * l;
      for (uint32_t n = c0 + tid; n < c1; n += T) {
        C<S> v;
        if (n == 0) {
          v = x0[1];
        } else {
          C<S> w = ws[p.perm_out[n - 1]];
          w.im = -w.im;
          v = x0[0] + w;
        }
        if (p.flags & PF_SCALE) v = cscale(v, sc);
        if (p.flags & PF_CONJ_OUT) v.im = -v.im;
        out[base + (int64_t)n * (int64_t)p.s] = v;
      }
    } else {
      const C<S>* __restrict__ ws = (const C<S>*)p.in + l * M;
      C<S>* __restrict__ out = (C<S>*)p.out;
      for (uint32_t k = c0 + tid; k < c1; k += T) {
        C<S> w = ws[k];
        w.im = -w.im;
        C<S> v = cmul(w, ctab ? ctab[k] : chirp<S>(k, N));
        if (p.flags & PF_SCALE) v = cscale(v, sc);
        if (p.flags & PF_CONJ_OUT) v.im = -v.im;
        out[base + (int64_t)k * (int64_t)p.s] = v;
      }
    }
  }
}

template <class S>
__global__ void __launch_bounds__(256) k_real_elem(const __grid_constant__ RealElemParams p) {
  const uint32_t tid = threadIdx.x, T = blockDim.x;
  const uint32_t N0 = p.N0, P = p.P;
  const uint32_t L = p.mode == RE_PACK ? P : N0;  // points per line this pass writes
  const uint64_t cpl = (L + kElemChunk - 1) / kElemChunk;
  for (uint64_t blk = blockIdx.x; blk < p.nlines * cpl; blk += gridDim.x) {
    const uint64_t l = blk / cpl;
    const uint32_t c0 = (uint32_t)(blk - l * cpl) * kElemChunk;
    const uint32_t c1 = c0 + kElemChunk < L ? c0 + kElemChunk : L;
    if (p.mode == RE_EXPAND) {
      const S* __restrict__ in = (const S*)p.in + l * N0;
      C<S>* __restrict__ out = (C<S>*)p.out + l * N0;
      for (uint32_t n = c0 + tid; n < c1; n += T) out[n] = {in[n], Scalar<S>::zero()};
    } else if (p.mode == RE_PACK) {
      const C<S>* __restrict__ in = (const C<S>*)p.in + l * N0;
      C<S>* __restrict__ out = (C<S>*)p.out + l * P;
      for (uint32_t k = c0 + tid; k < c1; k += T) out[k] = in[k];
    } else if (p.mode == RE_UNPACK) {
      const C<S>* __restrict__ in = (const C<S>*)p.in + l * P;
      C<S>* __restrict__ out = (C<S>*)p.out + l * N0;
      for (uint32_t k = c0 + tid; k < c1; k += T) {
        // X[k] for k < P; X[N0-k] = conj(X[k]) above; DC and Nyquist real
        C<S> v = (k < P) ? in[k] : conj(in[N0 - k]);
        if (k == 0 || 2 * k == N0) v.im = Scalar<S>::zero();
        out[k] = v;
      }
    } else {
      const C<S>* __restrict__ in = (const C<S>*)p.in + l * N0;
      S* __restrict__ out = (S*)p.out + l * N0;
      for (uint32_t n = c0 + tid; n < c1; n += T) out[n] = in[n].re;
    }
  }
}

template <class S>
__global__ void k_scale_copy(const C<S>* __restrict__ in, C<S>* __restrict__ out, uint64_t n,
                             double scale, int conj_flag) {
  const S sc = Scalar<S>::from_double(scale);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    C<S> v = cscale(in[i], sc);
    if (conj_flag) v.im = -v.im;
    out[i] = v;
  }
}

// ----------------------------------------------------------- small volume
// One CTA per volume (src/runtime/small_volume.rs:1-42): the volume sits in
// shared memory in its natural order; axis a's lines (outer o, inner c <
// stride, point i at o*N*stride + i*stride + c) are gathered into the work
// buffer at line l = o*stride + c, pitch LD, transformed by the Stockham
// engine and scattered back, so the volume crosses HBM once.
template <class S>
__global__ void __launch_bounds__(256) k_small_volume(const __grid_constant__ SmallVolumeParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int PAD = PadOf<S>::value;
  C<S>* vol = reinterpret_cast<C<S>*>(smem_raw);
  C<S>* A = vol + p.V;
  C<S>* B = A + p.buf;
  const uint32_t tid = threadIdx.x, T = blockDim.x, V = p.V;
  const uint64_t base = (uint64_t)blockIdx.x * V;
  const C<S>* __restrict__ in = (const C<S>*)p.in;
  const bool conj_in = p.flags & PF_CONJ_IN;
  for (uint32_t e = tid; e < V; e += T) {
    C<S> v = in[base + e];
    if (conj_in) v.im = -v.im;
    vol[e] = v;
  }
  __syncthreads();
  const C<S>* tw = (p.flags & PF_TW_TABLE) ? (const C<S>*)p.tw : nullptr;
#pragma unroll 1
  for (uint32_t a = 0; a < p.rank; ++a) {
    const uint32_t N = p.dims[a], s = p.strides[a], LD = p.LD[a];
    const uint32_t lines = V / N;
    // element e of the volume = (o, i, c): l = o*s + c
    for (uint32_t e = tid; e < V; e += T) {
      const uint32_t oi = fdiv(e, p.dS[a]), c = e - oi * s;
      const uint32_t o = fdiv(oi, p.dN[a]), i = oi - o * N;
      A[(o * s + c) * LD + pidx<PAD>(i)] = vol[e];
    }
    __syncthreads();
    const C<S>* r = fft_lines_smem<S>(A, B, p.sch[a], lines, LD, tid, T, tw);
    for (uint32_t e = tid; e < V; e += T) {
      const uint32_t oi = fdiv(e, p.dS[a]), c = e - oi * s;
      const uint32_t o = fdiv(oi, p.dN[a]), i = oi - o * N;
      vol[e] = r[(o * s + c) * LD + pidx<PAD>(i)];
    }
    __syncthreads();
  }
  C<S>* __restrict__ out = (C<S>*)p.out;
  const S sc = Scalar<S>::from_double(p.scale);
  for (uint32_t e = tid; e < V; e += T) {
    C<S> v = vol[e];
    if (p.flags & PF_SCALE) v = cscale(v, sc);
    if (p.flags & PF_CONJ_OUT) v.im = -v.im;
    out[base + e] = v;
  }
}

// --------------------------------------------------- templated launchers
// Raises the dynamic shared memory limit of a kernel once per (kernel,
// device); kernels are told apart by address, not by type.
template <class K>
static cudaError_t prepare(K kernel, size_t smem) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const std::pair<const void*, int> key((const void*)kernel, dev);
  std::lock_guard<std::mutex> lk(mu);
  if (done.count(key)) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)max_smem_per_block());
  if (e == cudaSuccess) done.insert(key);
  return e;
}

template <class K, class P>
static cudaError_t launch(K kernel, const P& prm, unsigned grid, unsigned threads, size_t smem,
                          cudaStream_t st) {
  cudaError_t e = prepare(kernel, smem);
  if (e != cudaSuccess) return e;
  kernel<<<grid, threads, smem, st>>>(prm);
  return cudaGetLastError();
}

template <class S>
cudaError_t launch_small_volume_t(const SmallVolumeParams& prm, unsigned threads, size_t smem,
                                  cudaStream_t st) {
  return launch(k_small_volume<S>, prm, (unsigned)prm.nvol, threads, smem, st);
}
template <class S>
cudaError_t launch_lines_t(const LinesParams& prm, unsigned grid, unsigned threads, size_t smem,
                           cudaStream_t st) {
  return launch(k_lines<S>, prm, grid, threads, smem, st);
}
template <class S>
cudaError_t launch_rader_t(const RaderParams& prm, unsigned grid, unsigned threads, size_t smem,
                           cudaStream_t st) {
  return launch(k_rader<S>, prm, grid, threads, smem, st);
}
template <class S>
cudaError_t launch_bluestein_t(const BluesteinParams& prm, unsigned grid, unsigned threads,
                               size_t smem, cudaStream_t st) {
  return launch(k_bluestein<S>, prm, grid, threads, smem, st);
}
template <class S>
cudaError_t launch_r2c_t(const RealParams& prm, unsigned grid, unsigned threads, size_t smem,
                         cudaStream_t st) {
  if (prm.N0 % 2 == 0) return launch(k_r2c_even<S>, prm, grid, threads, smem, st);
  return launch(k_r2c_odd<S>, prm, grid, threads, smem, st);
}
template <class S>
cudaError_t launch_c2r_t(const RealParams& prm, unsigned grid, unsigned threads, size_t smem,
                         cudaStream_t st) {
  if (prm.N0 % 2 == 0) return launch(k_c2r_even<S>, prm, grid, threads, smem, st);
  return launch(k_c2r_odd<S>, prm, grid, threads, smem, st);
}
template <class S>
cudaError_t launch_blue_elem_t(const BlueElemParams& prm, cudaStream_t st) {
  const uint64_t L = (prm.mode == BE_POST || prm.mode == BE_RADER_POST) ? prm.N : prm.M;
  const uint64_t work = prm.nlines * ((L + kElemChunk - 1) / kElemChunk);
  uint64_t blocks = work < 148ull * 16 ? work : 148ull * 16;
  if (blocks == 0) blocks = 1;
  k_blue_elem<S><<<(unsigned)blocks, 256, 0, st>>>(prm);
  return cudaGetLastError();
}

template <class S>
cudaError_t launch_real_elem_t(const RealElemParams& prm, cudaStream_t st) {
  const uint64_t L = prm.mode == RE_PACK ? prm.P : prm.N0;
  const uint64_t work = prm.nlines * ((L + kElemChunk - 1) / kElemChunk);
  uint64_t blocks = work < 148ull * 16 ? work : 148ull * 16;
  if (blocks == 0) blocks = 1;
  k_real_elem<S><<<(unsigned)blocks, 256, 0, st>>>(prm);
  return cudaGetLastError();
}

template <class S>
cudaError_t launch_scale_copy_t(const void* in, void* out, uint64_t n, double scale, bool conj,
                                cudaStream_t st) {
  const unsigned threads = 256;
  uint64_t blocks = (n + threads - 1) / threads;
  if (blocks > 148ull * 32) blocks = 148ull * 32;
  if (blocks == 0) blocks = 1;
  k_scale_copy<S><<<(unsigned)blocks, threads, 0, st>>>((const C<S>*)in, (C<S>*)out, n, scale,
                                                        conj ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace b2f
