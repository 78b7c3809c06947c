// Register-resident power-of-two line kernel with the line length fixed at
// compile time (f32, f64 and df64, N = 2^LOGN, 16 <= N <= 8192).
//
// The same algorithm as k_pow2 (regfft.cuh): E values a thread in
// registers, radix-16 stages then one radix 2, 4 or 8 stage, exchanges
// through shared memory in autosorted order, first-stage loads straight
// from HBM and last-stage stores straight back.  With N known, every stride
// of the schedule is a constant: the shared-memory exchanges and the
// contiguous loads and stores address value q of a butterfly as a fixed
// offset from one per-thread base (the pad of one slot per 16 values,
// i + (i >> 4), splits across the sum because every stride is a multiple
// of 16 and the first stage's bases are), the twiddle offsets are
// constants, and the stage loop unrolls.  The
// generic kernel recomputes those addresses per value from runtime strides
// (about a third of its instructions are integer addressing).
#pragma once
#include <type_traits>

#include "regfft.cuh"

namespace b2f {

// Pad shift of the power-of-two kernels' lines, every precision (the
// planner sizes a line as LD = N + N/16 + 1, as for the generic kernel).
constexpr int kPow2Pad = 4;

template <int LOGN>
struct P2Sched {
  static constexpr int N = 1 << LOGN;
  static constexpr int NST = (LOGN + 3) / 4;
  static constexpr int R(int s) { return s < LOGN / 4 ? 16 : (1 << (LOGN % 4)); }
  static constexpr int NS(int s) { return s == 0 ? 1 : NS(s - 1) * R(s - 1); }
  static constexpr int NR(int s) { return N / R(s); }
  // first twiddle of stage s in the plan table: stage i holds NS(i)*(R(i)-1)
  static constexpr int TW(int s) { return s == 0 ? 0 : TW(s - 1) + NS(s - 1) * (R(s - 1) - 1); }
};

// Offset of value b + x from the slot of b in a padded line (pidx<PAD>), for
// x a multiple of 2^PAD or b a multiple of 2^PAD with x < 16.
template <int PAD>
FFT_HD constexpr uint32_t fx_off(uint32_t x) { return x + (x >> PAD); }

// Stage s on the E register values: twiddles W_{NS R}^{q k} (k = j mod NS)
// from the plan table or computed, then the radix-R codelet.
template <class S, int LOGN, int s, int E>
FFT_D void fx_compute(cpx<S> (&v)[E], uint32_t t, const cpx<S>* __restrict__ tw) {
  using P = P2Sched<LOGN>;
  constexpr int R = P::R(s), NS = P::NS(s), NB = E / R, TL = P::N / E;
  if constexpr (NS > 1) {
#pragma unroll
    for (int u = 0; u < NB; ++u) {
      const uint32_t k = (t + u * TL) & (NS - 1);
      if (tw != nullptr) {
        const cpx<S>* tr = tw + P::TW(s) + k * (R - 1);
#pragma unroll
        for (int q = 1; q < R; ++q) v[u * R + q] = cmul(v[u * R + q], tr[q - 1]);
      } else {
        apply_stage_twiddles<S, R>(v + u * R, k, NS * R);
      }
    }
  }
#pragma unroll
  for (int u = 0; u < NB; ++u) dft<S, R>(v + u * R);
}

// Stage s's outputs into the line's shared buffer: output o + r*NS of
// butterfly j (o = (j - k) R + k).  NS is 1 (stage 0, R = 16: o is a
// multiple of 16) or a multiple of 16, so pad(o + r NS) = pad(o) + fx_off(r NS).
template <class S, int LOGN, int s, int E>
FFT_D void fx_write(const cpx<S> (&v)[E], cpx<S>* line, uint32_t t) {
  using P = P2Sched<LOGN>;
  constexpr int PAD = kPow2Pad;
  constexpr int R = P::R(s), NS = P::NS(s), NB = E / R, TL = P::N / E;
  static_assert(NS == 1 ? R == 16 : NS % 16 == 0, "separable padding");
#pragma unroll
  for (int u = 0; u < NB; ++u) {
    const uint32_t j = t + u * TL, k = j & (NS - 1);
    cpx<S>* d = line + pidx<PAD>((j - k) * R + k);
#pragma unroll
    for (int r = 0; r < R; ++r) d[fx_off<PAD>(r * NS)] = v[u * R + r];
  }
}

// Stage s's inputs from the line's shared buffer: value j + q*NR, NR a
// multiple of 16 for every stage after the first.
template <class S, int LOGN, int s, int E>
FFT_D void fx_read(cpx<S> (&v)[E], const cpx<S>* line, uint32_t t) {
  using P = P2Sched<LOGN>;
  constexpr int PAD = kPow2Pad;
  constexpr int R = P::R(s), NR = P::NR(s), NB = E / R, TL = P::N / E;
  static_assert(NR % 16 == 0, "separable padding");
#pragma unroll
  for (int u = 0; u < NB; ++u) {
    const cpx<S>* b = line + pidx<PAD>(t + u * TL);
#pragma unroll
    for (int q = 0; q < R; ++q) v[u * R + q] = b[fx_off<PAD>(q * NR)];
  }
}

// Stages s.. of the line (barriers between the exchanges), then the
// caller's store.
template <class S, int LOGN, int s, int E>
FFT_D void fx_stages(cpx<S> (&v)[E], cpx<S>* line, uint32_t t, const cpx<S>* __restrict__ tw) {
  using P = P2Sched<LOGN>;
  fx_compute<S, LOGN, s, E>(v, t, tw);
  if constexpr (s + 1 < P::NST) {
    fx_write<S, LOGN, s, E>(v, line, t);
    __syncthreads();
    fx_read<S, LOGN, s + 1, E>(v, line, t);
    __syncthreads();
    fx_stages<S, LOGN, s + 1, E>(v, line, t, tw);
  }
}

// G lines of N = 2^LOGN points; blockDim = G * N / E (256 for 16-value
// column tiles, up to 512 otherwise).  Shared memory: G * LD values,
// LD = N + N/16 + 1.  f32 register budgets: 64 for contiguous lines (4
// CTAs of 256 threads per SM), 85 for 16-value column tiles (3 per SM), 128
// for 32-value ones; f64 and df64: 128 (256 threads, 2 per SM).
template <class S, int E, bool COLMAJOR>
struct FxBounds {
  static constexpr bool wide = !std::is_same<S, float>::value;  // f64, df64
  static constexpr int threads = wide || (COLMAJOR && E == 16) ? 256 : 512;
  static constexpr int blocks = wide ? 2 : (COLMAJOR ? (E == 16 ? 3 : 1) : 2);
};
template <class S, int E, bool COLMAJOR, int LOGN>
__global__ void __launch_bounds__(FxBounds<S, E, COLMAJOR>::threads, FxBounds<S, E, COLMAJOR>::blocks)
    k_pow2_fx(const __grid_constant__ LinesParams p) {
  using P = P2Sched<LOGN>;
  using C = cpx<S>;
  constexpr int PAD = kPow2Pad;
  constexpr int N = P::N, TL = N / E, LAST = P::NST - 1;
  constexpr int R0 = P::R(0), NR0 = P::NR(0), RL = P::R(LAST), NSL = P::NS(LAST);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  const uint32_t tid = threadIdx.x;
  const uint32_t G = p.G, LD = p.LD;
  uint32_t c, t;
  if (COLMAJOR) {
    c = tid & (G - 1);
    t = tid >> (31 - __clz(G));
  } else {
    t = tid & (TL - 1);
    c = tid >> (31 - __clz(TL));
  }
  const Group g = group_of(p.io, G, blockIdx.x);
  const bool valid = c < g.nvalid;
  const C* tw = (p.flags & PF_TW_TABLE) ? (const C*)p.tw : nullptr;
  C v[E];
  // first stage: value t + u*TL + q*NR0 of line c straight from HBM
  if (valid) {
    const C* __restrict__ src = (const C*)p.in + g.in0 + (int64_t)c * g.dl_in;
    const int64_t es = COLMAJOR ? p.io.in_es : 1;
#pragma unroll
    for (int u = 0; u < E / R0; ++u) {
      const C* b = src + (int64_t)(t + u * TL) * es;
#pragma unroll
      for (int q = 0; q < R0; ++q) v[u * R0 + q] = b[(int64_t)q * NR0 * es];
    }
    if (p.flags & PF_CONJ_IN) {
#pragma unroll
      for (int i = 0; i < E; ++i) v[i].im = -v[i].im;
    }
  } else {
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = czero<S>();
  }
  C* line = sm + c * LD;
  fx_stages<S, LOGN, 0, E>(v, line, t, tw);
  const S sc = Scalar<S>::from_double(p.scale);
  const uint32_t fl = p.flags;
  if (!(fl & PF_STORE_SMEM)) {
    // last stage: output n = j + r*NSL (j < NSL) straight to HBM
    if (!valid) return;
    C* __restrict__ dst = (C*)p.out + g.out0 + (int64_t)c * g.dl_out;
    const int64_t es = COLMAJOR ? p.io.out_es : 1;
    const uint64_t row = (fl & PF_TW_STORE) ? fdiv((uint32_t)(g.c0 + c), p.d_tw) : 0;
    const C* __restrict__ ta = (const C*)p.tws_a;
    const C* __restrict__ tb = (const C*)p.tws_b;
    // twiddle W_M^{row n} (row n < M): from the power-of-two-split tables
    // with a 32-bit exponent stepped by row * NSL per output when M < 2^32
    const bool step_tw = ta != nullptr && p.d_tws.mul == 0 && p.tw_store_M <= 0xFFFFFFFFull;
    const uint32_t sh = p.d_tws.shift, msk = (1u << sh) - 1;
#pragma unroll
    for (int u = 0; u < E / RL; ++u) {
      const uint32_t j = t + u * TL;
      C* b = dst + (int64_t)j * es;
      uint32_t m32 = (uint32_t)row * j;
      const uint32_t dm = (uint32_t)row * NSL;
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        C x = v[u * RL + r];
        if (fl & PF_TW_STORE) {
          if (step_tw) {
            x = cmul(x, cmul(ta[m32 >> sh], tb[m32 & msk]));
            m32 += dm;
          } else {
            const uint64_t m = row * (uint64_t)(j + r * NSL);
            x = cmul(x, ta ? tw_two_level(ta, tb, m, p.d_tws) : twiddle<S>(m % p.tw_store_M, p.tw_store_M));
          }
        }
        if (fl & PF_SCALE) x = cscale(x, sc);
        if (fl & PF_CONJ_OUT) x.im = -x.im;
        b[(int64_t)r * NSL * es] = x;
      }
    }
    return;
  }
  // the output order wants adjacent lines first: one pass through shared
  // memory (last stage's outputs in natural order, then lines first)
#pragma unroll
  for (int u = 0; u < E / RL; ++u) {
    const uint32_t j = t + u * TL;
#pragma unroll
    for (int r = 0; r < RL; ++r) line[pidx<PAD>(j + r * NSL)] = v[u * RL + r];
  }
  __syncthreads();
  C* __restrict__ out = (C*)p.out;
  const uint32_t T = blockDim.x;
  for_each_elem(N, p.dN, G, p.dG, true, tid, T, [&](uint32_t cc, uint32_t n) {
    if (cc < g.nvalid) {
      C x = sm[cc * LD + pidx<PAD>(n)];
      if (fl & PF_TW_STORE) {
        const uint64_t row = fdiv((uint32_t)(g.c0 + cc), p.d_tw);
        const uint64_t m = row * (uint64_t)n;
        x = cmul(x, p.tws_a ? tw_two_level((const C*)p.tws_a, (const C*)p.tws_b, m, p.d_tws)
                            : twiddle<S>(m % p.tw_store_M, p.tw_store_M));
      }
      if (fl & PF_SCALE) x = cscale(x, sc);
      if (fl & PF_CONJ_OUT) x.im = -x.im;
      out[g.out0 + (int64_t)cc * g.dl_out + (int64_t)n * p.io.out_es] = x;
    }
  });
}

}  // namespace b2f

namespace b2f {

// Real transforms of even length N0 = 2h, h = 2^LOGH (16 <= h <= 4096),
// lines contiguous: the h-point complex FFT of the packed pairs runs in the
// fixed-length register kernel; G = blockDim / (h/16) lines per CTA, one
// shared-memory buffer of G * LD values (exchanges and the pre/post
// processing, which pairs k with h - k).  rtw: W_N0^k for k < h, built in
// FP64 and rounded once.
template <class S>
struct FxRealBounds {
  static constexpr int blocks = sizeof(S) == 8 ? 2 : 3;
};

// R2C: z[n] = x[2n] + i x[2n+1], Z = FFT_h(z), then for k <= h/2:
// X[k] = E + W^k O and X[h-k] = conj(E - W^k O), E = (Z[k] + conj Z[h-k])/2,
// O = -i (Z[k] - conj Z[h-k])/2, into the packed line of h + 1 values.
template <class S, int LOGH>
__global__ void __launch_bounds__(256, FxRealBounds<S>::blocks)
    k_r2c_fx(const __grid_constant__ RealParams p) {
  using P = P2Sched<LOGH>;
  using C = cpx<S>;
  constexpr int E = 16, PAD = kPow2Pad, H = P::N, TL = H / E, LAST = P::NST - 1;
  constexpr int NR0 = P::NR(0), RL = P::R(LAST), NSL = P::NS(LAST);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  const uint32_t tid = threadIdx.x, G = p.G, LD = p.LD;
  const uint32_t t = tid & (TL - 1), c = tid >> (31 - __clz(TL));
  const uint64_t l0 = (uint64_t)blockIdx.x * G;
  const bool valid = l0 + c < p.nlines;
  C v[E];
  if (valid) {
    const C* __restrict__ src = (const C*)p.in + (l0 + c) * H + t;
#pragma unroll
    for (int q = 0; q < E; ++q) v[q] = src[q * NR0];
  } else {
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = czero<S>();
  }
  C* line = sm + c * LD;
  fx_stages<S, LOGH, 0, E>(v, line, t, (p.flags & PF_TW_TABLE) ? (const C*)p.tw : nullptr);
  // Z in natural order (the last exchange's reads ended with a barrier)
#pragma unroll
  for (int u = 0; u < E / RL; ++u) {
    const uint32_t j = t + u * TL;
#pragma unroll
    for (int r = 0; r < RL; ++r) line[pidx<PAD>(j + r * NSL)] = v[u * RL + r];
  }
  __syncthreads();
  if (!valid) return;
  const C* __restrict__ rtw = (const C*)p.rtw;
  const S half = Scalar<S>::from_double(0.5);
  const S sc = Scalar<S>::from_double(p.scale);
  C* __restrict__ out = (C*)p.out + (l0 + c) * (H + 1);
  for (uint32_t k = t; k <= H / 2; k += TL) {
    const C a = line[pidx<PAD>(k)];
    const C b = conj(line[pidx<PAD>(k == 0 ? 0 : H - k)]);
    const C Ev = cscale(a + b, half);
    const C Ov = cscale(mul_neg_i(a - b), half);
    const C WO = cmul(Ov, rtw[k]);
    C xk = Ev + WO;
    C xh = conj(Ev - WO);
    if (p.flags & PF_SCALE) {
      xk = cscale(xk, sc);
      xh = cscale(xh, sc);
    }
    out[k] = xk;
    if (H - k != k) out[H - k] = xh;
  }
}

// C2R: Z[n] = conj(P + i conj(W^n) Q), P = X[n] + conj X[h-n], Q = X[n] -
// conj X[h-n] (imaginary parts of X[0] and X[h] ignored), for every n < h,
// built straight into the first stage's registers; the forward FFT of the
// conjugate, conjugated, gives (x[2n], x[2n+1]).
template <class S, int LOGH>
__global__ void __launch_bounds__(256, FxRealBounds<S>::blocks)
    k_c2r_fx(const __grid_constant__ RealParams p) {
  using P = P2Sched<LOGH>;
  using C = cpx<S>;
  constexpr int E = 16, PAD = kPow2Pad, H = P::N, TL = H / E, LAST = P::NST - 1;
  constexpr int NR0 = P::NR(0), RL = P::R(LAST), NSL = P::NS(LAST);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  const uint32_t tid = threadIdx.x, G = p.G, LD = p.LD;
  const uint32_t t = tid & (TL - 1), c = tid >> (31 - __clz(TL));
  const uint64_t l0 = (uint64_t)blockIdx.x * G;
  const bool valid = l0 + c < p.nlines;
  C* line = sm + c * LD;
  if (valid) {
    // the packed line (h + 1 values): all of a thread's loads issued before
    // its first shared-memory store, so they overlap
    const C* __restrict__ src = (const C*)p.in + (l0 + c) * (H + 1);
    C x[E];
#pragma unroll
    for (int i = 0; i < E; ++i) x[i] = src[t + i * TL];
    const C xh = t == 0 ? src[H] : czero<S>();
#pragma unroll
    for (int i = 0; i < E; ++i) line[pidx<PAD>(t + i * TL)] = x[i];
    if (t == 0) line[pidx<PAD>(H)] = xh;
  }
  __syncthreads();
  const C* __restrict__ rtw = (const C*)p.rtw;
  C v[E];
  if (valid) {
#pragma unroll
    for (int q = 0; q < E; ++q) {
      const uint32_t n = t + q * NR0;
      C Xk = line[pidx<PAD>(n)];
      C Xh = line[pidx<PAD>(H - n)];
      if (n == 0) {
        Xk.im = Scalar<S>::zero();
        Xh.im = Scalar<S>::zero();
      }
      const C Pp = Xk + conj(Xh);
      const C Q = Xk - conj(Xh);
      v[q] = conj(Pp + mul_i(cmulc(Q, rtw[n])));
    }
  } else {
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = czero<S>();
  }
  __syncthreads();  // every X read before the exchanges reuse the buffer
  fx_stages<S, LOGH, 0, E>(v, line, t, (p.flags & PF_TW_TABLE) ? (const C*)p.tw : nullptr);
  if (!valid) return;
  const S sc = Scalar<S>::from_double(p.scale);
  C* __restrict__ out = (C*)p.out + (l0 + c) * H;
#pragma unroll
  for (int u = 0; u < E / RL; ++u) {
    const uint32_t j = t + u * TL;
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      C x = conj(v[u * RL + r]);
      if (p.flags & PF_SCALE) x = cscale(x, sc);
      out[j + r * NSL] = x;
    }
  }
}

}  // namespace b2f
