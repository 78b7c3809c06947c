// Register-resident power-of-two line kernel with the line length fixed at
// compile time (f32, N = 2^LOGN, 16 <= N <= 8192).
//
// The same algorithm as k_pow2 (regfft.cuh): E values a thread in
// registers, radix-16 stages then one radix 2, 4 or 8 stage, exchanges
// through shared memory in autosorted order, first-stage loads straight
// from HBM and last-stage stores straight back.  With N known, every stride
// of the schedule is a constant: the shared-memory exchanges and the
// contiguous loads and stores address value q of a butterfly as a fixed
// offset from one per-thread base (the pad of one slot per 16 values,
// i + i/16, splits across the sum because every stride is a multiple of
// 16), the twiddle offsets are constants, and the stage loop unrolls.  The
// generic kernel recomputes those addresses per value from runtime strides
// (about a third of its instructions are integer addressing).
#pragma once
#include "regfft.cuh"

namespace b2f {

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

// Slot of value i in a padded line (pidx<4>).
FFT_HD constexpr uint32_t fx_pad(uint32_t i) { return i + (i >> 4); }

// Stage s on the E register values: twiddles W_{NS R}^{q k} (k = j mod NS)
// from the plan table or computed, then the radix-R codelet.
template <int LOGN, int s, int E>
FFT_D void fx_compute(cpx<float> (&v)[E], uint32_t t, const cpx<float>* __restrict__ tw) {
  using P = P2Sched<LOGN>;
  constexpr int R = P::R(s), NS = P::NS(s), NB = E / R, TL = P::N / E;
  if constexpr (NS > 1) {
#pragma unroll
    for (int u = 0; u < NB; ++u) {
      const uint32_t k = (t + u * TL) & (NS - 1);
      if (tw != nullptr) {
        const cpx<float>* tr = tw + P::TW(s) + k * (R - 1);
#pragma unroll
        for (int q = 1; q < R; ++q) v[u * R + q] = cmul(v[u * R + q], tr[q - 1]);
      } else {
        apply_stage_twiddles<float, R>(v + u * R, k, NS * R);
      }
    }
  }
#pragma unroll
  for (int u = 0; u < NB; ++u) dft<float, R>(v + u * R);
}

// Stage s's outputs into the line's shared buffer: output o + r*NS of
// butterfly j (o = (j - k) R + k).  NS is 1 (stage 0, R = 16: o is a
// multiple of 16) or a multiple of 16, so pad(o + r NS) = pad(o) + r pad-stride.
template <int LOGN, int s, int E>
FFT_D void fx_write(const cpx<float> (&v)[E], cpx<float>* line, uint32_t t) {
  using P = P2Sched<LOGN>;
  constexpr int R = P::R(s), NS = P::NS(s), NB = E / R, TL = P::N / E;
  constexpr uint32_t step = NS == 1 ? 1 : NS + NS / 16;
  static_assert(NS == 1 ? R == 16 : NS % 16 == 0, "separable padding");
#pragma unroll
  for (int u = 0; u < NB; ++u) {
    const uint32_t j = t + u * TL, k = j & (NS - 1);
    cpx<float>* d = line + fx_pad((j - k) * R + k);
#pragma unroll
    for (int r = 0; r < R; ++r) d[r * step] = v[u * R + r];
  }
}

// Stage s's inputs from the line's shared buffer: value j + q*NR, NR a
// multiple of 16 for every stage after the first.
template <int LOGN, int s, int E>
FFT_D void fx_read(cpx<float> (&v)[E], const cpx<float>* line, uint32_t t) {
  using P = P2Sched<LOGN>;
  constexpr int R = P::R(s), NR = P::NR(s), NB = E / R, TL = P::N / E;
  static_assert(NR % 16 == 0, "separable padding");
  constexpr uint32_t step = NR + NR / 16;
#pragma unroll
  for (int u = 0; u < NB; ++u) {
    const cpx<float>* b = line + fx_pad(t + u * TL);
#pragma unroll
    for (int q = 0; q < R; ++q) v[u * R + q] = b[q * step];
  }
}

// Stages s.. of the line (barriers between the exchanges), then the
// caller's store.
template <int LOGN, int s, int E>
FFT_D void fx_stages(cpx<float> (&v)[E], cpx<float>* line, uint32_t t,
                     const cpx<float>* __restrict__ tw) {
  using P = P2Sched<LOGN>;
  fx_compute<LOGN, s, E>(v, t, tw);
  if constexpr (s + 1 < P::NST) {
    fx_write<LOGN, s, E>(v, line, t);
    __syncthreads();
    fx_read<LOGN, s + 1, E>(v, line, t);
    __syncthreads();
    fx_stages<LOGN, s + 1, E>(v, line, t, tw);
  }
}

// G lines of N = 2^LOGN points; blockDim = G * N / E (256 for 16-value
// column tiles, up to 512 otherwise).  Shared memory: G * LD values,
// LD = N + N/16 + 1.  Register budgets: 64 for contiguous lines (4 CTAs of
// 256 threads per SM), 85 for 16-value column tiles (3 per SM), 128 for
// 32-value ones.
template <int E, bool COLMAJOR, int LOGN>
__global__ void __launch_bounds__(COLMAJOR && E == 16 ? 256 : 512,
                                  COLMAJOR ? (E == 16 ? 3 : 1) : 2)
    k_pow2_fx(const __grid_constant__ LinesParams p) {
  using P = P2Sched<LOGN>;
  using C = cpx<float>;
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
    for (int i = 0; i < E; ++i) v[i] = czero<float>();
  }
  C* line = sm + c * LD;
  fx_stages<LOGN, 0, E>(v, line, t, tw);
  const float sc = (float)p.scale;
  const uint32_t fl = p.flags;
  if (!(fl & PF_STORE_SMEM)) {
    // last stage: output n = j + r*NSL (j < NSL) straight to HBM
    if (!valid) return;
    C* __restrict__ dst = (C*)p.out + g.out0 + (int64_t)c * g.dl_out;
    const int64_t es = COLMAJOR ? p.io.out_es : 1;
    const uint64_t row = (fl & PF_TW_STORE) ? fdiv((uint32_t)(g.c0 + c), p.d_tw) : 0;
    const C* __restrict__ ta = (const C*)p.tws_a;
    const C* __restrict__ tb = (const C*)p.tws_b;
#pragma unroll
    for (int u = 0; u < E / RL; ++u) {
      const uint32_t j = t + u * TL;
      C* b = dst + (int64_t)j * es;
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        C x = v[u * RL + r];
        if (fl & PF_TW_STORE) {
          const uint64_t m = row * (uint64_t)(j + r * NSL);
          x = cmul(x, ta ? tw_two_level(ta, tb, m, p.d_tws) : twiddle<float>(m % p.tw_store_M, p.tw_store_M));
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
    for (int r = 0; r < RL; ++r) line[fx_pad(j + r * NSL)] = v[u * RL + r];
  }
  __syncthreads();
  C* __restrict__ out = (C*)p.out;
  const uint32_t T = blockDim.x;
  for_each_elem(N, p.dN, G, p.dG, true, tid, T, [&](uint32_t cc, uint32_t n) {
    if (cc < g.nvalid) {
      C x = sm[cc * LD + fx_pad(n)];
      if (fl & PF_TW_STORE) {
        const uint64_t row = fdiv((uint32_t)(g.c0 + cc), p.d_tw);
        const uint64_t m = row * (uint64_t)n;
        x = cmul(x, p.tws_a ? tw_two_level((const C*)p.tws_a, (const C*)p.tws_b, m, p.d_tws)
                            : twiddle<float>(m % p.tw_store_M, p.tw_store_M));
      }
      if (fl & PF_SCALE) x = cscale(x, sc);
      if (fl & PF_CONJ_OUT) x.im = -x.im;
      out[g.out0 + (int64_t)cc * g.dl_out + (int64_t)n * p.io.out_es] = x;
    }
  });
}

}  // namespace b2f
