// Register-resident power-of-two line kernel.
//
// Each thread keeps E values of its line in registers through every stage.
// The first stage's inputs come straight from HBM (E independent loads in
// flight per thread) and the last stage's outputs go straight back (or, when
// the output layout wants another thread order, through one shared-memory
// pass); between stages the values are exchanged through shared memory in
// their autosorted (Stockham) order.  Radix-16 stages, then one radix 2, 4, 8
// or 16 stage.  This replaces the reference's register-resident kernels
// (src/runtime/register_fft.rs:136-360) and its split passes.
//
// Thread layout: TL = N/E threads per line.  Line-major (t fastest) when a
// line's points are contiguous in memory; column-major (line fastest) for
// tiles of adjacent columns, so that a warp always touches consecutive
// addresses.
#pragma once
#include "kernels_impl.cuh"

namespace b2f {

// One stage of radix R on the E register values of a thread.
template <class S, int R, int E>
FFT_D void reg_stage_compute(C<S> (&v)[E], uint32_t t, uint32_t TL, uint32_t Ns,
                             const C<S>* __restrict__ tw, uint32_t tw_off) {
  constexpr int NB = E / R;
  if (Ns > 1) {
    const uint32_t M = Ns * R;
#pragma unroll
    for (int u = 0; u < NB; ++u) {
      const uint32_t j = t + u * TL;
      const uint32_t k = j & (Ns - 1);
      if (tw != nullptr) {
        const C<S>* tr = tw + tw_off + k * (R - 1);
#pragma unroll
        for (int q = 1; q < R; ++q) v[u * R + q] = cmul(v[u * R + q], tr[q - 1]);
      } else {
        apply_stage_twiddles<S, R>(v + u * R, k, M);
      }
    }
  }
#pragma unroll
  for (int u = 0; u < NB; ++u) dft<S, R>(v + u * R);
}

template <class S, int R, int E, int PAD>
FFT_D void reg_stage_write(const C<S> (&v)[E], C<S>* line, uint32_t t, uint32_t TL, uint32_t Ns) {
  constexpr int NB = E / R;
#pragma unroll
  for (int u = 0; u < NB; ++u) {
    const uint32_t j = t + u * TL;
    const uint32_t k = j & (Ns - 1);
    const uint32_t o = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) line[pidx<PAD>(o + r * Ns)] = v[u * R + r];
  }
}

template <class S, int R, int E, int PAD>
FFT_D void reg_stage_read(C<S> (&v)[E], const C<S>* line, uint32_t t, uint32_t TL, uint32_t NR) {
  constexpr int NB = E / R;
#pragma unroll
  for (int u = 0; u < NB; ++u) {
    const uint32_t j = t + u * TL;
#pragma unroll
    for (int q = 0; q < R; ++q) v[u * R + q] = line[pidx<PAD>(j + q * NR)];
  }
}

template <class S, int E, int PAD>
FFT_D void reg_read_any(uint32_t R, C<S> (&v)[E], const C<S>* line, uint32_t t, uint32_t TL,
                        uint32_t NR) {
  switch (R) {
    case 2: reg_stage_read<S, 2, E, PAD>(v, line, t, TL, NR); break;
    case 4: reg_stage_read<S, 4, E, PAD>(v, line, t, TL, NR); break;
    case 8: reg_stage_read<S, 8, E, PAD>(v, line, t, TL, NR); break;
    default: reg_stage_read<S, 16, E, PAD>(v, line, t, TL, NR); break;
  }
}

template <class S, int E, int PAD>
FFT_D void reg_compute_any(uint32_t R, C<S> (&v)[E], uint32_t t, uint32_t TL, uint32_t Ns,
                           const C<S>* __restrict__ tw, uint32_t tw_off) {
  switch (R) {
    case 2: reg_stage_compute<S, 2, E>(v, t, TL, Ns, tw, tw_off); break;
    case 4: reg_stage_compute<S, 4, E>(v, t, TL, Ns, tw, tw_off); break;
    case 8: reg_stage_compute<S, 8, E>(v, t, TL, Ns, tw, tw_off); break;
    default: reg_stage_compute<S, 16, E>(v, t, TL, Ns, tw, tw_off); break;
  }
}

template <class S, int E, int PAD>
FFT_D void reg_write_any(uint32_t R, const C<S> (&v)[E], C<S>* line, uint32_t t, uint32_t TL,
                         uint32_t Ns) {
  switch (R) {
    case 2: reg_stage_write<S, 2, E, PAD>(v, line, t, TL, Ns); break;
    case 4: reg_stage_write<S, 4, E, PAD>(v, line, t, TL, Ns); break;
    case 8: reg_stage_write<S, 8, E, PAD>(v, line, t, TL, Ns); break;
    default: reg_stage_write<S, 16, E, PAD>(v, line, t, TL, Ns); break;
  }
}

// Global load of the first stage: element (j + q*NR) of line c.
template <class S, int R, int E>
FFT_D void reg_load_global(C<S> (&v)[E], const C<S>* __restrict__ in, int64_t base, int64_t es,
                           uint32_t t, uint32_t TL, uint32_t NR, bool valid, bool conj_in) {
  constexpr int NB = E / R;
  if (!valid) {
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = czero<S>();
    return;
  }
#pragma unroll
  for (int u = 0; u < NB; ++u) {
    const uint32_t j = t + u * TL;
#pragma unroll
    for (int q = 0; q < R; ++q) v[u * R + q] = in[base + (int64_t)(j + q * NR) * es];
  }
  if (conj_in) {
#pragma unroll
    for (int i = 0; i < E; ++i) v[i].im = -v[i].im;
  }
}

template <class S, int E>
FFT_D void reg_load_any(uint32_t R, C<S> (&v)[E], const C<S>* __restrict__ in, int64_t base,
                        int64_t es, uint32_t t, uint32_t TL, uint32_t NR, bool valid, bool cj) {
  switch (R) {
    case 2: reg_load_global<S, 2, E>(v, in, base, es, t, TL, NR, valid, cj); break;
    case 4: reg_load_global<S, 4, E>(v, in, base, es, t, TL, NR, valid, cj); break;
    case 8: reg_load_global<S, 8, E>(v, in, base, es, t, TL, NR, valid, cj); break;
    default: reg_load_global<S, 16, E>(v, in, base, es, t, TL, NR, valid, cj); break;
  }
}

// Last stage: output n = j + r*Ns (k = j since j < Ns) straight to HBM.
template <class S, int R, int E>
FFT_D void reg_store_global(const C<S> (&v)[E], C<S>* __restrict__ out, int64_t base, int64_t es,
                            uint32_t t, uint32_t TL, uint32_t Ns, uint32_t fl, S sc,
                            uint64_t tw_row, const LinesParams& p) {
  constexpr int NB = E / R;
  const C<S>* __restrict__ ta = (const C<S>*)p.tws_a;
  const C<S>* __restrict__ tb = (const C<S>*)p.tws_b;
#pragma unroll
  for (int u = 0; u < NB; ++u) {
    const uint32_t j = t + u * TL;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const uint32_t n = j + r * Ns;
      C<S> x = v[u * R + r];
      // tw_row < M / N and n < N: the exponent stays below M
      if (fl & PF_TW_STORE)
        x = cmul(x, ta ? tw_two_level(ta, tb, tw_row * n, p.d_tws)
                       : twiddle<S>((tw_row * n) % p.tw_store_M, p.tw_store_M));
      if (fl & PF_SCALE) x = cscale(x, sc);
      if (fl & PF_CONJ_OUT) x.im = -x.im;
      out[base + (int64_t)n * es] = x;
    }
  }
}

template <class S, int E>
FFT_D void reg_store_any(uint32_t R, const C<S> (&v)[E], C<S>* __restrict__ out, int64_t base,
                         int64_t es, uint32_t t, uint32_t TL, uint32_t Ns, uint32_t fl, S sc,
                         uint64_t tw_row, const LinesParams& p) {
  switch (R) {
    case 2: reg_store_global<S, 2, E>(v, out, base, es, t, TL, Ns, fl, sc, tw_row, p); break;
    case 4: reg_store_global<S, 4, E>(v, out, base, es, t, TL, Ns, fl, sc, tw_row, p); break;
    case 8: reg_store_global<S, 8, E>(v, out, base, es, t, TL, Ns, fl, sc, tw_row, p); break;
    default: reg_store_global<S, 16, E>(v, out, base, es, t, TL, Ns, fl, sc, tw_row, p); break;
  }
}

// G lines of N = 2^m points (E*16 >= N >= 16); blockDim = G * N / E.
// Shared memory: G * LD elements, LD odd.
template <class S, int E, bool COLMAJOR>
__global__ void __launch_bounds__(sizeof(C<S>) == 8 ? 512 : 256)
    k_pow2(const __grid_constant__ LinesParams p) {
  constexpr int PAD = 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C<S>* sm = reinterpret_cast<C<S>*>(smem_raw);
  const uint32_t tid = threadIdx.x;
  const uint32_t N = p.N, G = p.G, LD = p.LD;
  const uint32_t TL = N / E;
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
  const C<S>* tw = (p.flags & PF_TW_TABLE) ? (const C<S>*)p.tw : nullptr;
  const Schedule& sch = p.sch;
  const uint32_t last = sch.nst - 1;
  C<S> v[E];
  C<S>* line = sm + c * LD;
  reg_load_any<S, E>(sch.st[0].R, v, (const C<S>*)p.in, g.in0 + (int64_t)c * g.dl_in, p.io.in_es,
                     t, TL, sch.st[0].NR, valid, p.flags & PF_CONJ_IN);
#pragma unroll 1
  for (uint32_t s = 0;; ++s) {
    const StageDesc& sd = sch.st[s];
    reg_compute_any<S, E, PAD>(sd.R, v, t, TL, sd.Ns, tw, sd.tw_off);
    if (s == last) break;
    reg_write_any<S, E, PAD>(sd.R, v, line, t, TL, sd.Ns);
    __syncthreads();
    reg_read_any<S, E, PAD>(sch.st[s + 1].R, v, line, t, TL, sch.st[s + 1].NR);
    __syncthreads();
  }
  const StageDesc& sl = sch.st[last];
  const S sc = Scalar<S>::from_double(p.scale);
  if (!(p.flags & PF_STORE_SMEM)) {
    if (valid) {
      const uint64_t row = (p.flags & PF_TW_STORE) ? fdiv((uint32_t)(g.c0 + c), p.d_tw) : 0;
      reg_store_any<S, E>(sl.R, v, (C<S>*)p.out, g.out0 + (int64_t)c * g.dl_out, p.io.out_es, t,
                          TL, sl.Ns, p.flags, sc, row, p);
    }
    return;
  }
  // the output order wants adjacent lines first: one pass through shared memory
  reg_write_any<S, E, PAD>(sl.R, v, line, t, TL, sl.Ns);
  __syncthreads();
  C<S>* __restrict__ out = (C<S>*)p.out;
  const uint32_t fl = p.flags;
  const uint32_t T = blockDim.x;
  for_each_elem(N, p.dN, G, p.dG, true, tid, T, [&](uint32_t cc, uint32_t n) {
    if (cc < g.nvalid) {
      C<S> x = sm[cc * LD + pidx<PAD>(n)];
      if (fl & PF_TW_STORE) {
        const uint64_t row = fdiv((uint32_t)(g.c0 + cc), p.d_tw);
        const uint64_t m = row * (uint64_t)n;
        x = cmul(x, p.tws_a ? tw_two_level((const C<S>*)p.tws_a, (const C<S>*)p.tws_b, m, p.d_tws)
                            : twiddle<S>(m % p.tw_store_M, p.tw_store_M));
      }
      if (fl & PF_SCALE) x = cscale(x, sc);
      if (fl & PF_CONJ_OUT) x.im = -x.im;
      out[g.out0 + (int64_t)cc * g.dl_out + (int64_t)n * p.io.out_es] = x;
    }
  });
}

template <class S, int E, bool COLMAJOR>
cudaError_t launch_pow2_t(const LinesParams& prm, unsigned grid, unsigned threads, size_t smem,
                          cudaStream_t st) {
  return launch(k_pow2<S, E, COLMAJOR>, prm, grid, threads, smem, st);
}

}  // namespace b2f
