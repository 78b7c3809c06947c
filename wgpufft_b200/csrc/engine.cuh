// Shared-memory Stockham engine: the per-line machinery every transform
// kernel of the library is built from.
//
// A CTA holds G lines of one length N in shared memory, line l at
// buf[l*LD + pidx(i)] (pidx pads one slot every 2^PAD elements so the radix-R
// strided accesses of a stage spread over the banks).  Two such buffers
// ping-pong: each stage of the runtime radix schedule reads the R inputs of
// a butterfly from one buffer, applies the stage twiddles and the codelet
// and writes the R outputs to their autosorted (Stockham) positions in the
// other, with one barrier per stage.  Only one butterfly's values are live
// in registers at a time.
//
// The reference's kernel families that this engine replaces are the
// Stockham stage (src/runtime/axis_plan.rs:3540-3664), the fused pow2 and
// fused smooth workgroup kernels (axis_plan.rs:1569-1820, 2573-3540) and the
// register-resident kernels (src/runtime/register_fft.rs:136-360); one
// engine with a runtime schedule covers all of them.
#pragma once
#include "dft.cuh"

#define FFT_MAX_STAGES 24

struct StageDesc {
  uint32_t R;       // radix of this stage
  uint32_t Ns;      // product of the radices before it
  uint32_t NR;      // N / R
  uint32_t tw_off;  // first entry of this stage's twiddles in the plan table
  FastDiv dNs, dNR;
};

struct Schedule {
  uint32_t N;
  uint32_t nst;
  StageDesc st[FFT_MAX_STAGES];
};

template <int PAD>
FFT_HD uint32_t pidx(uint32_t i) {
  return i + (i >> PAD);
}

// Padding shift per element size: one pad slot per 128 bytes of line.
template <class S>
struct PadOf {
  static constexpr int value = (sizeof(cpx<S>) == 8) ? 4 : 3;
};

// Stage twiddles W_M^{q k}, q = 1..R-1, computed in-kernel: W^k and W^{4k}
// from the octant-reduced sincospi, the others as products of at most three
// of those (each product adds about one rounding), so no table is read.
template <class S, int R>
FFT_D void apply_stage_twiddles(cpx<S>* v, uint32_t k, uint32_t M) {
  if constexpr (R <= 3) {
    const cpx<S> w1 = twiddle<S>(k, M);
    v[1] = cmul(v[1], w1);
    if constexpr (R == 3) v[2] = cmul(v[2], twiddle<S>(2 * k, M));
  } else {
    cpx<S> w[R];
    w[1] = twiddle<S>(k, M);
    w[2] = cmul(w[1], w[1]);
#pragma unroll
    for (int q = 3; q < R && q < 4; ++q) w[q] = cmul(w[q - 1], w[1]);
    if constexpr (R > 4) {
      w[4] = twiddle<S>(4 * k, M);
#pragma unroll
      for (int q = 5; q < R && q < 8; ++q) w[q] = cmul(w[4], w[q - 4]);
    }
    if constexpr (R > 8) {
      w[8] = cmul(w[4], w[4]);
#pragma unroll
      for (int q = 9; q < R; ++q) w[q] = cmul(w[8], w[q - 8]);
    }
#pragma unroll
    for (int q = 1; q < R; ++q) v[q] = cmul(v[q], w[q]);
  }
}

// One radix-R stage over the G lines of the CTA, src -> dst.  Butterfly b
// maps to line l = b / (N/R) and position j = b % (N/R); k = j % Ns selects
// the twiddles W_{Ns R}^{q k}.
template <class S, int R, int PAD>
FFT_D void fft_stage(const cpx<S>* __restrict__ src, cpx<S>* __restrict__ dst,
                     const StageDesc& sd, uint32_t G, uint32_t LD, uint32_t tid, uint32_t T,
                     const cpx<S>* __restrict__ tw) {
  const uint32_t total = G * sd.NR;
  const uint32_t M = sd.Ns * R;
#pragma unroll 1
  for (uint32_t b = tid; b < total; b += T) {
    const uint32_t l = fdiv(b, sd.dNR);
    const uint32_t j = b - l * sd.NR;
    const uint32_t k = j - fdiv(j, sd.dNs) * sd.Ns;
    const cpx<S>* sb = src + l * LD;
    cpx<S> v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = sb[pidx<PAD>(j + q * sd.NR)];
    if (sd.Ns > 1) {
      if (tw != nullptr) {
        const cpx<S>* t = tw + sd.tw_off + k * (R - 1);
#pragma unroll
        for (int q = 1; q < R; ++q) v[q] = cmul(v[q], t[q - 1]);
      } else {
        apply_stage_twiddles<S, R>(v, k, M);
      }
    }
    dft<S, R>(v);
    cpx<S>* db = dst + l * LD;
    const uint32_t o = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) db[pidx<PAD>(o + r * sd.Ns)] = v[r];
  }
}

// Runs the whole schedule from buffer a (ping-pong with b); returns the
// buffer holding the result.  The caller must have synchronised after
// writing `a`; the function ends with a barrier.
template <class S>
FFT_D cpx<S>* fft_lines_smem(cpx<S>* a, cpx<S>* b, const Schedule& sch, uint32_t G, uint32_t LD,
                             uint32_t tid, uint32_t T, const cpx<S>* __restrict__ tw) {
  constexpr int PAD = PadOf<S>::value;
#pragma unroll 1
  for (uint32_t s = 0; s < sch.nst; ++s) {
    const StageDesc& sd = sch.st[s];
    switch (sd.R) {
      case 2: fft_stage<S, 2, PAD>(a, b, sd, G, LD, tid, T, tw); break;
      case 3: fft_stage<S, 3, PAD>(a, b, sd, G, LD, tid, T, tw); break;
      case 4: fft_stage<S, 4, PAD>(a, b, sd, G, LD, tid, T, tw); break;
      case 5: fft_stage<S, 5, PAD>(a, b, sd, G, LD, tid, T, tw); break;
      case 7: fft_stage<S, 7, PAD>(a, b, sd, G, LD, tid, T, tw); break;
      case 8: fft_stage<S, 8, PAD>(a, b, sd, G, LD, tid, T, tw); break;
      case 9: fft_stage<S, 9, PAD>(a, b, sd, G, LD, tid, T, tw); break;
      case 11: fft_stage<S, 11, PAD>(a, b, sd, G, LD, tid, T, tw); break;
      case 13: fft_stage<S, 13, PAD>(a, b, sd, G, LD, tid, T, tw); break;
      case 16: fft_stage<S, 16, PAD>(a, b, sd, G, LD, tid, T, tw); break;
      default: break;
    }
    __syncthreads();
    cpx<S>* t = a;
    a = b;
    b = t;
  }
  return a;
}
