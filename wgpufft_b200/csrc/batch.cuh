// Batched launch of many 1D f32 lines of mixed lengths: the device side.
//
// Two persistent kernels share one execute call:
//  - k_batch_cta: each CTA repeatedly takes the next task from an atomic
//    counter; a task is up to G lines of one length whose FFT (mixed radix,
//    Rader or Bluestein) fits one CTA's shared memory;
//  - k_batch_cluster<P>: a thread-block cluster of P CTAs takes one long line
//    at a time and transforms it in a single HBM pass, the CTAs exchanging
//    data through distributed shared memory:
//      n = m + L*r (r = CTA rank, m < L = T/P),   k = P*k1 + k2,
//      X[P k1 + k2] = sum_m W_L^{m k1} [ W_T^{m k2} sum_r W_P^{r k2} x[m + L r] ],
//    i.e. a cross-CTA radix-P step with the W_T^{m k2} twiddle, a local
//    length-L FFT in each CTA, and a transposed read-out.  Bluestein lines
//    run their forward FFT this way, multiply by the chirp spectrum in the
//    transposed order, and run the inverse FFT in the mirrored order (local
//    FFT first, then the cross-CTA step), so the convolution never leaves
//    the chip.
// Work queue polls are bounded: a task index is taken with one atomicAdd and
// nothing ever waits on another CTA except the cluster barriers, which every
// CTA of a cluster reaches the same number of times.
#pragma once
#include <cooperative_groups.h>

#include "kernels_impl.cuh"
#include "regfft.cuh"

namespace b2f {

enum BatchKind : uint32_t {
  BK_MIXED = 0,     // one CTA, mixed radix
  BK_RADER = 1,     // one CTA, Rader
  BK_BLUE = 2,      // one CTA, Bluestein
  BK_CL_MIXED = 3,  // cluster, mixed radix (T = N)
  BK_CL_BLUE = 4,   // cluster, Bluestein (T = convolution length)
  BK_LONG = 5,      // one CTA, two passes N = N1*N2 through an L2-resident scratch slot
  BK_LONG_BLUE = 6, // one CTA, Bluestein over M = N1*N2: four passes through two slots
};

struct BatchLen {
  uint32_t kind;
  uint32_t N;     // line length
  uint32_t M;     // transform length: N, p-1, or the convolution length
  uint32_t G;     // lines per task (CTA kinds)
  uint32_t LD;    // shared-memory line pitch
  uint32_t P;     // cluster ranks in use (cluster kinds)
  uint32_t L;     // M / P (cluster kinds)
  float scale;    // normalisation of this length (f32, as the reference)
  const c32* bhat;
  const uint32_t* perm_in;
  const uint32_t* perm_out;
  FastDiv dN, dM, dMN, dP1;
  uint32_t N1, N2, LD1, LD2;  // BK_LONG: N = N1 * N2, pitches of the two passes
  // two-level tables of the inter-pass twiddle W_T^j, j = a*B + b (offsets
  // into BatchParams::tw): ta[a] = W_T^{a B}, tb[b] = W_T^b.
  //   BK_LONG: T = N, B = N2 (a < N1);  cluster kinds: T = M, B = L (a < P).
  uint32_t ta, tb;
  FastDiv dB;
  uint32_t lg;    // long kinds: log2 of the lines per column-pass group (G = 1 << lg)
  uint32_t lg2;   // long kinds: log2 of the lines per row-pass group
  uint32_t reg1, reg2;  // the column / row pass length is a power of two: register path
  Schedule sch;   // schedule of the per-CTA FFT length (N, p-1, M, L or N1)
  Schedule sch2;  // BK_LONG: schedule of N2
};

struct BatchTask {
  uint32_t len;    // index into the length table
  uint32_t first;  // first line (sorted order)
  uint32_t count;  // lines in the task
  uint32_t pad;
};

struct BatchParams {
  const c32* in;
  c32* out;
  c32* scratch;          // BK_LONG: one slot of slot_elems per CTA
  uint64_t slot_elems;
  const uint64_t* line_scratch;  // phased long lines: scratch offset of each line
  const c32* tw;         // stage and inter-pass twiddle tables (FP64-built, rounded once)
  const BatchLen* lens;
  const BatchTask* tasks;
  const uint64_t* line_off;  // complex offset of each line (sorted order)
  uint32_t ntasks;
  uint32_t inverse;
  unsigned int* counter;
};

constexpr int kBatchMaxG = 256;

// Asynchronous 8-byte global -> shared copy (sm_80+ LDGSTS): every thread
// keeps all of its loads in flight instead of waiting on each one.
FFT_D void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
FFT_D void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

template <class T>
FFT_D void copy_words(T* dst, const T* src, uint32_t tid, uint32_t nthreads) {
  static_assert(sizeof(T) % 4 == 0, "word copy");
  const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
  uint32_t* d = reinterpret_cast<uint32_t*>(dst);
  for (uint32_t i = tid; i < sizeof(T) / 4; i += nthreads) d[i] = s[i];
}

// Register-resident FFT of G power-of-two lines of N (16..512) already in
// shared memory (line c at sm[c*LD + pidx(n)]), transformed in place and
// left in natural order: each of the G*N/16 active threads keeps 16 values
// in registers through the radix-16 stages (regfft.cuh), shared memory is
// only the exchange between stages.  Ends with a barrier.
FFT_D void reg_fft_group_smem(c32* sm, uint32_t G, uint32_t N, uint32_t LD, uint32_t tid,
                              const Schedule& sch, const c32* __restrict__ tw) {
  constexpr int PAD = PadOf<float>::value;
  constexpr int E = 16;
  const uint32_t TL = N / E;
  const uint32_t c = tid / TL, t = tid - c * TL;
  const bool valid = c < G;
  c32* line = sm + (valid ? c : 0) * LD;
  c32 v[E];
  const uint32_t last = sch.nst - 1;
  for (uint32_t s = 0;; ++s) {
    const StageDesc& sd = sch.st[s];
    if (valid) {
      reg_read_any<float, E, PAD>(sd.R, v, line, t, TL, sd.NR);
      reg_compute_any<float, E, PAD>(sd.R, v, t, TL, sd.Ns, tw, sd.tw_off);
    }
    __syncthreads();
    if (valid) reg_write_any<float, E, PAD>(sd.R, v, line, t, TL, sd.Ns);
    __syncthreads();
    if (s == last) break;
  }
}

// W_T^j from the two-level table: j = a*B + b.
FFT_D c32 tw2(const BatchParams& bp, const BatchLen& L, uint32_t j, uint32_t B) {
  const uint32_t a = fdiv(j, L.dB), b = j - a * B;
  return cmul(bp.tw[L.ta + a], bp.tw[L.tb + b]);
}

// --------------------------------------------------------------- CTA tasks
FFT_D void batch_mixed(const BatchParams& bp, const BatchLen& L, const int64_t* base, uint32_t cnt,
                       c32* A, c32* B, uint32_t tid, uint32_t T) {
  constexpr int PAD = PadOf<float>::value;
  const uint32_t N = L.N, LD = L.LD;
  const bool inv = bp.inverse;
  for (uint32_t e = tid; e < cnt * N; e += T) {
    const uint32_t c = fdiv(e, L.dN), n = e - c * N;
    cp_async8(&A[c * LD + pidx<PAD>(n)], &bp.in[base[c] + n]);
  }
  cp_async_wait_all();
  if (inv) {
    for (uint32_t e = tid; e < cnt * N; e += T) {
      const uint32_t c = fdiv(e, L.dN), n = e - c * N;
      c32& v = A[c * LD + pidx<PAD>(n)];
      v.im = -v.im;
    }
  }
  __syncthreads();
  const c32* r = fft_lines_smem<float>(A, B, L.sch, cnt, LD, tid, T, bp.tw);
  const float sc = L.scale;
  for (uint32_t e = tid; e < cnt * N; e += T) {
    const uint32_t c = fdiv(e, L.dN), n = e - c * N;
    c32 v = r[c * LD + pidx<PAD>(n)];
    v.re *= sc;
    v.im = inv ? -v.im * sc : v.im * sc;
    bp.out[base[c] + n] = v;
  }
}

FFT_D void batch_rader(const BatchParams& bp, const BatchLen& L, const int64_t* base, uint32_t cnt,
                       c32* A, c32* B, c32* x0s, c32* X0s, uint32_t tid, uint32_t T) {
  constexpr int PAD = PadOf<float>::value;
  const uint32_t P = L.N, P1 = L.M, LD = L.LD;
  const bool inv = bp.inverse;
  for (uint32_t e = tid; e < cnt * P; e += T) {
    const uint32_t c = fdiv(e, L.dN), n = e - c * P;
    c32 v = bp.in[base[c] + n];
    if (inv) v.im = -v.im;
    A[c * LD + pidx<PAD>(n)] = v;
  }
  __syncthreads();
  if (tid < cnt) x0s[tid] = A[tid * LD];
  for (uint32_t e = tid; e < cnt * P1; e += T) {
    const uint32_t l = fdiv(e, L.dP1), q = e - l * P1;
    B[l * LD + pidx<PAD>(q)] = A[l * LD + pidx<PAD>(L.perm_in[q])];
  }
  __syncthreads();
  c32* r1 = fft_lines_smem<float>(B, A, L.sch, cnt, LD, tid, T, bp.tw);
  c32* o1 = (r1 == A) ? B : A;
  if (tid < cnt) X0s[tid] = x0s[tid] + r1[tid * LD];
  __syncthreads();
  for (uint32_t e = tid; e < cnt * P1; e += T) {
    const uint32_t l = fdiv(e, L.dP1), m = e - l * P1;
    c32 v = cmul(r1[l * LD + pidx<PAD>(m)], L.bhat[m]);
    v.im = -v.im;
    r1[l * LD + pidx<PAD>(m)] = v;
  }
  __syncthreads();
  const c32* r2 = fft_lines_smem<float>(r1, o1, L.sch, cnt, LD, tid, T, bp.tw);
  const float sc = L.scale;
  for (uint32_t e = tid; e < cnt * P; e += T) {
    const uint32_t c = fdiv(e, L.dN), n = e - c * P;
    c32 v;
    if (n == 0) {
      v = X0s[c];
    } else {
      c32 w = r2[c * LD + pidx<PAD>(L.perm_out[n - 1])];
      w.im = -w.im;
      v = x0s[c] + w;
    }
    v.re *= sc;
    v.im = inv ? -v.im * sc : v.im * sc;
    bp.out[base[c] + n] = v;
  }
}

FFT_D void batch_blue(const BatchParams& bp, const BatchLen& L, const int64_t* base, uint32_t cnt,
                      c32* A, c32* B, uint32_t tid, uint32_t T) {
  constexpr int PAD = PadOf<float>::value;
  const uint32_t N = L.N, M = L.M, LD = L.LD;
  const bool inv = bp.inverse;
  for (uint32_t e = tid; e < cnt * M; e += T) {
    const uint32_t c = fdiv(e, L.dM), m = e - c * M;
    c32 v = czero<float>();
    if (m < N) {
      v = bp.in[base[c] + m];
      if (inv) v.im = -v.im;
      v = cmul(v, chirp<float>(m, N));
    }
    A[c * LD + pidx<PAD>(m)] = v;
  }
  __syncthreads();
  c32* r1 = fft_lines_smem<float>(A, B, L.sch, cnt, LD, tid, T, bp.tw);
  c32* o1 = (r1 == A) ? B : A;
  for (uint32_t e = tid; e < cnt * M; e += T) {
    const uint32_t l = fdiv(e, L.dM), m = e - l * M;
    c32 v = cmul(r1[l * LD + pidx<PAD>(m)], L.bhat[m]);
    v.im = -v.im;
    r1[l * LD + pidx<PAD>(m)] = v;
  }
  __syncthreads();
  const c32* r2 = fft_lines_smem<float>(r1, o1, L.sch, cnt, LD, tid, T, bp.tw);
  const float sc = L.scale;
  for (uint32_t e = tid; e < cnt * N; e += T) {
    const uint32_t c = fdiv(e, L.dN), k = e - c * N;
    c32 w = r2[c * LD + pidx<PAD>(k)];
    w.im = -w.im;
    c32 v = cmul(w, chirp<float>(k, N));
    v.re *= sc;
    v.im = inv ? -v.im * sc : v.im * sc;
    bp.out[base[c] + k] = v;
  }
}

// Long lines in one CTA, through scratch slots (reused line after line, so
// they mostly stay in L2).  One length-T = N1*N2 FFT is two passes with
// n = N2*n1 + n2, k = k1 + N1*k2:
//   column pass: G adjacent columns n2 at a time, FFT_N1 over n1, the
//                W_T^{n2 k1} twiddle, stored at N2*k1 + n2;
//   row pass:    G rows k1 at a time, FFT_N2 over n2, X[k1 + N1*k2] (G
//                consecutive outputs per k2).
// The hooks decide where a pass reads and writes: the input of the column
// pass (a line of x, optionally chirped and zero-padded, or a slot) and the
// output of the row pass (the line of out, or a slot in natural order after
// the Bluestein spectrum product).
enum LongIn : uint32_t { LI_X = 0, LI_X_CHIRP = 1, LI_SLOT = 2 };
enum LongOut : uint32_t { LO_X = 0, LO_SLOT_SPECTRUM = 1, LO_X_CHIRP = 2 };

FFT_D void long_column_group(const BatchParams& bp, const BatchLen& L, int64_t base,
                             const c32* src_slot, c32* dst, LongIn mode, uint32_t c0, c32* A,
                             c32* B, uint32_t tid, uint32_t T) {
  constexpr int PAD = PadOf<float>::value;
  const uint32_t N = L.N, N1 = L.N1, N2 = L.N2, lg = L.lg, G = 1u << lg;
  const bool inv = bp.inverse;
  for (uint32_t e = tid; e < (N1 << lg); e += T) {
    const uint32_t n1 = e >> lg, c = e & (G - 1);
    c32* d = &A[c * L.LD1 + pidx<PAD>(n1)];
    const uint32_t n = N2 * n1 + c0 + c;
    if (c0 + c >= N2) {
      *d = czero<float>();
    } else if (mode == LI_SLOT) {
      cp_async8(d, &src_slot[n]);
    } else if (mode == LI_X) {
      cp_async8(d, &bp.in[base + n]);
    } else {  // chirped, zero beyond the line
      if (n < N) {
        c32 v = bp.in[base + n];
        if (inv) v.im = -v.im;
        *d = cmul(v, chirp<float>(n, N));
      } else {
        *d = czero<float>();
      }
    }
  }
  cp_async_wait_all();
  if (inv && mode == LI_X) {
    for (uint32_t e = tid; e < (N1 << lg); e += T) {
      const uint32_t n1 = e >> lg, c = e & (G - 1);
      c32& v = A[c * L.LD1 + pidx<PAD>(n1)];
      v.im = -v.im;
    }
  }
  __syncthreads();
  const c32* r;
  if (L.reg1) {
    reg_fft_group_smem(A, G, N1, L.LD1, tid, L.sch, bp.tw);
    r = A;
  } else {
    r = fft_lines_smem<float>(A, B, L.sch, G, L.LD1, tid, T, bp.tw);
  }
  for (uint32_t e = tid; e < (N1 << lg); e += T) {
    const uint32_t k1 = e >> lg, c = e & (G - 1);
    if (c0 + c < N2) {
      c32 v = r[c * L.LD1 + pidx<PAD>(k1)];
      v = cmul(v, tw2(bp, L, (c0 + c) * k1, N2));
      dst[(uint64_t)N2 * k1 + c0 + c] = v;
    }
  }
  __syncthreads();
}

FFT_D void long_column_pass(const BatchParams& bp, const BatchLen& L, int64_t base,
                            const c32* src_slot, c32* dst, LongIn mode, c32* A, c32* B,
                            uint32_t tid, uint32_t T) {
  for (uint32_t c0 = 0; c0 < L.N2; c0 += 1u << L.lg)
    long_column_group(bp, L, base, src_slot, dst, mode, c0, A, B, tid, T);
}

FFT_D void long_row_group(const BatchParams& bp, const BatchLen& L, int64_t base, const c32* slot,
                          c32* dst_slot, LongOut mode, uint32_t k0, c32* A, c32* B, uint32_t tid,
                          uint32_t T) {
  constexpr int PAD = PadOf<float>::value;
  const uint32_t N = L.N, N1 = L.N1, N2 = L.N2, lg = L.lg2, G = 1u << lg;
  const bool inv = bp.inverse;
  const float sc = L.scale;
#pragma unroll 1
  for (uint32_t rr = 0; rr < G; ++rr) {
    const bool ok = k0 + rr < N1;
    const c32* row = slot + (uint64_t)N2 * (k0 + rr);
    for (uint32_t n2 = tid; n2 < N2; n2 += T) {
      if (ok) cp_async8(&A[rr * L.LD2 + pidx<PAD>(n2)], &row[n2]);
      else A[rr * L.LD2 + pidx<PAD>(n2)] = czero<float>();
    }
  }
  cp_async_wait_all();
  __syncthreads();
  const c32* r;
  if (L.reg2) {
    reg_fft_group_smem(A, G, N2, L.LD2, tid, L.sch2, bp.tw);
    r = A;
  } else {
    r = fft_lines_smem<float>(A, B, L.sch2, G, L.LD2, tid, T, bp.tw);
  }
  for (uint32_t e = tid; e < (N2 << lg); e += T) {
    const uint32_t k2 = e >> lg, rr = e & (G - 1);
    if (k0 + rr >= N1) continue;
    const uint32_t k = k0 + rr + N1 * k2;
    c32 v = r[rr * L.LD2 + pidx<PAD>(k2)];
    if (mode == LO_X) {
      v.re *= sc;
      v.im = inv ? -v.im * sc : v.im * sc;
      bp.out[base + k] = v;
    } else if (mode == LO_SLOT_SPECTRUM) {
      v = cmul(v, L.bhat[k]);
      v.im = -v.im;  // conjugated: the next forward FFT computes the inverse
      dst_slot[k] = v;
    } else if (k < N) {
      v.im = -v.im;
      v = cmul(v, chirp<float>(k, N));
      v.re *= sc;
      v.im = inv ? -v.im * sc : v.im * sc;
      bp.out[base + k] = v;
    }
  }
  __syncthreads();
}

FFT_D void long_row_pass(const BatchParams& bp, const BatchLen& L, int64_t base, const c32* slot,
                         c32* dst_slot, LongOut mode, c32* A, c32* B, uint32_t tid, uint32_t T) {
  for (uint32_t k0 = 0; k0 < L.N1; k0 += 1u << L.lg2)
    long_row_group(bp, L, base, slot, dst_slot, mode, k0, A, B, tid, T);
}

// One phase of a long line, one pass group per task (task.pad = phase,
// task.count = first column / row of the group):
//   smooth lines:    1 column pass x -> scratch, 2 row pass scratch -> out;
//   Bluestein lines: 1 chirped column pass x -> s1, 2 row pass + spectrum
//                    product s1 -> s2, 3 column pass s2 -> s1, 4 row pass
//                    + chirp s1 -> out.
// Consecutive phases are consecutive launches, so every task of a phase
// sees the previous phase's scratch complete.
FFT_D void long_phase_task(const BatchParams& bp, const BatchLen& L, int64_t base, c32* slot,
                           uint32_t phase, uint32_t g0, c32* A, c32* B, uint32_t tid,
                           uint32_t T) {
  const bool blue = L.kind == BK_LONG_BLUE;
  c32* s1 = slot;
  c32* s2 = slot + L.M;
  switch (phase) {
    case 1: long_column_group(bp, L, base, nullptr, s1, blue ? LI_X_CHIRP : LI_X, g0, A, B, tid, T); break;
    case 2: long_row_group(bp, L, base, s1, s2, blue ? LO_SLOT_SPECTRUM : LO_X, g0, A, B, tid, T); break;
    case 3: long_column_group(bp, L, base, s2, s1, LI_SLOT, g0, A, B, tid, T); break;
    case 4: long_row_group(bp, L, base, s1, nullptr, LO_X_CHIRP, g0, A, B, tid, T); break;
    default: break;
  }
}

// A long smooth line: two passes through one slot.
FFT_D void batch_long(const BatchParams& bp, const BatchLen& L, int64_t base, c32* slot, c32* A,
                      c32* B, uint32_t tid, uint32_t T) {
  long_column_pass(bp, L, base, nullptr, slot, LI_X, A, B, tid, T);
  long_row_pass(bp, L, base, slot, nullptr, LO_X, A, B, tid, T);
}

// A long Bluestein line, convolution M = N1*N2: chirped column pass and row
// pass into the spectrum product (slot 2, natural order, conjugated), then
// the column and row passes of the second FFT, chirped into the output.
FFT_D void batch_long_blue(const BatchParams& bp, const BatchLen& L, int64_t base, c32* slot,
                           c32* A, c32* B, uint32_t tid, uint32_t T) {
  c32* s1 = slot;
  c32* s2 = slot + L.M;
  long_column_pass(bp, L, base, nullptr, s1, LI_X_CHIRP, A, B, tid, T);
  long_row_pass(bp, L, base, s1, s2, LO_SLOT_SPECTRUM, A, B, tid, T);
  long_column_pass(bp, L, base, s2, s1, LI_SLOT, A, B, tid, T);
  long_row_pass(bp, L, base, s1, nullptr, LO_X_CHIRP, A, B, tid, T);
}

// Persistent CTA kernel: blockDim.x threads, dynamic shared memory holds the
// two line buffers of the largest task plus Rader's x0/X0 slots.
__global__ void __launch_bounds__(256, 4) k_batch_cta(const __grid_constant__ BatchParams bp,
                                                   uint32_t buf_elems) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ BatchLen s_len;
  __shared__ int64_t s_base[kBatchMaxG];
  __shared__ uint32_t s_task;
  uint32_t s_len_idx = 0xFFFFFFFFu;  // length descriptor currently in s_len (same in every thread)
  c32* A = reinterpret_cast<c32*>(smem_raw);
  c32* B = A + buf_elems;
  c32* x0s = B + buf_elems;
  c32* X0s = x0s + kBatchMaxG;
  const uint32_t tid = threadIdx.x, T = blockDim.x;
  for (;;) {
    if (tid == 0) s_task = atomicAdd(bp.counter, 1u);
    __syncthreads();
    const uint32_t t = s_task;
    if (t >= bp.ntasks) break;
    const BatchTask task = bp.tasks[t];
    if (task.len != s_len_idx) copy_words(&s_len, bp.lens + task.len, tid, T);
    s_len_idx = task.len;
    const uint32_t nbase = task.pad != 0 ? 1u : task.count;
    for (uint32_t c = tid; c < nbase; c += T) s_base[c] = (int64_t)bp.line_off[task.first + c];
    __syncthreads();
    if (task.pad != 0) {  // one phase group of a long line
      long_phase_task(bp, s_len, s_base[0], bp.scratch + bp.line_scratch[task.first], task.pad,
                      task.count, A, B, tid, T);
      __syncthreads();
      continue;
    }
    switch (s_len.kind) {
      case BK_MIXED: batch_mixed(bp, s_len, s_base, task.count, A, B, tid, T); break;
      case BK_RADER: batch_rader(bp, s_len, s_base, task.count, A, B, x0s, X0s, tid, T); break;
      case BK_BLUE: batch_blue(bp, s_len, s_base, task.count, A, B, tid, T); break;
      case BK_LONG:
        batch_long(bp, s_len, s_base[0], bp.scratch + (uint64_t)blockIdx.x * bp.slot_elems, A, B,
                   tid, T);
        break;
      case BK_LONG_BLUE:
        batch_long_blue(bp, s_len, s_base[0], bp.scratch + (uint64_t)blockIdx.x * bp.slot_elems,
                        A, B, tid, T);
        break;
      default: break;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------- cluster tasks
template <int P>
FFT_D void cluster_radix_p(cooperative_groups::cluster_group& cl, c32* src_local, c32* dst_local,
                           uint32_t Lr, uint32_t Mt, uint32_t rank, uint32_t tid, uint32_t T,
                           bool twiddle_first, const BatchParams& bp, const BatchLen& L) {
  // For m in this CTA's share: v[r] = src[r][m]; (twiddle_first: v[r] *= W_Mt^{m r});
  // DFT_P; (else: v[k2] *= W_Mt^{m k2}); dst[k2][m] = v[k2].
  constexpr int PAD = PadOf<float>::value;
  const uint32_t m0 = (uint32_t)(((uint64_t)rank * Lr) / P);
  const uint32_t m1 = (uint32_t)(((uint64_t)(rank + 1) * Lr) / P);
  for (uint32_t m = m0 + tid; m < m1; m += T) {
    c32 v[P];
    const uint32_t pm = pidx<PAD>(m);
#pragma unroll
    for (int r = 0; r < P; ++r) v[r] = cl.map_shared_rank(src_local, r)[pm];
    if (twiddle_first) {
#pragma unroll
      for (int r = 1; r < P; ++r) v[r] = cmul(v[r], tw2(bp, L, m * r, Lr));
    }
    dft<float, P>(v);
    if (!twiddle_first) {
#pragma unroll
      for (int r = 1; r < P; ++r) v[r] = cmul(v[r], tw2(bp, L, m * r, Lr));
    }
#pragma unroll
    for (int r = 0; r < P; ++r) cl.map_shared_rank(dst_local, r)[pm] = v[r];
  }
}

template <int P>
__global__ void __launch_bounds__(512, 1) k_batch_cluster(const __grid_constant__ BatchParams bp,
                                                          uint32_t buf_elems) {
  namespace cg = cooperative_groups;
  constexpr int PAD = PadOf<float>::value;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ BatchLen s_len;
  __shared__ uint32_t s_task;
  c32* A = reinterpret_cast<c32*>(smem_raw);
  c32* B = A + buf_elems;
  const uint32_t tid = threadIdx.x, T = blockDim.x;
  const uint32_t rank = cl.block_rank();
  for (;;) {
    if (rank == 0 && tid == 0) s_task = atomicAdd(bp.counter, 1u);
    cl.sync();
    const uint32_t t = *cl.map_shared_rank(&s_task, 0);
    cl.sync();  // rank 0 may not leave or move on while others read its slot
    if (t >= bp.ntasks) break;
    const BatchTask task = bp.tasks[t];
    copy_words(&s_len, bp.lens + task.len, tid, T);
    __syncthreads();
    const BatchLen& L = s_len;
    const uint32_t N = L.N, Mt = L.M, Lr = L.L;
    const bool inv = bp.inverse;
    const bool blue = L.kind == BK_CL_BLUE;
    const int64_t base = (int64_t)bp.line_off[task.first];
    const bool active = rank < L.P;  // ranks beyond P idle through the task
    // 1. this CTA's contiguous chunk n = rank*L + m
    if (active) {
      for (uint32_t m = tid; m < Lr; m += T) {
        const uint32_t n = rank * Lr + m;
        c32 v = czero<float>();
        if (n < N) {
          v = bp.in[base + n];
          if (inv) v.im = -v.im;
          if (blue) v = cmul(v, chirp<float>(n, N));
        }
        A[pidx<PAD>(m)] = v;
      }
    }
    cl.sync();
    // 2. cross-CTA radix-P step, twiddle after: A (all ranks) -> B (all ranks)
    if (L.P == P) {
      cluster_radix_p<P>(cl, A, B, Lr, Mt, rank, tid, T, false, bp, L);
    } else if (active) {
      switch (L.P) {
        case 2: cluster_radix_p<2>(cl, A, B, Lr, Mt, rank, tid, T, false, bp, L); break;
        case 3: cluster_radix_p<3>(cl, A, B, Lr, Mt, rank, tid, T, false, bp, L); break;
        case 4: cluster_radix_p<4>(cl, A, B, Lr, Mt, rank, tid, T, false, bp, L); break;
        case 5: cluster_radix_p<5>(cl, A, B, Lr, Mt, rank, tid, T, false, bp, L); break;
        case 7: cluster_radix_p<7>(cl, A, B, Lr, Mt, rank, tid, T, false, bp, L); break;
        default: break;
      }
    }
    cl.sync();
    // 3. local FFT_L of B (every rank runs it so barriers match; idle ranks on garbage)
    c32* r = fft_lines_smem<float>(B, A, L.sch, 1, L.LD, tid, T, bp.tw);
    c32* o = (r == A) ? B : A;
    if (!blue) {
      cl.sync();
      // 4. output n = P*k1 + k2 of this rank's chunk from rank k2, slot k1
      if (active) {
        const float sc = L.scale;
        for (uint32_t m = tid; m < Lr; m += T) {
          const uint32_t n = rank * Lr + m;
          const uint32_t k1 = n / L.P, k2 = n - k1 * L.P;
          c32 v = cl.map_shared_rank(r, k2)[pidx<PAD>(k1)];
          v.re *= sc;
          v.im = inv ? -v.im * sc : v.im * sc;
          bp.out[base + n] = v;
        }
      }
      cl.sync();
      continue;
    }
    // Bluestein: r holds F[P*k1 + rank] at slot k1; product with the chirp
    // spectrum, conjugated for the inverse through the forward kernels
    if (active) {
      for (uint32_t k1 = tid; k1 < Lr; k1 += T) {
        c32 v = cmul(r[pidx<PAD>(k1)], L.bhat[(uint64_t)k1 * L.P + rank]);
        v.im = -v.im;
        r[pidx<PAD>(k1)] = v;
      }
    }
    __syncthreads();
    // inverse in the mirrored order: local FFT_L first ...
    c32* r2 = fft_lines_smem<float>(r, o, L.sch, 1, L.LD, tid, T, bp.tw);
    c32* o2 = (r2 == r) ? o : r;
    cl.sync();
    // ... then the twiddle and the cross-CTA radix-P step: r2 -> o2
    if (L.P == P) {
      cluster_radix_p<P>(cl, r2, o2, Lr, Mt, rank, tid, T, true, bp, L);
    } else if (active) {
      switch (L.P) {
        case 2: cluster_radix_p<2>(cl, r2, o2, Lr, Mt, rank, tid, T, true, bp, L); break;
        case 3: cluster_radix_p<3>(cl, r2, o2, Lr, Mt, rank, tid, T, true, bp, L); break;
        case 4: cluster_radix_p<4>(cl, r2, o2, Lr, Mt, rank, tid, T, true, bp, L); break;
        case 5: cluster_radix_p<5>(cl, r2, o2, Lr, Mt, rank, tid, T, true, bp, L); break;
        case 7: cluster_radix_p<7>(cl, r2, o2, Lr, Mt, rank, tid, T, true, bp, L); break;
        default: break;
      }
    }
    cl.sync();
    // rank r holds y[r*L + m]; the convolution is conj(y)
    if (active) {
      const float sc = L.scale;
      for (uint32_t m = tid; m < Lr; m += T) {
        const uint32_t n = rank * Lr + m;
        if (n < N) {
          c32 w = o2[pidx<PAD>(m)];
          w.im = -w.im;
          c32 v = cmul(w, chirp<float>(n, N));
          v.re *= sc;
          v.im = inv ? -v.im * sc : v.im * sc;
          bp.out[base + n] = v;
        }
      }
    }
    cl.sync();
  }
}

}  // namespace b2f
