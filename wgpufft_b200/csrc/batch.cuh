// Batched launch of many 1D f32 lines of mixed lengths: the device side.
//
// Persistent kernels share one execute call:
//  - k_batch_cta: each CTA repeatedly takes the next task from an atomic
//    counter; a task is up to G lines of one length whose FFT (mixed radix,
//    Rader or Bluestein) fits one CTA's shared memory;
//  - k_long_pass (longpass.cuh): the longer lines, as column and row passes
//    through a scratch region;
//  - k_batch_cluster<P> (optional route for the longer lines): a thread-block cluster of P CTAs takes one long line
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

namespace b2f {

enum BatchKind : uint32_t {
  BK_MIXED = 0,     // one CTA, mixed radix
  BK_RADER = 1,     // one CTA, Rader
  BK_BLUE = 2,      // one CTA, Bluestein
  BK_CL_MIXED = 3,  // cluster, mixed radix (T = N)
  BK_CL_BLUE = 4,   // cluster, Bluestein (T = convolution length)
  BK_LONG = 5,      // long line: two passes N = N1*N2 through scratch (k_long_pass)
  BK_LONG_BLUE = 6, // long Bluestein line: three passes over M = N1*N2 (k_long_pass)
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
  // two-level table of the cross-CTA twiddle W_M^j of the cluster kinds,
  // j = a*L + b (offsets into BatchParams::tw): ta[a] = W_M^{a L}, tb[b] = W_M^b.
  uint32_t ta, tb;
  FastDiv dB;
  Schedule sch;   // schedule of the per-CTA FFT length (N, p-1, M or L)
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
  const c32* tw;         // stage and inter-pass twiddle tables (FP64-built, rounded once)
  const BatchLen* lens;
  const BatchTask* tasks;
  const uint64_t* line_off;  // complex offset of each line in `in` (sorted order)
  const uint64_t* line_off_out;  // its offset in `out`, or null: the same as in `in`
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

// W_T^j from the two-level table: j = a*B + b.
FFT_D c32 tw2(const BatchParams& bp, const BatchLen& L, uint32_t j, uint32_t B) {
  const uint32_t a = fdiv(j, L.dB), b = j - a * B;
  return cmul(bp.tw[L.ta + a], bp.tw[L.tb + b]);
}

// --------------------------------------------------------------- CTA tasks
FFT_D void batch_mixed(const BatchParams& bp, const BatchLen& L, const int64_t* base, const int64_t* obase, uint32_t cnt,
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
    bp.out[obase[c] + n] = v;
  }
}

FFT_D void batch_rader(const BatchParams& bp, const BatchLen& L, const int64_t* base, const int64_t* obase, uint32_t cnt,
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
    bp.out[obase[c] + n] = v;
  }
}

FFT_D void batch_blue(const BatchParams& bp, const BatchLen& L, const int64_t* base, const int64_t* obase, uint32_t cnt,
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
    bp.out[obase[c] + k] = v;
  }
}

// Persistent CTA kernel: blockDim.x threads, dynamic shared memory holds the
// two line buffers of the largest task plus Rader's x0/X0 slots.
__global__ void __launch_bounds__(256, 4) k_batch_cta(const __grid_constant__ BatchParams bp,
                                                   uint32_t buf_elems) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ BatchLen s_len;
  __shared__ int64_t s_base[kBatchMaxG];
  __shared__ int64_t s_obase[kBatchMaxG];
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
    for (uint32_t c = tid; c < task.count; c += T) {
      s_base[c] = (int64_t)bp.line_off[task.first + c];
      s_obase[c] = (int64_t)(bp.line_off_out ? bp.line_off_out : bp.line_off)[task.first + c];
    }
    __syncthreads();
    switch (s_len.kind) {
      case BK_MIXED: batch_mixed(bp, s_len, s_base, s_obase, task.count, A, B, tid, T); break;
      case BK_RADER:
        batch_rader(bp, s_len, s_base, s_obase, task.count, A, B, x0s, X0s, tid, T);
        break;
      case BK_BLUE: batch_blue(bp, s_len, s_base, s_obase, task.count, A, B, tid, T); break;
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
