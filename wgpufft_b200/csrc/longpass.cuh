// Long lines of a batch (a line, or a Bluestein convolution, too long for
// one CTA's shared memory): two or three HBM passes of a persistent kernel.
//
// A length T = N1 * N2 FFT (T = N, or the convolution length M) runs as
//   column pass: for each n2, FFT_N1 over n1 of x[N2 n1 + n2], times
//                W_T^{n2 k1}, into the scratch row k1 (natural [k1][n2]);
//   row pass:    for each k1, FFT_N2 over n2 of scratch row k1, giving
//                X[k1 + N1 k2].
// A task is G (16, 8 or 4) adjacent columns or rows of one line, so every
// global access is a segment of G consecutive complex values (128 bytes at
// G = 16): rows of columns n2..n2+G-1, or the outputs k1..k1+G-1 of one k2.
// The G lines of a task sit interleaved in shared memory, element (i, l) at
// i*(G+1) + l: the 16 threads of a half-warp take the same position i of 16
// lines, so the Stockham stages and the column segments are conflict-free,
// and the pitch G+1 keeps the transposed row loads (consecutive i, fixed l)
// conflict-free too.  Each thread keeps one line l and walks the butterflies
// j = s, s+S, ... of every stage with incrementally updated offsets.
//
// Bluestein lines (convolution M = N1 N2) take three passes: the chirped
// column pass; a middle row pass that runs the forward row FFT, multiplies
// by the chirp spectrum, and runs the row half of the inverse FFT
// (y[N2 n1 + n2] = sum_k1 W_N1^{-n1 k1} W_M^{-n2 k1} sum_k2 W_N2^{-n2 k2} Y[k1 + N1 k2],
// computed on conjugates with the forward codelets) in place on the rows;
// and the inverse column pass, chirped into the output.  One scratch region
// of M values per line.
//
// Loads are asynchronous (cp.async): while a CTA transforms one task, the
// copies of its next task are already in flight into the other landing
// buffer, together with the twiddle tables of its length (stage twiddles,
// W_M^{a N2} and W_M^b) when they differ from the ones that buffer last
// held.  The work queue hands out chunks of consecutive tasks (mostly one
// line), so the tables change rarely; nothing waits on another CTA.
#pragma once
#include "batch.cuh"

namespace b2f {

constexpr uint32_t kLongThreads = 256;
constexpr uint32_t kLongThreadsLog2 = 8;
static_assert(kLongThreads == 1u << kLongThreadsLog2, "thread count is a power of two");
constexpr int kLongMaxStages = 10;  // pass lengths <= 512
constexpr uint32_t kLongChunk = 4;  // consecutive tasks per work-queue claim
// k_long_pass claims the first two chunks before its loop and every later
// one when the chunk before it opens (three tasks ahead): that covers every
// chunk only when a chunk holds at least three tasks
static_assert(kLongChunk >= 3, "the prologue claims chunks 0 and 1 only");
// table area of one landing buffer (complex values): stage twiddles of the
// pass (length - 1 <= 511), W_M^{a N2} (a < N1 <= 512), W_M^b (b < N2 <= 512);
// the Bluestein inverse column pass holds the chirp tables W_2N^{a B} and
// W_2N^b (B = ceil(sqrt(2N)) <= 512) where the last two are
constexpr uint32_t kTabSt = 0, kTabTa = 512, kTabTb = 1024;
constexpr uint32_t kLongTab = 1536;

enum LongPassKind : uint32_t {
  LP_COL = 0,    // smooth line, column pass: x -> scratch
  LP_ROW = 1,    // smooth line, row pass: scratch -> out
  LP_BCOL1 = 2,  // Bluestein, chirped column pass: x -> scratch
  LP_BMID = 3,   // Bluestein, rows: FFT, spectrum product, inverse-row FFT, in place
  LP_BCOL3 = 4,  // Bluestein, inverse column pass, chirped: scratch -> out
};

struct LongSched {
  uint32_t nst;
  StageDesc st[kLongMaxStages];
};

struct LongLenDesc {
  uint32_t N, M, N1, N2;
  uint32_t lgc, lgr;  // log2 of the lines per column / row task
  uint32_t blue;
  float scale;
  const c32* bhat;    // Bluestein: spectrum of the conjugate chirp / M, natural order
  // two-level tables (offsets into the twiddle table) with rows of
  // L = 2^tsplit >= sqrt(M): W_M^j = W_M^{L a} * W_M^b, j = a L + b,
  // a < ceil(M / L) <= 512, b < L <= 512; the Bluestein chirp W_2N^q
  // likewise with rows of 2^csplit >= sqrt(2N)
  uint32_t ta, tb, tsplit;
  uint32_t ca, cb, csplit;
  LongSched s1, s2;   // schedules of N1 (columns) and N2 (rows)
};

// One task: G adjacent columns or rows of one line.  Self-contained, so
// that the kernel can prefetch it with asynchronous copies (no dependent
// load of a line record).
struct LongTask {
  uint64_t base;     // complex offset of the line in the input buffer
  uint64_t scratch;  // complex offset of its scratch region (M values)
  uint32_t len;      // index into the length table
  uint32_t g0;       // first column (column passes) or row (row passes) of the task
  uint64_t obase;    // complex offset of the line in the output buffer
};
static_assert(sizeof(LongTask) == 32, "task records are copied as four 8-byte words");

struct LongParams {
  const c32* in;
  c32* out;
  c32* scratch;
  const c32* tw;
  const LongLenDesc* lens;
  const LongTask* tasks;
  uint32_t ntasks;
  uint32_t phase;    // 1: column pass, 2: row pass, 3: Bluestein inverse columns
  uint32_t inverse;
  uint32_t cap;      // complex elements per shared-memory buffer
  unsigned int* counter;  // work queue: chunks of kLongChunk tasks handed out in order
};

FFT_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
FFT_D void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

FFT_D uint32_t long_kind(uint32_t phase, bool blue) {
  if (phase == 1) return blue ? LP_BCOL1 : LP_COL;
  if (phase == 2) return blue ? LP_BMID : LP_ROW;
  return LP_BCOL3;
}

// W^j from a two-level table with rows of 2^sh: j = a*2^sh + b, value
// ta[a] * tb[b] (a shift and a mask, no division).
FFT_D c32 tw_two(const c32* __restrict__ tw, uint32_t ta, uint32_t tb, uint32_t j, uint32_t sh) {
  return cmul(tw[ta + (j >> sh)], tw[tb + (j & ((1u << sh) - 1))]);
}

// Where the last stage of a pass puts its results: back into shared memory
// (EpiNone), or straight from registers to global memory, the R outputs
// v[r] of one butterfly of line l at positions o + r*Ns: the column pass's
// scratch store with the inter-pass twiddle (EpiCol), the row pass's output
// store (EpiRow).  Addresses and twiddle exponents advance by a fixed step
// per output.  A half-warp holds one position of 16 lines, so each store is
// one G-value segment.
struct EpiNone {
  static constexpr bool active = false;
  template <int R>
  FFT_D void store(uint32_t, uint32_t, const c32*) const {}
};
struct EpiCol {  // scratch[N2 pos + c] = v * W_M^{c pos}
  static constexpr bool active = true;
  c32* dst;  // scratch of the line + c
  const c32* T;
  uint32_t N2, c, sh;
  bool ok;
  template <int R>
  FFT_D void store(uint32_t o, uint32_t Ns, const c32* v) const {
    if (!ok) return;
    uint32_t e = c * o;  // c * pos < M
    const uint32_t de = c * Ns;
    c32* dp = dst + (uint64_t)N2 * o;
    const uint64_t step = (uint64_t)N2 * Ns;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      *dp = cmul(v[r], tw_two(T, kTabTa, kTabTb, e, sh));
      e += de;
      dp += step;
    }
  }
};
struct EpiRow {  // out[k1 + N1 pos], scaled, conjugated back for inverse transforms
  static constexpr bool active = true;
  c32* dst;  // out of the line + k1
  uint32_t N1;
  float sc, sci;  // scale of the real and imaginary parts (sci = -sc for inverse)
  bool ok;
  template <int R>
  FFT_D void store(uint32_t o, uint32_t Ns, const c32* v) const {
    if (!ok) return;
    c32* dp = dst + (uint64_t)N1 * o;
    const uint64_t step = (uint64_t)N1 * Ns;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      *dp = c32{v[r].re * sc, v[r].im * sci};
      dp += step;
    }
  }
};

// One radix-R stage over G interleaved lines, src -> dst (or, for the last
// stage with an active epilogue, src -> epi): thread (l, s) runs the
// butterflies j = s, s+S, ... of line l; k = j mod Ns advances by S mod Ns.
// tws: this stage's twiddles, row k at k*(R-1).
template <int R, class Epi>
FFT_D void ilv_stage(const c32* __restrict__ src, c32* __restrict__ dst, const StageDesc& sd,
                     uint32_t lg, uint32_t tid, const c32* __restrict__ tws, bool to_epi,
                     const Epi& epi) {
  const uint32_t G = 1u << lg, P = G + 1;
  const uint32_t l = tid & (G - 1), s = tid >> lg, S = kLongThreads >> lg;
  const uint32_t NR = sd.NR, Ns = sd.Ns;
  if (s >= NR) return;
  const uint32_t qs = NR * P, rs = Ns * P;
  uint32_t k = 0, kinc = 0;
  if (Ns > 1) {
    k = s - fdiv(s, sd.dNs) * Ns;
    kinc = S - fdiv(S, sd.dNs) * Ns;
  }
#pragma unroll(R <= 8 ? 2 : 1)
  for (uint32_t j = s; j < NR; j += S) {
    const c32* sb = src + j * P + l;
    c32 v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = sb[q * qs];
    if (Ns > 1) {
      const c32* t = tws + k * (R - 1);
#pragma unroll
      for (int q = 1; q < R; ++q) v[q] = cmul(v[q], t[q - 1]);
    }
    dft<float, R>(v);
    const uint32_t o = (j - k) * R + k;
    if (Epi::active && to_epi) {
      epi.template store<R>(o, Ns, v);
    } else {
      c32* db = dst + o * P + l;
#pragma unroll
      for (int r = 0; r < R; ++r) db[r * rs] = v[r];
    }
    k += kinc;
    if (k >= Ns) k -= Ns;
  }
}

// The whole schedule, a <-> b; returns the buffer holding the result (with
// an active epilogue the last stage goes to epi and the return value is
// meaningless).  T: the table area (stage twiddles from offset kTabSt,
// global table offsets relative to the first stage's).  The caller
// synchronises before; every stage that writes shared memory ends with a
// barrier.
template <class Epi>
FFT_D c32* ilv_fft(c32* a, c32* b, const LongSched& sch, uint32_t lg, uint32_t tid, const c32* T,
                   const Epi& epi) {
  const uint32_t tw0 = sch.st[0].tw_off;
#pragma unroll 1
  for (uint32_t s = 0; s < sch.nst; ++s) {
    const StageDesc& sd = sch.st[s];
    const c32* tws = T + kTabSt + (sd.tw_off - tw0);
    const bool to_epi = Epi::active && s + 1 == sch.nst;
    switch (sd.R) {
      case 2: ilv_stage<2>(a, b, sd, lg, tid, tws, to_epi, epi); break;
      case 3: ilv_stage<3>(a, b, sd, lg, tid, tws, to_epi, epi); break;
      case 4: ilv_stage<4>(a, b, sd, lg, tid, tws, to_epi, epi); break;
      case 5: ilv_stage<5>(a, b, sd, lg, tid, tws, to_epi, epi); break;
      case 7: ilv_stage<7>(a, b, sd, lg, tid, tws, to_epi, epi); break;
      case 8: ilv_stage<8>(a, b, sd, lg, tid, tws, to_epi, epi); break;
      case 9: ilv_stage<9>(a, b, sd, lg, tid, tws, to_epi, epi); break;
      case 11: ilv_stage<11>(a, b, sd, lg, tid, tws, to_epi, epi); break;
      case 13: ilv_stage<13>(a, b, sd, lg, tid, tws, to_epi, epi); break;
      case 16: ilv_stage<16>(a, b, sd, lg, tid, tws, to_epi, epi); break;
      default: break;
    }
    if (to_epi) break;
    __syncthreads();
    c32* t = a;
    a = b;
    b = t;
  }
  return a;
}

// x mod m for x < 2^50, m < 2^32, inv = 1/m rounded to double: the
// quotient estimate trunc(x * inv) is off by at most one (its relative
// error is below 2^-51, x / m below 2^50), so one correction either way
// gives the remainder.  A 64-bit integer modulo is a long software routine
// on the GPU; this is a few instructions.
FFT_D uint32_t mod_u50(uint64_t x, uint32_t m, double inv) {
  const uint64_t q = (uint64_t)((double)x * inv);
  int64_t r = (int64_t)x - (int64_t)(q * m);
  if (r < 0) r += m;
  else if (r >= (int64_t)m) r -= m;
  return (uint32_t)r;
}

// Chirp exp(-i pi n^2 / N) at n, n + D, n + 2D, ... : q = n^2 mod 2N kept
// incrementally ((n + D)^2 = n^2 + 2nD + D^2); W_2N^q from the length's
// two-level chirp table (q = a B + b: ca[a] * cb[b]), read through the
// read-only cache (value_ldg) or from a shared-memory copy (value).
// n < 2^24 and D < 2^24 (the residues below need n^2, 2nD, 2D^2 < 2^50).
struct ChirpWalk {
  uint32_t q, u, dsq, u2, twoN, sh, mask;
  const c32* ca;
  const c32* cb;
  FFT_D void init(uint64_t n, uint32_t D, uint32_t N, const c32* ta, const c32* tb,
                  uint32_t split) {
    ca = ta;
    cb = tb;
    sh = split;
    mask = (1u << split) - 1;
    twoN = 2 * N;
    const double inv = 1.0 / (double)twoN;
    q = mod_u50(n * n, twoN, inv);
    u = mod_u50(2 * n * (uint64_t)D, twoN, inv);
    dsq = mod_u50((uint64_t)D * D, twoN, inv);
    u2 = mod_u50(2 * (uint64_t)D * D, twoN, inv);
  }
  FFT_D void step() {
    q += u;
    if (q >= twoN) q -= twoN;
    q += dsq;
    if (q >= twoN) q -= twoN;
    u += u2;
    if (u >= twoN) u -= twoN;
  }
  FFT_D c32 value_ldg() const {
    const float2 x = __ldg(reinterpret_cast<const float2*>(ca + (q >> sh)));
    const float2 y = __ldg(reinterpret_cast<const float2*>(cb + (q & mask)));
    return cmul(c32{x.x, x.y}, c32{y.x, y.y});
  }
  FFT_D c32 value() const { return cmul(ca[q >> sh], cb[q & mask]); }
};

FFT_D void copy_async(c32* dst, const c32* src, uint32_t n, uint32_t tid) {
  for (uint32_t e = tid; e < n; e += kLongThreads) cp_async8(dst + e, src + e);
}

// Issues the copies of one task into the landing buffer X (zero-filled
// where the task has no data) and, with tables, of its length's twiddle
// tables into the table area T.
FFT_D void long_issue(const LongParams& p, const LongLenDesc& d, const LongTask& ln, uint32_t kind,
                      c32* X, c32* T, bool tables, uint32_t tid) {
  const uint32_t g0 = ln.g0;
  const bool colk = kind == LP_COL || kind == LP_BCOL1 || kind == LP_BCOL3;
  if (tables) {
    const LongSched& sch = colk ? d.s1 : d.s2;
    const uint32_t nx = colk ? d.N1 : d.N2;
    copy_async(T + kTabSt, p.tw + sch.st[0].tw_off, nx - 1, tid);
    if (kind == LP_COL || kind == LP_BCOL1 || kind == LP_BMID) {
      copy_async(T + kTabTa, p.tw + d.ta, (d.M + (1u << d.tsplit) - 1) >> d.tsplit, tid);
      copy_async(T + kTabTb, p.tw + d.tb, 1u << d.tsplit, tid);
    } else if (kind == LP_BCOL3) {
      // the chirp tables (ceil(2N / B) <= B <= 512 values each) in their place
      copy_async(T + kTabTa, p.tw + d.ca, (2 * d.N + (1u << d.csplit) - 1) >> d.csplit, tid);
      copy_async(T + kTabTb, p.tw + d.cb, 1u << d.csplit, tid);
    }
  }
  if (colk) {
    // columns g0..g0+G-1: row n1 is the segment src[N2 n1 + g0 + l]; rows
    // n1 < nv of column c hold data (N2 n1 + c < lim), the rest are zeros
    // (columns past N2, the zero-padded half of a chirped column) written
    // directly: this buffer's previous task finished before the barrier
    const uint32_t lg = d.lgc, G = 1u << lg, P = G + 1;
    const uint32_t l = tid & (G - 1), S = kLongThreads >> lg;
    const uint32_t N2 = d.N2, Nx = d.N1;
    const uint32_t c = g0 + l;
    const c32* src = (kind == LP_BCOL3) ? p.scratch + ln.scratch : p.in + ln.base;
    const uint32_t lim = (kind == LP_BCOL1) ? d.N : d.M;  // chirped pass: zero beyond the line
    const uint32_t nv = c < N2 ? min(Nx, (lim - c + N2 - 1) / N2) : 0u;
    uint32_t i = tid >> lg;
    c32* dp = X + i * P + l;
    const c32* sp = src + ((uint64_t)N2 * i + c);
    const uint64_t sstep = (uint64_t)S * N2;
#pragma unroll 4
    for (; i < nv; i += S) {
      cp_async8(dp, sp);
      sp += sstep;
      dp += S * P;
    }
    for (; i < Nx; i += S) {
      *dp = czero<float>();
      dp += S * P;
    }
  } else {
    // rows g0..g0+G-1 of the scratch: kLongThreads / G threads per row
    // (a half-warp, a warp or two), each a run of consecutive values;
    // rows past N1 are zeros
    const uint32_t lg = d.lgr, P = (1u << lg) + 1;
    const uint32_t N2 = d.N2, N1 = d.N1;
    const uint32_t tpr = kLongThreads >> lg, r = tid >> (kLongThreadsLog2 - lg), lane = tid & (tpr - 1);
    c32* dp = X + lane * P + r;
    if (g0 + r < N1) {
      const c32* sp = p.scratch + ln.scratch + (uint64_t)(g0 + r) * N2 + lane;
#pragma unroll 4
      for (uint32_t n2 = lane; n2 < N2; n2 += tpr) {
        cp_async8(dp, sp);
        sp += tpr;
        dp += tpr * P;
      }
    } else {
      for (uint32_t n2 = lane; n2 < N2; n2 += tpr) {
        *dp = czero<float>();
        dp += tpr * P;
      }
    }
  }
}

// Transforms the task whose data sits in X (W: the ping-pong partner, T:
// its table area) and stores its results.  Ends without a barrier.
FFT_D void long_compute(const LongParams& p, const LongLenDesc& d, const LongTask& ln, uint32_t kind,
                        c32* X, c32* W, const c32* T, uint32_t tid) {
  const uint32_t g0 = ln.g0;
  const bool inv = p.inverse != 0;
  const bool colk = kind == LP_COL || kind == LP_BCOL1 || kind == LP_BCOL3;
  const uint32_t lg = colk ? d.lgc : d.lgr, G = 1u << lg, P = G + 1;
  const uint32_t l = tid & (G - 1), S = kLongThreads >> lg, i0 = tid >> lg;
  const uint32_t N1 = d.N1, N2 = d.N2;
  // input conjugation (inverse transforms) and the chirp of the first
  // Bluestein pass, in place
  if (kind == LP_BCOL1) {
    const uint32_t c = g0 + l;
    if (c < N2) {
      uint32_t n = N2 * i0 + c;
      ChirpWalk cw;
      cw.init(n, S * N2, d.N, p.tw + d.ca, p.tw + d.cb, d.csplit);
      c32* dp = X + i0 * P + l;
      const uint32_t dn = S * N2;
      uint32_t i = i0;
      // four chirp values' loads in flight together
      constexpr int U = 4;
      for (; i + (U - 1) * S < N1 && n + (U - 1) * dn < d.N; i += U * S) {
        c32 w[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          w[u] = cw.value_ldg();
          cw.step();
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          c32 v = dp[u * S * P];
          if (inv) v.im = -v.im;
          dp[u * S * P] = cmul(v, w[u]);
        }
        n += U * dn;
        dp += U * S * P;
      }
      for (; i < N1 && n < d.N; i += S) {
        c32 v = *dp;
        if (inv) v.im = -v.im;
        *dp = cmul(v, cw.value_ldg());
        cw.step();
        n += dn;
        dp += S * P;
      }
    }
    __syncthreads();
  } else if (kind == LP_COL && inv) {
    for (uint32_t e = tid; e < N1 * P; e += kLongThreads) X[e].im = -X[e].im;
    __syncthreads();
  }
  const LongSched& sch = colk ? d.s1 : d.s2;
  if (kind == LP_COL || kind == LP_BCOL1) {
    // scratch[k1][g0 + l] = X[k1] * W_M^{(g0+l) k1}, from the last stage
    EpiCol e;
    e.c = g0 + l;
    e.ok = e.c < N2;
    e.dst = p.scratch + ln.scratch + (e.ok ? e.c : 0);
    e.sh = d.tsplit;
    e.T = T;
    e.N2 = N2;
    ilv_fft(X, W, sch, lg, tid, T, e);
    return;
  }
  if (kind == LP_ROW) {
    // out[k1 + N1 k2], k1 = g0 + l, from the last stage
    EpiRow e;
    e.ok = g0 + l < N1;
    e.dst = p.out + ln.obase + (e.ok ? g0 + l : 0);
    e.N1 = N1;
    e.sc = d.scale;
    e.sci = inv ? -d.scale : d.scale;
    ilv_fft(X, W, sch, lg, tid, T, e);
    return;
  }
  c32* r = X;
  c32* o = W;
  // the Bluestein middle pass multiplies by the chirp spectrum at
  // k = k1 + N1 k2 (k1 = g0 + l, k2 = i0 + m S): its values are loaded into
  // registers now, so the loads overlap the first FFT (m < ceil(N2 / S) <= 13
  // for the row-task shapes: G = 16 up to 208 points, 8 up to 393, 4 up to 512)
  constexpr int kBh = 13;
  c32 bhv[kBh];
  const uint32_t k1m = g0 + l;
  if (kind == LP_BMID) {
    const c32* bh = d.bhat + (k1m < N1 ? k1m : 0) + (uint64_t)N1 * i0;
#pragma unroll
    for (int m = 0; m < kBh; ++m)
      bhv[m] = (i0 + m * S < N2) ? bh[(uint64_t)m * S * N1] : czero<float>();
  }
  // one FFT; the Bluestein middle pass runs two with the conjugated spectrum
  // product between them: the forward row FFT of the conjugate is the
  // inverse row FFT
  const int nfft = kind == LP_BMID ? 2 : 1;
#pragma unroll 1
  for (int f = 0; f < nfft; ++f) {
    c32* res = ilv_fft(r, o, sch, lg, tid, T, EpiNone());
    o = (res == r) ? o : r;
    r = res;
    if (f + 1 == nfft) break;
    if (k1m < N1) {
      c32* dp = r + i0 * P + l;
#pragma unroll
      for (int m = 0; m < kBh; ++m) {
        if (i0 + m * S < N2) {
          c32 v = cmul(dp[m * S * P], bhv[m]);
          v.im = -v.im;
          dp[m * S * P] = v;
        }
      }
    }
    __syncthreads();
  }
  // stores
  if (kind == LP_BMID) {
    // scratch row k1 = g0 + rr, position n2: V * W_M^{n2 k1}
    // (kLongThreads / G threads per row, each a run of consecutive values)
    const uint32_t tpr = kLongThreads >> lg, rr = tid >> (kLongThreadsLog2 - lg), lane = tid & (tpr - 1);
    const uint32_t k1 = g0 + rr;
    if (k1 < N1) {
      c32* row = p.scratch + ln.scratch + (uint64_t)k1 * N2;
      const c32* sp = r + lane * P + rr;
#pragma unroll 4
      for (uint32_t n2 = lane; n2 < N2; n2 += tpr) {
        row[n2] = cmul(*sp, tw_two(T, kTabTa, kTabTb, n2 * k1, d.tsplit));
        sp += tpr * P;
      }
    }
  } else {  // LP_BCOL3: out[n] = conj(Y[n]) * chirp(n), n = N2 n1 + g0 + l < N
    const uint32_t c = g0 + l;
    if (c < N2) {
      const float sc = d.scale;
      uint32_t n = N2 * i0 + c;
      ChirpWalk cw;
      cw.init(n, S * N2, d.N, T + kTabTa, T + kTabTb, d.csplit);
      c32* dst = p.out + ln.obase + n;
      const c32* sp = r + i0 * P + l;
      for (uint32_t n1 = i0; n1 < N1 && n < d.N; n1 += S) {
        c32 wv = *sp;
        wv.im = -wv.im;
        c32 v = cmul(wv, cw.value());
        v.re *= sc;
        v.im = inv ? -v.im * sc : v.im * sc;
        *dst = v;
        cw.step();
        n += S * N2;
        dst += (uint64_t)S * N2;
        sp += S * P;
      }
    }
  }
}

// Persistent kernel of one long-line phase.  CTAs take chunks of
// kLongChunk consecutive tasks from a work queue (one atomicAdd per
// chunk), claimed a chunk ahead: the claim for the CTA's chunk c + 1 is
// issued when it starts using chunk c and its result is stored after that
// iteration's transform, so the atomic's latency is hidden too.  While
// iteration k transforms the CTA's task k, asynchronous copies run three
// stages ahead: the data and tables of task k + 1 (into the other landing
// buffer), the length descriptor of task k + 2 (a ring of three) and the
// record of task k + 3 (a ring of four), committed as one group and
// waited for at the top of iteration k + 1, so no descriptor load sits on
// the critical path.
// One instantiation per phase PH (= p.phase), so each holds only the code
// of its two task kinds.  Dynamic shared memory: two landing buffers and
// one work buffer of p.cap complex values, then the two table areas of
// kLongTab values (one per landing buffer).
template <uint32_t PH>
__global__ void __launch_bounds__(kLongThreads, 2) k_long_pass(const __grid_constant__ LongParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ LongLenDesc s_len[3];
  __shared__ LongTask s_task[4];
  __shared__ uint32_t s_chunk[4];  // first task of the CTA's chunk c, at c % 4
  static_assert(sizeof(LongLenDesc) % 8 == 0, "descriptors are copied as 8-byte words");
  c32* const base = reinterpret_cast<c32*>(smem_raw);
  c32* const work = base + 2 * p.cap;
  c32* const tab = base + 3 * p.cap;
  const uint32_t tid = threadIdx.x;
  constexpr uint32_t kNone = 0xFFFFFFFFu;
  // the CTA's k-th task (its chunk claimed and visible); kNone from the
  // first one past the end (the queue hands out chunks in increasing order)
  auto task_of = [&](uint32_t k) -> uint32_t {
    const uint64_t t = (uint64_t)s_chunk[(k / kLongChunk) & 3] + k % kLongChunk;
    return t < p.ntasks ? (uint32_t)t : kNone;
  };
  if (tid == 0) {
    s_chunk[0] = atomicAdd(p.counter, 1u) * kLongChunk;
    s_chunk[1] = atomicAdd(p.counter, 1u) * kLongChunk;
  }
  __syncthreads();
  uint32_t held0 = kNone, held1 = kNone;        // length whose tables landing buffer 0/1 holds
  uint32_t ring0 = kNone, ring1 = kNone, ring2 = kNone;  // length each descriptor slot holds
  // record of task k into s_task[k % 4]
  auto fetch_task = [&](uint32_t k) {
    const uint32_t t = task_of(k);
    if (t != kNone && tid < 4)
      cp_async8(reinterpret_cast<uint64_t*>(&s_task[k & 3]) + tid,
                reinterpret_cast<const uint64_t*>(p.tasks + t) + tid);
  };
  // length descriptor of task k (whose record has landed) into s_len[k % 3],
  // unless that slot holds it already
  auto fetch_len = [&](uint32_t k) {
    if (task_of(k) == kNone) return;
    const uint32_t len = s_task[k & 3].len, r = k % 3;
    const uint32_t had = r == 0 ? ring0 : (r == 1 ? ring1 : ring2);
    if (had == len) return;
    if (r == 0) ring0 = len;
    else if (r == 1) ring1 = len;
    else ring2 = len;
    const uint64_t* src = reinterpret_cast<const uint64_t*>(p.lens + len);
    uint64_t* dst = reinterpret_cast<uint64_t*>(&s_len[r]);
    for (uint32_t i = tid; i < sizeof(LongLenDesc) / 8; i += kLongThreads)
      cp_async8(dst + i, src + i);
  };
  // data of task k (whose record and descriptor have landed) into landing
  // buffer k % 2, with its length's tables when that buffer's differ
  auto fetch_data = [&](uint32_t k) {
    if (task_of(k) == kNone) return;
    const LongTask& tk = s_task[k & 3];
    const LongLenDesc& d = s_len[k % 3];
    const uint32_t slot = k & 1;
    const bool tables = tk.len != (slot ? held1 : held0);
    if (slot) held1 = tk.len;
    else held0 = tk.len;
    long_issue(p, d, tk, long_kind(PH, d.blue != 0), base + slot * p.cap, tab + slot * kLongTab,
               tables, tid);
  };
  fetch_task(0);
  fetch_task(1);
  fetch_task(2);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  fetch_len(0);
  fetch_len(1);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  fetch_data(0);
  cp_async_commit();
#pragma unroll 1
  for (uint32_t k = 0; task_of(k) != kNone; ++k) {
    cp_async_wait<0>();
    __syncthreads();  // task k's data, k + 1's descriptor and k + 2's record have landed,
                      // and every thread is past task k - 1
    // task k + 3 opens chunk c = (k + 3) / kLongChunk: claim chunk c + 1
    const bool claim = tid == 0 && (k + 3) % kLongChunk == 0;
    const uint32_t claimed = claim ? atomicAdd(p.counter, 1u) * kLongChunk : 0u;
    fetch_data(k + 1);
    fetch_len(k + 2);
    fetch_task(k + 3);
    cp_async_commit();
    const LongLenDesc& d = s_len[k % 3];
    const uint32_t slot = k & 1;
    long_compute(p, d, s_task[k & 3], long_kind(PH, d.blue != 0), base + slot * p.cap, work,
                 tab + slot * kLongTab, tid);
    // first read at iteration k + 4, after the barriers between
    if (claim) s_chunk[((k + 3) / kLongChunk + 1) & 3] = claimed;
  }
  cp_async_wait<0>();
}

}  // namespace b2f
