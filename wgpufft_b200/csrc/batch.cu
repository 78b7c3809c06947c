// Batched launch of many 1D f32 lines of mixed lengths: host planner and
// C ABI (b2f_batch_*).  The lines of all the transforms share persistent
// launches driven by device work queues; the reference has no counterpart
// (it records one dispatch chain per plan).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <thread>

#include "batch.cuh"
#include "longpass.cuh"
#include "hostfft.h"
#include "linebatch.h"
#include "plan.h"

namespace b2f {

static bool smooth7(uint64_t n) {
  if (n == 0) return false;
  for (uint64_t r : {2, 3, 5, 7})
    while (n % r == 0) n /= r;
  return n == 1;
}

static uint32_t ld_f32(uint64_t n) { return (uint32_t)(n + (n >> 4) + 1); }

static Schedule schedule_for(uint64_t n) {
  Schedule sch;
  std::memset(&sch, 0, sizeof(sch));
  const std::vector<uint32_t> rad = stage_radices(n);
  sch.N = (uint32_t)n;
  sch.nst = (uint32_t)rad.size();
  uint64_t Ns = 1;
  for (size_t s = 0; s < rad.size(); ++s) {
    StageDesc& d = sch.st[s];
    d.R = rad[s];
    d.Ns = (uint32_t)Ns;
    d.NR = (uint32_t)(n / rad[s]);
    d.tw_off = 0;
    d.dNs = make_fastdiv((uint32_t)Ns);
    d.dNR = make_fastdiv((uint32_t)(n / rad[s]));
    Ns *= rad[s];
  }
  return sch;
}

// Appends the stage twiddles of sch (rows k*(R-1) + q-1 per stage) to tw
// once per FFT length and points the stages at them.
static void attach_stage_table(Schedule& sch, std::vector<cd>& tw,
                               std::map<uint32_t, uint32_t>& cache) {
  auto it = cache.find(sch.N);
  uint32_t base;
  if (it != cache.end()) {
    base = it->second;
  } else {
    base = (uint32_t)tw.size();
    cache[sch.N] = base;
    for (uint32_t s = 0; s < sch.nst; ++s) {
      const uint32_t R = sch.st[s].R, Ns = sch.st[s].Ns;
      for (uint64_t k = 0; k < Ns; ++k)
        for (uint32_t q = 1; q < R; ++q) tw.push_back(root_fwd(q * k, (uint64_t)Ns * R));
    }
  }
  uint32_t off = base;
  for (uint32_t s = 0; s < sch.nst; ++s) {
    sch.st[s].tw_off = off;
    off += sch.st[s].Ns * (sch.st[s].R - 1);
  }
}

static uint64_t mod_pow64(uint64_t b, uint64_t e, uint64_t m) {
  uint64_t r = 1;
  b %= m;
  while (e) {
    if (e & 1) r = (unsigned __int128)r * b % m;
    b = (unsigned __int128)b * b % m;
    e >>= 1;
  }
  return r;
}

// Host-buffer execution (b2f_batch_execute_host) pipelines the lines in
// chunks: contiguous runs of lines (in offset order), about kHostChunkBytes
// each and at most kHostChunks (smaller at both ends), each copied in,
// transformed and copied out on its own (smaller chunks shorten the
// pipeline's fill and drain, which are all that the copies do not hide).
constexpr uint32_t kHostChunks = 32;
constexpr uint64_t kHostChunkBytes = 32ull << 20;
// Copy boundaries are rounded down to multiples of 4 KiB: copies out to
// pinned host memory that start and end at arbitrary 8-byte offsets ran
// 7 % slower alone and 10-14 % slower beside the copies in (32 chunks of the
// 1.27 GB mixed-length workload: 29.2 against 27.5 ms for both directions)
constexpr uint64_t kHostCopyAlign = 4096;
constexpr uint32_t kNoWait = 0xFFFFFFFFu;
// work-queue counters, zeroed by every execute: [0] CTA queue, [1] and [2]
// cluster queues, [4 + ph] long-line phase ph; per chunk c of a host
// execution, [8 + 4c] its CTA tasks and [9 + 4c + ph] its long phase ph
constexpr unsigned kBatchCounters = 8 + 4 * kHostChunks;

struct BatchPlan {
  int device = 0;
  int32_t direction = B2F_FORWARD, normalization = B2F_NORM_INVERSE;
  uint64_t nlines = 0, extent = 0;  // extent: complex elements the buffers must hold
  // device state
  BatchLen* d_lens = nullptr;
  BatchTask* d_tasks = nullptr;  // CTA tasks then cluster tasks
  BatchTask* d_tasks_chunked = nullptr;  // CTA tasks chunk by chunk
  uint64_t* d_off = nullptr;
  unsigned int* d_counters = nullptr;  // [0] CTA queue, [1] cluster queue
  std::vector<void*> tables;
  uint32_t n_cta = 0, n_cl = 0, n_big = 0;
  // long lines (k_long_pass): length descriptors, lines, and the tasks of
  // the column, row and Bluestein inverse-column phases, one launch each
  LongLenDesc* d_long_lens = nullptr;
  LongTask* d_long_tasks = nullptr;
  LongTask* d_long_tasks_chunked = nullptr;
  uint32_t long_first[3] = {0, 0, 0}, long_count[3] = {0, 0, 0};
  // chunks of host execution: element ranges [chunk_lo, chunk_hi) of the
  // buffers, and each chunk's tasks (CTA queue; long phases, relative to
  // long_first) -- every task list is ordered by chunk
  uint32_t n_chunks = 1;  // chunks in use (<= kHostChunks)
  uint64_t chunk_lo[kHostChunks] = {}, chunk_hi[kHostChunks] = {};
  // the copies: piece j = bytes [piece_lo, piece_hi), cut at kHostCopyAlign
  // multiples near the chunk boundaries; chunk c's transform waits for the
  // copy in of piece in_wait[c], piece j's copy out for the transform of
  // chunk out_wait[j] (kNoWait: none)
  uint64_t piece_lo[kHostChunks] = {}, piece_hi[kHostChunks] = {};
  uint32_t in_wait[kHostChunks] = {}, out_wait[kHostChunks] = {};
  uint32_t cta_cfirst[kHostChunks] = {}, cta_ccount[kHostChunks] = {};
  uint32_t long_cfirst[3][kHostChunks] = {}, long_ccount[3][kHostChunks] = {};
  cudaStream_t hs[3] = {nullptr, nullptr, nullptr};  // copy in, transform, copy out
  cudaEvent_t hev_start = nullptr, hev_done = nullptr;
  cudaEvent_t hev_in[kHostChunks] = {}, hev_c[kHostChunks] = {};
  uint32_t long_cap = 0;
  size_t smem_long = 0;
  unsigned grid_long = 0;
  uint64_t lines_long = 0, elems_long = 0;
  unsigned grid_big = 0;
  uint32_t buf_cta = 0, buf_cl = 0;
  size_t smem_cta = 0, smem_cl = 0;
  unsigned grid_cta = 0, grid_cl = 0;
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  // description
  uint64_t lines_cta = 0, lines_cl = 0, distinct = 0, table_bytes = 0;
  uint64_t elems_cta = 0, elems_cl = 0;
  c32* d_scratch = nullptr;  // long lines: M values per line
  c32* d_tw = nullptr;
  uint64_t tw_bytes = 0;
  uint64_t scratch_bytes = 0;
  uint64_t kind_lines[7] = {0, 0, 0, 0, 0, 0, 0};
  std::string diag;
  ~BatchPlan() {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    for (void* p : tables) cudaFree(p);
    cudaFree(d_lens);
    cudaFree(d_tasks);
    cudaFree(d_tasks_chunked);
    cudaFree(d_off);
    cudaFree(d_counters);
    cudaFree(d_scratch);
    cudaFree(d_tw);
    cudaFree(d_long_lens);
    cudaFree(d_long_tasks);
    cudaFree(d_long_tasks_chunked);
    if (side) cudaStreamDestroy(side);
    for (auto h : hs)
      if (h) cudaStreamDestroy(h);
    for (uint32_t c = 0; c < kHostChunks; ++c) {
      if (hev_in[c]) cudaEventDestroy(hev_in[c]);
      if (hev_c[c]) cudaEventDestroy(hev_c[c]);
    }
    if (hev_start) cudaEventDestroy(hev_start);
    if (hev_done) cudaEventDestroy(hev_done);
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    if (prev >= 0) cudaSetDevice(prev);
  }
};

constexpr int kClusterP = 8;
constexpr int kClusterBig = 16;  // non-portable cluster size for the longest Bluestein lines
constexpr unsigned kCtaThreads = 256;
constexpr unsigned kClusterThreads = 512;

struct LenInfo {
  BatchLen d;
  std::vector<cd> bhat;
  std::vector<uint32_t> pin, pout;
  double cost = 0;
  LongLenDesc lng;      // long kinds
  Schedule s1, s2;      // long kinds: schedules of N1 and N2
};


// Lines per task of a long-line pass of length nx (log2): 16 up to 208
// points, 8 up to 393, 4 up to 512, so that a task's buffer of nx*(G+1)
// values stays within 3540 (three buffers and the two table areas of two
// CTAs fit one SM).
static uint32_t long_lines_log2(uint64_t nx) { return nx <= 208 ? 4 : (nx <= 393 ? 3 : 2); }

// Estimated cost of one task of a long-line pass of length nx (2..512,
// 13-smooth): for each stage of radix R, the butterfly rounds the task's 256
// threads take (ceil(NR / S) rounds of S threads per line, idle threads
// included) times R points each, weighted by an instruction estimate per
// point (about 10 for the shared-memory traffic, addressing and twiddle
// product, plus the radix-R codelet's arithmetic).  0 for other lengths.
static const std::vector<double>& long_task_costs() {
  static const std::vector<double> tab = [] {
    std::vector<double> t(513, 0.0);
    for (uint32_t nx = 2; nx <= 512; ++nx) {
      const std::vector<uint32_t> rad = stage_radices(nx);
      if (rad.empty()) continue;
      const uint32_t S = kLongThreads >> long_lines_log2(nx);
      double c = 0;
      for (uint32_t R : rad) {
        double f = 0;
        switch (R) {
          case 2: f = 2.0; break;
          case 3: case 4: f = 4.0; break;
          case 5: f = 6.4; break;
          case 7: f = 10.3; break;
          case 8: f = 6.5; break;
          case 9: f = 8.9; break;
          case 11: f = 12.7; break;
          case 13: f = 13.8; break;
          default: f = 9.0; break;  // 16
        }
        const uint32_t rounds = (nx / R + S - 1) / S;
        c += (double)rounds * R * kLongThreads * (10.0 + f);
      }
      t[nx] = c;
    }
    return t;
  }();
  return tab;
}

// Estimated cost of a long line over T = a * (T / a): `ffts` transforms
// through both passes (1 for a smooth line; 2 for Bluestein, forward and
// inverse) and `passes` HBM passes of about 30 instructions per point.
static double long_cost(uint64_t T, uint64_t a, int ffts, int passes) {
  const std::vector<double>& t = long_task_costs();
  const uint64_t b = T / a;
  const uint64_t Ga = 1u << long_lines_log2(a), Gb = 1u << long_lines_log2(b);
  return ffts * (t[a] * (double)((b + Ga - 1) / Ga) + t[b] * (double)((a + Gb - 1) / Gb)) +
         passes * 30.0 * (double)T;
}

// T = N1 * N2 with both factors 13-smooth in [2, 512]: the split of the
// lowest estimated cost (*cost); 0 when none exists.
static uint64_t long_split(uint64_t T, int ffts = 1, int passes = 2, double* cost = nullptr) {
  const std::vector<double>& t = long_task_costs();
  uint64_t best_a = 0;
  double best = 1e300;
  for (uint64_t a = 2; a <= 512; ++a) {
    if (T % a || T / a > 512 || T / a < 2 || t[a] == 0 || t[T / a] == 0) continue;
    const double c = long_cost(T, a, ffts, passes);
    if (c < best) {
      best = c;
      best_a = a;
    }
  }
  if (cost) *cost = best;
  return best_a;
}

// Long-line descriptor of length N over the transform length T = n1 * (T / n1)
// (pass lengths <= 512, so at most 9 stages each).
static void set_long(LenInfo& li, uint64_t N, uint64_t T, uint64_t n1, bool blue) {
  BatchLen& d = li.d;
  LongLenDesc& g = li.lng;
  std::memset(&g, 0, sizeof(g));
  d.kind = blue ? BK_LONG_BLUE : BK_LONG;
  d.M = (uint32_t)T;
  d.G = 1;
  g.N = (uint32_t)N;
  g.M = (uint32_t)T;
  g.N1 = (uint32_t)n1;
  g.N2 = (uint32_t)(T / n1);
  g.lgc = long_lines_log2(g.N1);
  g.lgr = long_lines_log2(g.N2);
  g.blue = blue ? 1u : 0u;
  g.scale = d.scale;
  li.s1 = schedule_for(g.N1);
  li.s2 = schedule_for(g.N2);
}

// The two-level tables of a long line (appended to tw; offsets relative to
// `base`) with rows of L = the power of two >= sqrt(M): W_M^{L a}
// (a < ceil(M / L)) and W_M^b (b < L) for the inter-pass twiddle, and for
// Bluestein lines the chirp W_2N likewise, so the kernel splits an exponent
// with a shift and a mask (M <= 512 * 512 keeps both within 512 values).
static void long_split_tables(LongLenDesc& g, std::vector<cd>& tw, uint64_t base) {
  auto two_level = [&](uint64_t M, uint32_t* ta, uint32_t* tb, uint32_t* split) {
    uint32_t sh = 0;
    while ((1ull << (2 * sh)) < M) ++sh;
    const uint64_t L = 1ull << sh;
    *split = sh;
    *ta = (uint32_t)(base + tw.size());
    for (uint64_t a = 0; a * L < M; ++a) tw.push_back(root_fwd(a * L, M));
    *tb = (uint32_t)(base + tw.size());
    for (uint64_t b = 0; b < L; ++b) tw.push_back(root_fwd(b, M));
  };
  two_level(g.M, &g.ta, &g.tb, &g.tsplit);
  if (g.blue) two_level(2ull * g.N, &g.ca, &g.cb, &g.csplit);
}

// Chooses the execution of one distinct length.
static bool classify(uint64_t N, int32_t direction, int32_t normalization, size_t cta_cap,
                     size_t cl_cap, bool clusters, LenInfo& li) {
  BatchLen& d = li.d;
  std::memset(&d, 0, sizeof(d));
  d.N = (uint32_t)N;
  const bool inv = direction == B2F_INVERSE;
  float sc = 1.0f;
  if ((normalization == B2F_NORM_INVERSE && inv) || (normalization == B2F_NORM_FORWARD && !inv))
    sc = 1.0f / (float)N;
  else if (normalization == B2F_NORM_ORTHOGONAL)
    sc = 1.0f / sqrtf((float)N);
  d.scale = sc;
  d.dN = make_fastdiv((uint32_t)N);
  const auto cta_bytes = [](uint64_t lbuf) { return 2 * (size_t)ld_f32(lbuf) * 8; };
  uint64_t n1 = 0;
  if (is_smooth13(N) && cta_bytes(N) > cta_cap && !clusters) n1 = long_split(N);
  uint32_t cl_split = 0;
  if (clusters && is_smooth13(N) && cta_bytes(N) > cta_cap)
    for (uint32_t P : {8u, 7u, 5u, 4u, 3u, 2u})
      if (N % P == 0 && cta_bytes(N / P) <= cl_cap) {
        cl_split = P;
        break;
      }
  if (cl_split) {
    d.kind = BK_CL_MIXED;
    d.M = (uint32_t)N;
    d.P = cl_split;
    d.L = (uint32_t)(N / cl_split);
    d.LD = ld_f32(d.L);
    d.sch = schedule_for(d.L);
    d.G = 1;
    li.cost = (double)N * std::log2((double)N);
    return true;
  }
  const bool smooth = is_smooth13(N) && (cta_bytes(N) <= cta_cap || n1);
  if (smooth && cta_bytes(N) <= cta_cap) {
    d.kind = BK_MIXED;
    d.M = (uint32_t)N;
    d.LD = ld_f32(N);
    d.sch = schedule_for(N);
  } else if (smooth) {
    set_long(li, N, N, n1, false);
  } else if (is_prime_u64(N) && N >= 3 && is_smooth13(N - 1) && cta_bytes(N) <= cta_cap) {
    d.kind = BK_RADER;
    d.M = (uint32_t)(N - 1);
    d.LD = ld_f32(N);
    d.sch = schedule_for(N - 1);
    d.dP1 = make_fastdiv((uint32_t)(N - 1));
    const uint64_t g = primitive_root(N), ginv = mod_pow64(g, N - 2, N);
    li.pin.resize(N - 1);
    li.pout.resize(N - 1);
    li.bhat.resize(N - 1);
    uint64_t v = 1;
    for (uint64_t q = 0; q + 1 < N; ++q) {
      li.pin[q] = (uint32_t)v;
      v = v * g % N;
    }
    v = 1;
    for (uint64_t r = 0; r + 1 < N; ++r) {
      li.pout[v - 1] = (uint32_t)r;
      li.bhat[r] = root_fwd(v, N);
      v = v * ginv % N;
    }
    host_fft_fwd(li.bhat);
    for (auto& x : li.bhat) x /= (double)(N - 1);
  } else {
    uint64_t M = 2 * N - 1;
    while (!smooth7(M)) ++M;
    uint64_t mlong = 0, a = 0;
    if (cta_bytes(M) > cta_cap && !clusters) {
      // the 13-smooth convolution length in [2N - 1, 2.25 N] (and its split
      // into factors <= 512) of the lowest estimated cost: a slightly longer
      // convolution with fewer, larger-radix stages is often cheaper
      double best = 1e300;
      for (uint64_t m = 2 * N - 1; m <= 262144 && (m <= 9 * N / 4 || !mlong); ++m) {
        if (!is_smooth13(m)) continue;
        double c = 0;
        const uint64_t am = long_split(m, 2, 3, &c);
        if (am && c < best) {
          best = c;
          mlong = m;
          a = am;
        }
      }
    }
    if (cta_bytes(M) <= cta_cap) {
      d.kind = BK_BLUE;
      d.M = (uint32_t)M;
      d.LD = ld_f32(M);
      d.sch = schedule_for(M);
    } else if (mlong) {
      M = mlong;
      set_long(li, N, M, a, true);
    } else {
      // cluster Bluestein: convolution P*L >= 2N-1, L 7-smooth and fitting
      uint32_t P = kClusterP;
      uint64_t L = (2 * N - 1 + P - 1) / P;
      while (!smooth7(L)) ++L;
      if (cta_bytes(L) > cl_cap) {
        P = kClusterBig;
        L = (2 * N - 1 + P - 1) / P;
        while (!smooth7(L)) ++L;
        if (cta_bytes(L) > cl_cap) return false;
      }
      M = L * P;
      d.kind = BK_CL_BLUE;
      d.M = (uint32_t)M;
      d.P = P;
      d.L = (uint32_t)L;
      d.LD = ld_f32(L);
      d.sch = schedule_for(L);
    }
    d.dM = make_fastdiv((uint32_t)M);
    d.dMN = make_fastdiv((uint32_t)(M - N));
    li.bhat = chirp_spectrum(N, M);
  }
  const double T = d.M;
  li.cost = T * std::log2(std::max(2.0, T)) * (d.kind == BK_BLUE || d.kind == BK_CL_BLUE ? 3 : 1);
  if (d.kind == BK_LONG || d.kind == BK_LONG_BLUE) {
    d.G = 1;
  } else if (d.kind == BK_MIXED || d.kind == BK_RADER || d.kind == BK_BLUE) {
    uint64_t G = std::max<uint64_t>(1, 4096 / d.M);
    G = std::min<uint64_t>(G, kBatchMaxG);
    while (G > 1 && G * cta_bytes(d.kind == BK_RADER ? N : d.M) > cta_cap) --G;
    d.G = (uint32_t)G;
  } else {
    d.G = 1;
  }
  return true;
}

// Opts the kernel in to `smem` bytes of dynamic shared memory (needed as
// soon as static plus dynamic shared memory exceeds 48 KB).
template <class K>
static cudaError_t set_smem(K kernel, size_t smem) {
  // the attribute is per kernel for the whole process, shared by every
  // batch and line registry: always raise it to the device's limit, so no
  // later, smaller setting can make another object's launch fail
  // (less the kernel's static shared memory)
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaFuncAttributes fa{};
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
      cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) {
    cudaGetLastError();
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  const int room = optin - (int)fa.sharedSizeBytes;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              std::max<int>(room, (int)smem));
}

static b2f_status create_batch(const uint64_t* lengths, const uint64_t* offsets, uint64_t nlines,
                               int32_t direction, int32_t normalization, int device,
                               uint32_t flags, BatchPlan** out) {
  *out = nullptr;
  if (!lengths || !offsets || nlines == 0) return fail(B2F_ERR_INVALID_ARGUMENT, "empty batch");
  if (direction != B2F_FORWARD && direction != B2F_INVERSE)
    return fail(B2F_ERR_INVALID_ARGUMENT, "direction must be 0 or 1");
  if (normalization < 0 || normalization > 3)
    return fail(B2F_ERR_INVALID_ARGUMENT, "normalization must be 0..=3");
  // lines must be non-empty and disjoint
  std::vector<uint64_t> order(nlines);
  for (uint64_t i = 0; i < nlines; ++i) {
    order[i] = i;
    if (lengths[i] == 0) return fail(B2F_ERR_ZERO_LENGTH, "ZeroLength: line " + std::to_string(i));
    if (lengths[i] > 0xFFFFFFFFull) return fail(B2F_ERR_LENGTH_TOO_LARGE, "LengthTooLarge");
    if (offsets[i] > (UINT64_MAX >> 4) - lengths[i])  // byte sizes must fit 64 bits
      return fail(B2F_ERR_INVALID_ARGUMENT, "batch line " + std::to_string(i) + " lies beyond the addressable range");
  }
  std::sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) { return offsets[a] < offsets[b]; });
  uint64_t extent = 0;
  for (uint64_t i = 0; i < nlines; ++i) {
    const uint64_t l = order[i];
    if (i && offsets[l] < offsets[order[i - 1]] + lengths[order[i - 1]])
      return fail(B2F_ERR_INVALID_ARGUMENT, "batch lines overlap");
    extent = std::max(extent, offsets[l] + lengths[l]);
  }
  int prev = -1;
  cudaGetDevice(&prev);
  if (device < 0) device = prev < 0 ? 0 : prev;
  if (cudaSetDevice(device) != cudaSuccess) return fail(B2F_ERR_DEVICE, "cudaSetDevice failed");
  std::unique_ptr<BatchPlan> bp(new BatchPlan());
  bp->device = device;
  bp->direction = direction;
  bp->normalization = normalization;
  bp->nlines = nlines;
  bp->extent = extent;
  int smem_optin = 0;
  cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  const size_t static_smem = sizeof(BatchLen) + 2 * kBatchMaxG * 8 + 64;
  const size_t cta_cap = 44 * 1024;  // line buffers of four CTAs per SM
  const size_t cl_cap = (size_t)smem_optin - static_smem - 1024;
  // distinct lengths
  std::map<uint64_t, std::vector<uint64_t>> by_len;
  for (uint64_t i = 0; i < nlines; ++i) by_len[lengths[i]].push_back(i);
  std::vector<uint64_t> lens_list;
  for (auto& kv : by_len) lens_list.push_back(kv.first);
  std::vector<LenInfo> infos(lens_list.size());
  std::vector<int> ok(lens_list.size(), 0);
  {
    const unsigned nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (unsigned w = 0; w < nth; ++w)
      th.emplace_back([&, w] {
        for (size_t i = w; i < lens_list.size(); i += nth)
          ok[i] = classify(lens_list[i], direction, normalization, cta_cap, cl_cap,
                           (flags & 1u) != 0, infos[i]);
      });
    for (auto& t : th) t.join();
  }
  for (size_t i = 0; i < lens_list.size(); ++i)
    if (!ok[i]) {
      if (prev >= 0) cudaSetDevice(prev);
      return fail(B2F_ERR_UNSUPPORTED_LENGTH,
                  "UnsupportedLength { len: " + std::to_string(lens_list[i]) + " } in a batch");
    }
  bp->distinct = lens_list.size();
  // twiddle tables shared by every length of the batch
  {
    std::vector<cd> tw;
    std::map<uint32_t, uint32_t> cache;
    for (auto& li : infos) {
      BatchLen& d = li.d;
      if (d.kind == BK_LONG || d.kind == BK_LONG_BLUE) {
        // stage tables of both passes and W_M^{a N2} / W_M^b
        LongLenDesc& g = li.lng;
        attach_stage_table(li.s1, tw, cache);
        attach_stage_table(li.s2, tw, cache);
        for (int w = 0; w < 2; ++w) {
          const Schedule& sc = w ? li.s2 : li.s1;
          LongSched& ls = w ? g.s2 : g.s1;
          ls.nst = sc.nst;
          for (uint32_t k = 0; k < sc.nst; ++k) ls.st[k] = sc.st[k];
        }
        long_split_tables(g, tw, 0);
        continue;
      }
      attach_stage_table(d.sch, tw, cache);
      if (d.kind == BK_CL_MIXED || d.kind == BK_CL_BLUE) {
        d.ta = (uint32_t)tw.size();
        for (uint32_t a = 0; a < d.P; ++a) tw.push_back(root_fwd((uint64_t)a * d.L, d.M));
        d.tb = (uint32_t)tw.size();
        for (uint32_t c = 0; c < d.L; ++c) tw.push_back(root_fwd(c, d.M));
        d.dB = make_fastdiv(d.L);
      }
    }
    std::vector<float> f(std::max<size_t>(2, tw.size() * 2));
    for (size_t i = 0; i < tw.size(); ++i) {
      f[2 * i] = (float)tw[i].real();
      f[2 * i + 1] = (float)tw[i].imag();
    }
    if (cudaMalloc(&bp->d_tw, f.size() * 4) != cudaSuccess ||
        cudaMemcpy(bp->d_tw, f.data(), f.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
      if (prev >= 0) cudaSetDevice(prev);
      return fail(B2F_ERR_RESOURCE_ALLOCATION, "batch twiddle table allocation failed");
    }
    bp->tw_bytes = f.size() * 4;
  }
  // tables
  auto upload = [&](const void* src, size_t bytes, void** dst) -> bool {
    if (bytes == 0) {
      *dst = nullptr;
      return true;
    }
    if (cudaMalloc(dst, bytes) != cudaSuccess) return false;
    bp->tables.push_back(*dst);
    bp->table_bytes += bytes;
    return cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
  };
  for (auto& li : infos) {
    if (!li.bhat.empty()) {
      std::vector<float> f(li.bhat.size() * 2);
      for (size_t i = 0; i < li.bhat.size(); ++i) {
        f[2 * i] = (float)li.bhat[i].real();
        f[2 * i + 1] = (float)li.bhat[i].imag();
      }
      void* p;
      if (!upload(f.data(), f.size() * 4, &p)) return fail(B2F_ERR_RESOURCE_ALLOCATION, "batch table allocation failed");
      li.d.bhat = (const c32*)p;
      li.lng.bhat = (const c32*)p;
    }
    if (!li.pin.empty()) {
      void *a, *b;
      if (!upload(li.pin.data(), li.pin.size() * 4, &a) || !upload(li.pout.data(), li.pout.size() * 4, &b))
        return fail(B2F_ERR_RESOURCE_ALLOCATION, "batch table allocation failed");
      li.d.perm_in = (const uint32_t*)a;
      li.d.perm_out = (const uint32_t*)b;
    }
  }
  // chunks of host execution: lines in offset order, cut into runs of about
  // equal bytes, except that with 8 chunks or more the first three and the
  // last three hold 1/8, 1/4 and 1/2 of the others' share, so that the
  // pipeline's fill (the first copy in) and drain (the last transform and
  // copy out) are short
  std::vector<uint32_t> chunk_of(nlines, 0);
  {
    uint64_t total = 0, acc = 0;
    for (uint64_t i = 0; i < nlines; ++i) total += lengths[i];
    for (uint32_t c = 0; c < kHostChunks; ++c) bp->chunk_lo[c] = bp->chunk_hi[c] = 0;
    bp->n_chunks = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>(kHostChunks, (total * 8 + kHostChunkBytes - 1) / kHostChunkBytes));
    const uint32_t K = bp->n_chunks;
    bool seen[kHostChunks] = {};
    uint64_t cum[kHostChunks + 1] = {};  // chunk c: acc / total in [cum[c], cum[c + 1]) / cum[K]
    for (uint32_t c = 0; c < K; ++c) {
      const uint32_t e = std::min(c, K - 1 - c);
      cum[c + 1] = cum[c] + (K >= 8 && e < 3 ? 1u << e : 8u);
    }
    uint32_t cc = 0;
    for (uint64_t i = 0; i < nlines; ++i) {
      const uint64_t l = order[i];
      while (cc + 1 < K && acc * cum[K] >= total * cum[cc + 1]) ++cc;
      chunk_of[l] = cc;
      if (!seen[cc]) bp->chunk_lo[cc] = offsets[l];
      seen[cc] = true;
      bp->chunk_hi[cc] = offsets[l] + lengths[l];
      acc += lengths[l];
    }
    // copy pieces: piece c starts at chunk c's first byte rounded down (not
    // before the previous piece's end; the first piece at its first byte)
    // and ends where the next non-empty chunk's piece starts, or at chunk
    // c's last byte when unused bytes follow; an empty chunk has an empty piece
    uint64_t end_all = 0, pos = 0;
    for (uint32_t c = 0; c < K; ++c)
      if (seen[c]) end_all = std::max(end_all, bp->chunk_hi[c] * 8);
    bool first = true;
    for (uint32_t c = 0; c < K; ++c) {
      if (!seen[c]) {
        bp->piece_lo[c] = bp->piece_hi[c] = pos;
        continue;
      }
      const uint64_t lo = bp->chunk_lo[c] * 8, hi = bp->chunk_hi[c] * 8;
      const uint64_t start = first ? lo : std::max(pos, lo / kHostCopyAlign * kHostCopyAlign);
      uint32_t c2 = c + 1;
      while (c2 < K && !seen[c2]) ++c2;
      uint64_t end = end_all;
      if (c2 < K) {
        const uint64_t nb = bp->chunk_lo[c2] * 8 / kHostCopyAlign * kHostCopyAlign;
        end = nb <= hi ? std::max(start, nb) : hi;
      }
      bp->piece_lo[c] = start;
      bp->piece_hi[c] = end;
      pos = end;
      first = false;
    }
    // chunk c's lines end in the first piece whose end reaches chunk_hi[c];
    // piece j holds outputs of the chunks that start before its end
    for (uint32_t c = 0; c < K; ++c) {
      uint32_t j = 0;
      while (j + 1 < K && bp->piece_hi[j] < bp->chunk_hi[c] * 8) ++j;
      bp->in_wait[c] = j;
    }
    for (uint32_t j = 0; j < K; ++j) {
      uint32_t w = kNoWait;
      for (uint32_t c = 0; c < K; ++c)
        if (seen[c] && bp->chunk_lo[c] * 8 < bp->piece_hi[j] && bp->chunk_hi[c] * 8 > bp->piece_lo[j])
          w = c;
      bp->out_wait[j] = w;
    }
  }
  // tasks: CTA tasks (groups of G lines of one length and one chunk),
  // cluster tasks (one line each)
  std::vector<uint64_t> sorted_off;
  std::vector<BatchTask> cta_tasks, cl_tasks, big_tasks, cta_ch_tasks;
  std::vector<double> cta_cost, cl_cost, big_cost, cta_ch_cost;
  // lines sorted by length index; CTA tasks reference contiguous runs.
  // Long lines get one task per column or row group in each of their
  // phases (1: columns, 2: rows, 3: Bluestein inverse columns).
  uint64_t n_long_lines = 0;
  std::vector<LongTask> long_tasks[3];
  std::vector<uint32_t> long_task_chunk[3];
  uint64_t scratch_total = 0;
  for (size_t li = 0; li < lens_list.size(); ++li) {
    const auto& lines = by_len[lens_list[li]];
    const BatchLen& d = infos[li].d;
    bp->kind_lines[d.kind] += lines.size();
    const bool cl = d.kind == BK_CL_MIXED || d.kind == BK_CL_BLUE;
    if (d.kind == BK_LONG || d.kind == BK_LONG_BLUE) {
      const LongLenDesc& g = infos[li].lng;
      const uint32_t Gc = 1u << g.lgc, Gr = 1u << g.lgr;
      for (uint64_t line : lines) {
        const uint64_t lbase = offsets[line], lscr = scratch_total;
        ++n_long_lines;
        scratch_total += g.M;
        bp->elems_long += lens_list[li];
        bp->lines_long += 1;
        const uint32_t ch = chunk_of[line];
        for (uint32_t g0 = 0; g0 < g.N2; g0 += Gc) {
          long_tasks[0].push_back(LongTask{lbase, lscr, (uint32_t)li, g0, lbase});
          long_task_chunk[0].push_back(ch);
        }
        for (uint32_t g0 = 0; g0 < g.N1; g0 += Gr) {
          long_tasks[1].push_back(LongTask{lbase, lscr, (uint32_t)li, g0, lbase});
          long_task_chunk[1].push_back(ch);
        }
        if (g.blue)
          for (uint32_t g0 = 0; g0 < g.N2; g0 += Gc) {
            long_tasks[2].push_back(LongTask{lbase, lscr, (uint32_t)li, g0, lbase});
            long_task_chunk[2].push_back(ch);
          }
      }
      continue;
    }
    // the length's lines in chunk order, their offsets stored once; the
    // whole-batch tasks take runs of up to G of them, the host-execution
    // tasks runs of up to G within one chunk
    std::vector<uint64_t> ls = lines;
    std::stable_sort(ls.begin(), ls.end(),
                     [&](uint64_t a, uint64_t b) { return chunk_of[a] < chunk_of[b]; });
    const uint32_t first = (uint32_t)sorted_off.size();
    for (uint64_t l : ls) sorted_off.push_back(offsets[l]);
    auto make = [&](size_t s, size_t e, uint32_t ch) {
      BatchTask t;
      t.len = (uint32_t)li;
      t.first = first + (uint32_t)s;
      t.count = (uint32_t)(e - s);
      t.pad = ch;  // chunk (not read by the kernels)
      return t;
    };
    if (cl) {
      for (size_t s = 0; s < ls.size(); ++s) {
        const BatchTask t = make(s, s + 1, chunk_of[ls[s]]);
        if (d.P == kClusterBig) {
          big_tasks.push_back(t);
          big_cost.push_back(infos[li].cost);
        } else {
          cl_tasks.push_back(t);
          cl_cost.push_back(infos[li].cost);
        }
        bp->lines_cl += 1;
        bp->elems_cl += lens_list[li];
      }
      continue;
    }
    for (size_t s = 0; s < ls.size(); s += d.G) {
      const BatchTask t = make(s, std::min<size_t>(ls.size(), s + d.G), 0);
      cta_tasks.push_back(t);
      cta_cost.push_back(infos[li].cost * t.count);
      bp->lines_cta += t.count;
      bp->elems_cta += lens_list[li] * t.count;
    }
    for (size_t s = 0; s < ls.size();) {
      const uint32_t ch = chunk_of[ls[s]];
      size_t e = s;
      while (e < ls.size() && chunk_of[ls[e]] == ch && e - s < d.G) ++e;
      cta_ch_tasks.push_back(make(s, e, ch));
      cta_ch_cost.push_back(infos[li].cost * (double)(e - s));
      s = e;
    }
  }
  // longest first (the queue hands them out in order)
  auto sort_by_cost = [](std::vector<BatchTask>& t, std::vector<double>& c) {
    std::vector<size_t> idx(t.size());
    for (size_t i = 0; i < idx.size(); ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return c[a] > c[b]; });
    std::vector<BatchTask> out(t.size());
    for (size_t i = 0; i < idx.size(); ++i) out[i] = t[idx[i]];
    t.swap(out);
  };
  sort_by_cost(cta_tasks, cta_cost);
  // the host-execution tasks chunk by chunk (longest first within each)
  sort_by_cost(cta_ch_tasks, cta_ch_cost);
  std::vector<BatchTask> cta_chunked = cta_ch_tasks;
  std::stable_sort(cta_chunked.begin(), cta_chunked.end(),
                   [](const BatchTask& a, const BatchTask& b) { return a.pad < b.pad; });
  for (size_t i = 0; i < cta_chunked.size(); ++i) {
    const uint32_t c = cta_chunked[i].pad;
    if (bp->cta_ccount[c] == 0) bp->cta_cfirst[c] = (uint32_t)i;
    ++bp->cta_ccount[c];
  }
  // within each phase, the smooth lines' tasks before the Bluestein lines',
  // and within each kind by the length of the pass (N1 for the column
  // phases, N2 for the rows): consecutive tasks run the same code, which
  // keeps the instruction cache warm
  for (int ph = 0; ph < 3; ++ph) {
    std::vector<size_t> idx(long_tasks[ph].size());
    for (size_t i = 0; i < idx.size(); ++i) idx[i] = i;
    auto key = [&](size_t i) {
      const LongLenDesc& g = infos[long_tasks[ph][i].len].lng;
      return std::make_pair(g.blue, ph == 1 ? g.N2 : g.N1);
    };
    std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return key(a) < key(b); });
    std::vector<LongTask> t(idx.size());
    std::vector<uint32_t> c(idx.size());
    for (size_t i = 0; i < idx.size(); ++i) {
      t[i] = long_tasks[ph][idx[i]];
      c[i] = long_task_chunk[ph][idx[i]];
    }
    long_tasks[ph].swap(t);
    long_task_chunk[ph].swap(c);
  }
  // long tasks of each phase chunk by chunk, likewise
  std::vector<LongTask> long_chunked[3];
  for (int ph = 0; ph < 3; ++ph) {
    std::vector<size_t> idx(long_tasks[ph].size());
    for (size_t i = 0; i < idx.size(); ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
      return long_task_chunk[ph][a] < long_task_chunk[ph][b];
    });
    long_chunked[ph].resize(idx.size());
    for (size_t i = 0; i < idx.size(); ++i) {
      long_chunked[ph][i] = long_tasks[ph][idx[i]];
      const uint32_t c = long_task_chunk[ph][idx[i]];
      if (bp->long_ccount[ph][c] == 0) bp->long_cfirst[ph][c] = (uint32_t)i;
      ++bp->long_ccount[ph][c];
    }
  }
  sort_by_cost(cl_tasks, cl_cost);
  sort_by_cost(big_tasks, big_cost);
  bp->n_cta = (uint32_t)cta_tasks.size();
  bp->n_cl = (uint32_t)cl_tasks.size();
  bp->n_big = (uint32_t)big_tasks.size();
  // shared memory of each kernel: the largest task it runs
  uint32_t buf_cta = 1, buf_cl = 1;
  for (auto& li : infos) {
    const BatchLen& d = li.d;
    if (d.kind == BK_CL_MIXED || d.kind == BK_CL_BLUE) buf_cl = std::max(buf_cl, d.LD);
    else if (d.kind == BK_LONG || d.kind == BK_LONG_BLUE) {
      const LongLenDesc& g = li.lng;
      bp->long_cap = std::max(bp->long_cap, g.N1 * ((1u << g.lgc) + 1));
      bp->long_cap = std::max(bp->long_cap, g.N2 * ((1u << g.lgr) + 1));
    } else {
      buf_cta = std::max<uint32_t>(buf_cta, d.G * d.LD);
    }
  }
  bp->buf_cta = buf_cta;
  bp->buf_cl = buf_cl;
  bp->smem_cta = 2 * (size_t)buf_cta * 8 + 2 * kBatchMaxG * 8;
  bp->smem_cl = 2 * (size_t)buf_cl * 8;
  // device arrays
  std::vector<BatchLen> dl(infos.size());
  for (size_t i = 0; i < infos.size(); ++i) dl[i] = infos[i].d;
  std::vector<BatchTask> all = cta_tasks;
  all.insert(all.end(), cl_tasks.begin(), cl_tasks.end());
  all.insert(all.end(), big_tasks.begin(), big_tasks.end());
  bool okc = cudaMalloc(&bp->d_lens, dl.size() * sizeof(BatchLen)) == cudaSuccess &&
             cudaMalloc(&bp->d_tasks, std::max<size_t>(1, all.size()) * sizeof(BatchTask)) == cudaSuccess &&
             cudaMalloc(&bp->d_off, sorted_off.size() * 8) == cudaSuccess &&
             cudaMalloc(&bp->d_counters, kBatchCounters * sizeof(unsigned int)) == cudaSuccess &&
             cudaMalloc(&bp->d_tasks_chunked, std::max<size_t>(1, cta_chunked.size()) * sizeof(BatchTask)) ==
                 cudaSuccess;
  if (!okc) return fail(B2F_ERR_RESOURCE_ALLOCATION, "batch allocation failed");
  if (!cta_chunked.empty())
    cudaMemcpy(bp->d_tasks_chunked, cta_chunked.data(), cta_chunked.size() * sizeof(BatchTask),
               cudaMemcpyHostToDevice);
  cudaMemcpy(bp->d_lens, dl.data(), dl.size() * sizeof(BatchLen), cudaMemcpyHostToDevice);
  if (!all.empty()) cudaMemcpy(bp->d_tasks, all.data(), all.size() * sizeof(BatchTask), cudaMemcpyHostToDevice);
  cudaMemcpy(bp->d_off, sorted_off.data(), sorted_off.size() * 8, cudaMemcpyHostToDevice);
  // long lines: descriptors (indexed like the length table), lines, tasks
  if (n_long_lines) {
    std::vector<LongLenDesc> gl(infos.size());
    std::memset(gl.data(), 0, gl.size() * sizeof(LongLenDesc));
    for (size_t i = 0; i < infos.size(); ++i)
      if (infos[i].d.kind == BK_LONG || infos[i].d.kind == BK_LONG_BLUE) gl[i] = infos[i].lng;
    std::vector<LongTask> lt, ltc;
    for (int ph = 0; ph < 3; ++ph) {
      bp->long_first[ph] = (uint32_t)lt.size();
      bp->long_count[ph] = (uint32_t)long_tasks[ph].size();
      lt.insert(lt.end(), long_tasks[ph].begin(), long_tasks[ph].end());
      ltc.insert(ltc.end(), long_chunked[ph].begin(), long_chunked[ph].end());
    }
    const bool okl =
        cudaMalloc(&bp->d_long_lens, gl.size() * sizeof(LongLenDesc)) == cudaSuccess &&
        cudaMalloc(&bp->d_long_tasks, lt.size() * sizeof(LongTask)) == cudaSuccess &&
        cudaMalloc(&bp->d_long_tasks_chunked, ltc.size() * sizeof(LongTask)) == cudaSuccess &&
        cudaMalloc(&bp->d_scratch, scratch_total * 8) == cudaSuccess;
    if (!okl) return fail(B2F_ERR_RESOURCE_ALLOCATION, "batch long-line allocation failed");
    bp->scratch_bytes = scratch_total * 8;
    cudaMemcpy(bp->d_long_lens, gl.data(), gl.size() * sizeof(LongLenDesc), cudaMemcpyHostToDevice);
    cudaMemcpy(bp->d_long_tasks, lt.data(), lt.size() * sizeof(LongTask), cudaMemcpyHostToDevice);
    cudaMemcpy(bp->d_long_tasks_chunked, ltc.data(), ltc.size() * sizeof(LongTask), cudaMemcpyHostToDevice);
  }
  // launch shapes
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  if (bp->n_cta) {
    if (set_smem(k_batch_cta, bp->smem_cta) != cudaSuccess)
      return fail(B2F_ERR_DEVICE, "batch CTA kernel shared memory");
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_cta, kCtaThreads, bp->smem_cta);
    per_sm = std::max(per_sm, 1);
    bp->grid_cta = (unsigned)std::min<uint64_t>((uint64_t)nsm * per_sm, bp->n_cta);
  }
  if (n_long_lines) {
    bp->smem_long = (3 * (size_t)bp->long_cap + 2 * kLongTab) * 8;
    if (set_smem(k_long_pass<1>, bp->smem_long) != cudaSuccess ||
        set_smem(k_long_pass<2>, bp->smem_long) != cudaSuccess ||
        set_smem(k_long_pass<3>, bp->smem_long) != cudaSuccess)
      return fail(B2F_ERR_DEVICE, "long-line kernel shared memory");
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_long_pass<2>, kLongThreads, bp->smem_long);
    per_sm = std::max(per_sm, 1);
    uint32_t most = std::max(bp->long_count[0], std::max(bp->long_count[1], bp->long_count[2]));
    bp->grid_long = (unsigned)std::min<uint64_t>((uint64_t)nsm * per_sm,
                                                 (most + kLongChunk - 1) / kLongChunk);
  }
  if (bp->n_cl) {
    if (set_smem(k_batch_cluster<kClusterP>, bp->smem_cl) != cudaSuccess)
      return fail(B2F_ERR_DEVICE, "batch cluster kernel shared memory");
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClusterP;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(kClusterP * 64, 1, 1);
    cfg.blockDim = dim3(kClusterThreads, 1, 1);
    cfg.dynamicSmemBytes = bp->smem_cl;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, k_batch_cluster<kClusterP>, &cfg) != cudaSuccess ||
        nclusters <= 0) {
      cudaGetLastError();
      return fail(B2F_ERR_DEVICE, "no thread-block cluster of 8 CTAs fits this device");
    }
    bp->grid_cl = (unsigned)(kClusterP * std::min<uint64_t>((uint64_t)nclusters, bp->n_cl));
  }
  if (bp->n_big) {
    if (set_smem(k_batch_cluster<kClusterBig>, bp->smem_cl) != cudaSuccess ||
        cudaFuncSetAttribute(k_batch_cluster<kClusterBig>,
                             cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
      return fail(B2F_ERR_DEVICE, "batch 16-CTA cluster kernel attributes");
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClusterBig;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(kClusterBig * 16, 1, 1);
    cfg.blockDim = dim3(kClusterThreads, 1, 1);
    cfg.dynamicSmemBytes = bp->smem_cl;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, k_batch_cluster<kClusterBig>, &cfg) != cudaSuccess ||
        nclusters <= 0) {
      cudaGetLastError();
      return fail(B2F_ERR_UNSUPPORTED_LENGTH,
                  "UnsupportedLength: a Bluestein line needs a 16-CTA cluster, which this device cannot schedule");
    }
    bp->grid_big = (unsigned)(kClusterBig * std::min<uint64_t>((uint64_t)nclusters, bp->n_big));
  }
  if (cudaStreamCreateWithFlags(&bp->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&bp->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&bp->join, cudaEventDisableTiming) != cudaSuccess)
    return fail(B2F_ERR_DEVICE, "batch stream creation failed");
  {
    bool okh = cudaEventCreateWithFlags(&bp->hev_start, cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&bp->hev_done, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; i < 3 && okh; ++i)
      okh = cudaStreamCreateWithFlags(&bp->hs[i], cudaStreamNonBlocking) == cudaSuccess;
    for (uint32_t c = 0; c < kHostChunks && okh; ++c)
      okh = cudaEventCreateWithFlags(&bp->hev_in[c], cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&bp->hev_c[c], cudaEventDisableTiming) == cudaSuccess;
    if (!okh) return fail(B2F_ERR_DEVICE, "batch host-pipeline stream creation failed");
  }
  std::ostringstream os;
  os << "{\"lines\":" << nlines << ",\"distinct_lengths\":" << bp->distinct
     << ",\"cta_lines\":" << bp->lines_cta << ",\"cluster_lines\":" << bp->lines_cl
     << ",\"cta_elements\":" << bp->elems_cta << ",\"cluster_elements\":" << bp->elems_cl
     << ",\"long_lines\":" << bp->lines_long << ",\"long_elements\":" << bp->elems_long
     << ",\"cta_tasks\":" << bp->n_cta << ",\"cta_launches\":" << (bp->n_cta > 0)
     << ",\"long_tasks\":[" << bp->long_count[0] << "," << bp->long_count[1] << ","
     << bp->long_count[2] << "],\"long_launches\":"
     << ((bp->long_count[0] > 0) + (bp->long_count[1] > 0) + (bp->long_count[2] > 0))
     << ",\"long_grid\":" << bp->grid_long << ",\"long_threads\":" << kLongThreads
     << ",\"long_smem\":" << bp->smem_long << ",\"host_chunks\":" << bp->n_chunks
     << ",\"cluster_tasks\":" << bp->n_cl
     << ",\"kind_lines\":{\"mixed\":" << bp->kind_lines[0] << ",\"rader\":" << bp->kind_lines[1]
     << ",\"bluestein\":" << bp->kind_lines[2] << ",\"cluster_mixed\":" << bp->kind_lines[3]
     << ",\"cluster_bluestein\":" << bp->kind_lines[4] << ",\"two_pass\":" << bp->kind_lines[5]
     << ",\"two_pass_bluestein\":" << bp->kind_lines[6] << "}"
     << ",\"scratch_bytes\":" << bp->scratch_bytes << ",\"twiddle_table_bytes\":" << bp->tw_bytes
     << ",\"cta_grid\":" << bp->grid_cta << ",\"cta_threads\":" << kCtaThreads
     << ",\"cta_smem\":" << bp->smem_cta << ",\"cluster_grid\":" << bp->grid_cl
     << ",\"cluster_size\":" << kClusterP << ",\"cluster16_tasks\":" << bp->n_big
     << ",\"cluster16_grid\":" << bp->grid_big << ",\"cluster_threads\":" << kClusterThreads
     << ",\"cluster_smem\":" << bp->smem_cl << ",\"table_bytes\":" << bp->table_bytes
     << ",\"required_buffer_size_bytes\":" << extent * 8 << "}";
  bp->diag = os.str();
  if (prev >= 0) cudaSetDevice(prev);
  *out = bp.release();
  return B2F_OK;
}

static void launch_long(const BatchPlan& bp, cudaStream_t st, const void* in, void* out, int chunk,
                        cudaError_t* err);

static b2f_status run_batch(const BatchPlan& bp, cudaStream_t st, const void* in, void* out,
                            uint32_t parts = 7, bool sequential = false) {
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != bp.device) cudaSetDevice(bp.device);
  cudaError_t e = cudaMemsetAsync(bp.d_counters, 0, kBatchCounters * sizeof(unsigned int), st);
  BatchParams p{};
  p.in = (const c32*)in;
  p.out = (c32*)out;
  p.lens = bp.d_lens;
  p.line_off = bp.d_off;
  p.inverse = bp.direction == B2F_INVERSE ? 1u : 0u;
  p.tw = bp.d_tw;
  const bool run_cl = (bp.n_cl || bp.n_big) && (parts & 2);
  const bool run_cta = bp.n_cta && (parts & 1);
  cudaStream_t cl_stream = sequential ? st : bp.side;
  if (e == cudaSuccess && run_cl) {
    // long lines on a forked stream, concurrently with the CTA queue
    if (!sequential) {
      e = cudaEventRecord(bp.fork, st);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(bp.side, bp.fork, 0);
    }
    BatchParams pc = p;
    pc.tasks = bp.d_tasks + bp.n_cta;
    pc.ntasks = bp.n_cl;
    pc.counter = bp.d_counters + 1;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClusterP;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(bp.grid_cl, 1, 1);
    cfg.blockDim = dim3(kClusterThreads, 1, 1);
    cfg.dynamicSmemBytes = bp.smem_cl;
    cfg.stream = cl_stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (e == cudaSuccess && bp.n_cl) e = cudaLaunchKernelEx(&cfg, k_batch_cluster<kClusterP>, pc, bp.buf_cl);
    if (e == cudaSuccess && bp.n_big) {
      BatchParams pb = p;
      pb.tasks = bp.d_tasks + bp.n_cta + bp.n_cl;
      pb.ntasks = bp.n_big;
      pb.counter = bp.d_counters + 2;
      attr[0].val.clusterDim.x = kClusterBig;
      cfg.gridDim = dim3(bp.grid_big, 1, 1);
      e = cudaLaunchKernelEx(&cfg, k_batch_cluster<kClusterBig>, pb, bp.buf_cl);
    }
  }
  // without cluster lines, the CTA queue runs on the forked stream,
  // concurrently with the long-line phases (no line is in both)
  const bool cta_side = run_cta && !run_cl && !sequential && (parts & 4) && bp.lines_long;
  if (e == cudaSuccess && cta_side) {
    e = cudaEventRecord(bp.fork, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(bp.side, bp.fork, 0);
  }
  if (e == cudaSuccess && run_cta) {
    BatchParams pt = p;
    pt.tasks = bp.d_tasks;
    pt.ntasks = bp.n_cta;
    pt.counter = bp.d_counters;
    k_batch_cta<<<bp.grid_cta, kCtaThreads, bp.smem_cta, cta_side ? bp.side : st>>>(pt, bp.buf_cta);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && (parts & 4) && bp.lines_long) {
    launch_long(bp, st, in, out, -1, &e);
  }
  if (e == cudaSuccess && ((run_cl && !sequential) || cta_side)) {
    e = cudaEventRecord(bp.join, bp.side);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, bp.join, 0);
  }
  if (prev >= 0 && prev != bp.device) cudaSetDevice(prev);
  if (e != cudaSuccess) return fail(B2F_ERR_DEVICE, std::string("batch launch failed: ") + cudaGetErrorString(e));
  return B2F_OK;
}

// The long-line phases of every line (chunk < 0) or of one chunk.
static void launch_long(const BatchPlan& bp, cudaStream_t st, const void* in, void* out, int chunk,
                        cudaError_t* err) {
  cudaError_t e = cudaSuccess;
  {
    LongParams lp{};
    lp.in = (const c32*)in;
    lp.out = (c32*)out;
    lp.scratch = bp.d_scratch;
    lp.tw = bp.d_tw;
    lp.lens = bp.d_long_lens;
    lp.cap = bp.long_cap;
    lp.inverse = bp.direction == B2F_INVERSE ? 1u : 0u;
    for (uint32_t ph = 0; ph < 3 && e == cudaSuccess; ++ph) {
      const uint32_t first = chunk < 0 ? 0 : bp.long_cfirst[ph][chunk];
      const uint32_t count = chunk < 0 ? bp.long_count[ph] : bp.long_ccount[ph][chunk];
      if (count == 0) continue;
      lp.tasks = (chunk < 0 ? bp.d_long_tasks : bp.d_long_tasks_chunked) + bp.long_first[ph] + first;
      lp.ntasks = count;
      lp.phase = ph + 1;
      lp.counter = bp.d_counters + (chunk < 0 ? 4 + ph : 9 + 4 * chunk + ph);
      const unsigned grid = (unsigned)std::min<uint64_t>(bp.grid_long, (count + kLongChunk - 1) / kLongChunk);
      if (ph == 0) k_long_pass<1><<<grid, kLongThreads, bp.smem_long, st>>>(lp);
      else if (ph == 1) k_long_pass<2><<<grid, kLongThreads, bp.smem_long, st>>>(lp);
      else k_long_pass<3><<<grid, kLongThreads, bp.smem_long, st>>>(lp);
      e = cudaGetLastError();
    }
  }
  *err = e;
}

// One chunk of a host execution: its CTA tasks and long phases on st (the
// chunk's counters were zeroed by the caller).
static cudaError_t run_chunk(const BatchPlan& bp, cudaStream_t st, const void* in, void* out,
                             int chunk) {
  cudaError_t e = cudaSuccess;
  if (bp.cta_ccount[chunk]) {
    BatchParams pt{};
    pt.in = (const c32*)in;
    pt.out = (c32*)out;
    pt.lens = bp.d_lens;
    pt.line_off = bp.d_off;
    pt.inverse = bp.direction == B2F_INVERSE ? 1u : 0u;
    pt.tw = bp.d_tw;
    pt.tasks = bp.d_tasks_chunked + bp.cta_cfirst[chunk];
    pt.ntasks = bp.cta_ccount[chunk];
    pt.counter = bp.d_counters + 8 + 4 * chunk;
    const unsigned grid = (unsigned)std::min<uint64_t>(bp.grid_cta, bp.cta_ccount[chunk]);
    k_batch_cta<<<grid, kCtaThreads, bp.smem_cta, st>>>(pt, bp.buf_cta);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && bp.lines_long) launch_long(bp, st, in, out, chunk, &e);
  return e;
}

// Host buffers in and out: the chunks' copies in (stream hs[0]), transforms
// (hs[1]) and copies out (hs[2]) overlap, chunk c's transform waiting for
// its copy in and its copy out for its transform; `st` orders the whole
// call with the caller's other work.  Cluster routes run unchunked.
static b2f_status run_batch_host(const BatchPlan& bp, cudaStream_t st, const void* host_in,
                                 void* host_out, void* dev_in, void* dev_out) {
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != bp.device) cudaSetDevice(bp.device);
  const uint64_t bytes = bp.extent * 8;
  cudaError_t e = cudaSuccess;
  auto finish = [&]() -> b2f_status {
    if (prev >= 0 && prev != bp.device) cudaSetDevice(prev);
    if (e != cudaSuccess)
      return fail(B2F_ERR_DEVICE, std::string("batch host execution failed: ") + cudaGetErrorString(e));
    return B2F_OK;
  };
  if (bp.n_cl || bp.n_big) {
    e = cudaMemcpyAsync(dev_in, host_in, bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
      const b2f_status r = run_batch(bp, st, dev_in, dev_out);  // restores the device itself
      if (r != B2F_OK) {
        if (prev >= 0 && prev != bp.device) cudaSetDevice(prev);
        return r;  // its message stands
      }
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(host_out, dev_out, bytes, cudaMemcpyDeviceToHost, st);
    return finish();
  }
  cudaStream_t sin = bp.hs[0], sc = bp.hs[1], sout = bp.hs[2];
  e = cudaEventRecord(bp.hev_start, st);
  for (int i = 0; i < 3 && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(bp.hs[i], bp.hev_start, 0);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(bp.d_counters, 0, kBatchCounters * sizeof(unsigned int), sc);
  for (uint32_t j = 0; j < bp.n_chunks && e == cudaSuccess; ++j) {
    const uint64_t lo = bp.piece_lo[j], n = bp.piece_hi[j] - bp.piece_lo[j];
    if (n) e = cudaMemcpyAsync((char*)dev_in + lo, (const char*)host_in + lo, n, cudaMemcpyHostToDevice, sin);
    if (e == cudaSuccess) e = cudaEventRecord(bp.hev_in[j], sin);
  }
  for (uint32_t c = 0; c < bp.n_chunks && e == cudaSuccess; ++c) {
    e = cudaStreamWaitEvent(sc, bp.hev_in[bp.in_wait[c]], 0);
    if (e == cudaSuccess) e = run_chunk(bp, sc, dev_in, dev_out, (int)c);
    if (e == cudaSuccess) e = cudaEventRecord(bp.hev_c[c], sc);
  }
  for (uint32_t j = 0; j < bp.n_chunks && e == cudaSuccess; ++j) {
    const uint64_t lo = bp.piece_lo[j], n = bp.piece_hi[j] - bp.piece_lo[j];
    if (bp.out_wait[j] == kNoWait) continue;  // no line's bytes
    e = cudaStreamWaitEvent(sout, bp.hev_c[bp.out_wait[j]], 0);
    if (e == cudaSuccess && n)
      e = cudaMemcpyAsync((char*)host_out + lo, (const char*)dev_out + lo, n, cudaMemcpyDeviceToHost, sout);
  }
  if (e == cudaSuccess) e = cudaEventRecord(bp.hev_done, sout);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(st, bp.hev_done, 0);
  return finish();
}

// ------------------------------------------------------- line registry
// Lengths registered once per (device, direction, normalization): their
// descriptors at fixed indices of two device arrays, their twiddles in one
// device arena (offsets never move, so launches in flight are unaffected by
// later registrations) and their Rader/Bluestein tables in allocations of
// their own.
constexpr uint32_t kRegLengths = 8192;
constexpr uint64_t kRegTwiddles = 4ull << 20;  // complex values in the arena (32 MiB)

struct LineRegistry {
  int device = 0;
  int32_t direction = B2F_FORWARD, normalization = B2F_NORM_INVERSE;
  std::mutex mu;
  std::map<uint64_t, int64_t> index;  // length -> descriptor index, -1 = not accepted
  std::vector<std::unique_ptr<LenInfo>> infos;
  BatchLen* d_lens = nullptr;
  LongLenDesc* d_long_lens = nullptr;
  c32* d_tw = nullptr;
  uint64_t tw_used = 0;
  std::vector<void*> tables;
  uint64_t table_bytes = 0;
  size_t cl_cap = 0;
  int nsm = 148;
  int cta_per_sm = 0, long_per_sm = 0;
  size_t cta_smem_set = 0, long_smem_set = 0;
  ~LineRegistry() {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    for (void* p : tables) cudaFree(p);
    cudaFree(d_lens);
    cudaFree(d_long_lens);
    cudaFree(d_tw);
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// The twiddles one length reads (stage tables of its passes, the inter-pass
// two-level table, the chirp tables), with offsets relative to `base`.
static void length_twiddles(LenInfo& li, std::vector<cd>& tw, uint64_t base) {
  std::map<uint32_t, uint32_t> cache;
  BatchLen& d = li.d;
  if (d.kind == BK_LONG || d.kind == BK_LONG_BLUE) {
    LongLenDesc& g = li.lng;
    attach_stage_table(li.s1, tw, cache);
    attach_stage_table(li.s2, tw, cache);
    for (int w = 0; w < 2; ++w) {
      const Schedule& sc = w ? li.s2 : li.s1;
      LongSched& ls = w ? g.s2 : g.s1;
      ls.nst = sc.nst;
      for (uint32_t k = 0; k < sc.nst; ++k) {
        ls.st[k] = sc.st[k];
        ls.st[k].tw_off += (uint32_t)base;
      }
    }
    long_split_tables(g, tw, base);
    return;
  }
  attach_stage_table(d.sch, tw, cache);
  for (uint32_t k = 0; k < d.sch.nst; ++k) d.sch.st[k].tw_off += (uint32_t)base;
}

LineRegistry* line_registry_new(int device, int32_t direction, int32_t normalization) {
  std::unique_ptr<LineRegistry> r(new LineRegistry());
  r->device = device;
  r->direction = direction;
  r->normalization = normalization;
  int prev = -1;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return nullptr;
  int smem_optin = 0;
  cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  cudaDeviceGetAttribute(&r->nsm, cudaDevAttrMultiProcessorCount, device);
  r->cl_cap = (size_t)smem_optin;
  const bool ok = cudaMalloc(&r->d_lens, kRegLengths * sizeof(BatchLen)) == cudaSuccess &&
                  cudaMalloc(&r->d_long_lens, kRegLengths * sizeof(LongLenDesc)) == cudaSuccess &&
                  cudaMalloc(&r->d_tw, kRegTwiddles * sizeof(c32)) == cudaSuccess;
  if (prev >= 0) cudaSetDevice(prev);
  if (!ok) {
    cudaGetLastError();
    return nullptr;
  }
  return r.release();
}

void line_registry_free(LineRegistry* reg) { delete reg; }

uint64_t line_registry_bytes(const LineRegistry* reg) {
  if (!reg) return 0;
  return kRegLengths * (sizeof(BatchLen) + sizeof(LongLenDesc)) + kRegTwiddles * sizeof(c32) +
         reg->table_bytes;
}

// Registers length n (lock held, device current); returns its index or -1.
static int64_t registry_add(LineRegistry& r, uint64_t n) {
  auto it = r.index.find(n);
  if (it != r.index.end()) return it->second;
  int64_t idx = -1;
  std::unique_ptr<LenInfo> li(new LenInfo());
  const size_t cta_cap = 44 * 1024;  // the batch kernels' four-CTA share of an SM
  if (n >= 2 && n <= 0xFFFFFFFFull && r.infos.size() < kRegLengths &&
      classify(n, r.direction, r.normalization, cta_cap, r.cl_cap, false, *li) &&
      li->d.kind != BK_CL_MIXED && li->d.kind != BK_CL_BLUE) {
    std::vector<cd> tw;
    length_twiddles(*li, tw, r.tw_used);
    bool ok = r.tw_used + tw.size() <= kRegTwiddles;
    if (ok && !tw.empty()) {
      std::vector<float> f(tw.size() * 2);
      for (size_t i = 0; i < tw.size(); ++i) {
        f[2 * i] = (float)tw[i].real();
        f[2 * i + 1] = (float)tw[i].imag();
      }
      ok = cudaMemcpy(r.d_tw + r.tw_used, f.data(), f.size() * 4, cudaMemcpyHostToDevice) ==
           cudaSuccess;
    }
    auto upload = [&](const void* src, size_t bytes, void** dst) -> bool {
      if (cudaMalloc(dst, bytes) != cudaSuccess) return false;
      r.tables.push_back(*dst);
      r.table_bytes += bytes;
      return cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
    };
    if (ok && !li->bhat.empty()) {
      std::vector<float> f(li->bhat.size() * 2);
      for (size_t i = 0; i < li->bhat.size(); ++i) {
        f[2 * i] = (float)li->bhat[i].real();
        f[2 * i + 1] = (float)li->bhat[i].imag();
      }
      void* p = nullptr;
      ok = upload(f.data(), f.size() * 4, &p);
      li->d.bhat = (const c32*)p;
      li->lng.bhat = (const c32*)p;
    }
    if (ok && !li->pin.empty()) {
      void *a = nullptr, *b = nullptr;
      ok = upload(li->pin.data(), li->pin.size() * 4, &a) &&
           upload(li->pout.data(), li->pout.size() * 4, &b);
      li->d.perm_in = (const uint32_t*)a;
      li->d.perm_out = (const uint32_t*)b;
    }
    if (ok) {
      idx = (int64_t)r.infos.size();
      LongLenDesc g = li->lng;
      if (li->d.kind != BK_LONG && li->d.kind != BK_LONG_BLUE) std::memset(&g, 0, sizeof(g));
      ok = cudaMemcpy(r.d_lens + idx, &li->d, sizeof(BatchLen), cudaMemcpyHostToDevice) ==
               cudaSuccess &&
           cudaMemcpy(r.d_long_lens + idx, &g, sizeof(LongLenDesc), cudaMemcpyHostToDevice) ==
               cudaSuccess;
      if (ok) {
        r.tw_used += tw.size();
        r.infos.push_back(std::move(li));
      } else {
        idx = -1;
      }
    }
    if (!ok) cudaGetLastError();
  }
  r.index[n] = idx;
  return idx;
}

bool line_registry_accepts(LineRegistry* reg, uint64_t n) {
  if (!reg) return false;
  std::lock_guard<std::mutex> lk(reg->mu);
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != reg->device) cudaSetDevice(reg->device);
  const bool ok = registry_add(*reg, n) >= 0;
  if (prev >= 0 && prev != reg->device) cudaSetDevice(prev);
  return ok;
}

b2f_status line_batch_run(LineRegistry* reg, cudaStream_t st, const uint64_t* lengths,
                          const uint64_t* in_off, const uint64_t* out_off, uint64_t n,
                          const void* in, void* out, uint64_t* device_bytes) {
  if (device_bytes) *device_bytes = 0;
  if (!reg || !lengths || !in_off || !out_off || !in || !out || n == 0)
    return fail(B2F_ERR_INVALID_ARGUMENT, "empty or null line batch");
  std::lock_guard<std::mutex> lk(reg->mu);
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != reg->device) cudaSetDevice(reg->device);
  auto done = [&](b2f_status s) {
    if (prev >= 0 && prev != reg->device) cudaSetDevice(prev);
    return s;
  };
  // an error left by an unrelated earlier call of this thread must not be
  // read back as this launch's (launch errors are read with cudaGetLastError)
  cudaGetLastError();
  // lines by descriptor index
  std::map<int64_t, std::vector<uint64_t>> by_idx;
  for (uint64_t i = 0; i < n; ++i) {
    const int64_t idx = registry_add(*reg, lengths[i]);
    if (idx < 0)
      return done(fail(B2F_ERR_UNSUPPORTED_LENGTH,
                       "UnsupportedLength { len: " + std::to_string(lengths[i]) +
                           " } (not a batched-launch length)"));
    by_idx[idx].push_back(i);
  }
  std::vector<BatchTask> cta;
  std::vector<double> cta_cost;
  std::vector<uint64_t> off_in, off_out;
  std::vector<LongTask> lt[3];
  uint64_t scratch = 0;
  uint32_t buf_cta = 1, long_cap = 0;
  for (auto& kv : by_idx) {
    const LenInfo& li = *reg->infos[kv.first];
    const BatchLen& d = li.d;
    if (d.kind == BK_LONG || d.kind == BK_LONG_BLUE) {
      const LongLenDesc& g = li.lng;
      const uint32_t Gc = 1u << g.lgc, Gr = 1u << g.lgr;
      long_cap = std::max(long_cap, std::max(g.N1 * (Gc + 1), g.N2 * (Gr + 1)));
      for (uint64_t line : kv.second) {
        const uint64_t sc = scratch;
        scratch += g.M;
        for (uint32_t g0 = 0; g0 < g.N2; g0 += Gc)
          lt[0].push_back(LongTask{in_off[line], sc, (uint32_t)kv.first, g0, out_off[line]});
        for (uint32_t g0 = 0; g0 < g.N1; g0 += Gr)
          lt[1].push_back(LongTask{in_off[line], sc, (uint32_t)kv.first, g0, out_off[line]});
        if (g.blue)
          for (uint32_t g0 = 0; g0 < g.N2; g0 += Gc)
            lt[2].push_back(LongTask{in_off[line], sc, (uint32_t)kv.first, g0, out_off[line]});
      }
      continue;
    }
    buf_cta = std::max<uint32_t>(buf_cta, d.G * d.LD);
    const uint32_t first = (uint32_t)off_in.size();
    for (uint64_t line : kv.second) {
      off_in.push_back(in_off[line]);
      off_out.push_back(out_off[line]);
    }
    for (size_t s = 0; s < kv.second.size(); s += d.G) {
      BatchTask t;
      t.len = (uint32_t)kv.first;
      t.first = first + (uint32_t)s;
      t.count = (uint32_t)std::min<size_t>(d.G, kv.second.size() - s);
      t.pad = 0;
      cta.push_back(t);
      cta_cost.push_back(li.cost * t.count);
    }
  }
  // longest CTA tasks first; long tasks by kind and pass length
  {
    std::vector<size_t> idx(cta.size());
    for (size_t i = 0; i < idx.size(); ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return cta_cost[a] > cta_cost[b]; });
    std::vector<BatchTask> o(cta.size());
    for (size_t i = 0; i < idx.size(); ++i) o[i] = cta[idx[i]];
    cta.swap(o);
  }
  for (int ph = 0; ph < 3; ++ph)
    std::stable_sort(lt[ph].begin(), lt[ph].end(), [&](const LongTask& a, const LongTask& b) {
      const LongLenDesc& ga = reg->infos[a.len]->lng;
      const LongLenDesc& gb = reg->infos[b.len]->lng;
      return std::make_pair(ga.blue, ph == 1 ? ga.N2 : ga.N1) <
             std::make_pair(gb.blue, ph == 1 ? gb.N2 : gb.N1);
    });
  // one stream-ordered block: counters, CTA tasks, offsets, long tasks, scratch
  auto align = [](uint64_t b) { return (b + 255) / 256 * 256; };
  const uint64_t nlt = lt[0].size() + lt[1].size() + lt[2].size();
  const uint64_t b_cnt = align(kBatchCounters * 4), b_cta = align(cta.size() * sizeof(BatchTask));
  const uint64_t b_off = align(off_in.size() * 8), b_lt = align(nlt * sizeof(LongTask));
  const uint64_t b_scr = align(scratch * 8);
  const uint64_t total = b_cnt + b_cta + 2 * b_off + b_lt + b_scr;
  char* blk = nullptr;
  if (cudaMallocAsync((void**)&blk, total, st) != cudaSuccess) {
    cudaGetLastError();
    return done(fail(B2F_ERR_RESOURCE_ALLOCATION, "line batch allocation failed"));
  }
  if (device_bytes) *device_bytes = total;
  unsigned int* counters = (unsigned int*)blk;
  BatchTask* d_cta = (BatchTask*)(blk + b_cnt);
  uint64_t* d_off_in = (uint64_t*)(blk + b_cnt + b_cta);
  uint64_t* d_off_out = (uint64_t*)(blk + b_cnt + b_cta + b_off);
  LongTask* d_lt = (LongTask*)(blk + b_cnt + b_cta + 2 * b_off);
  c32* d_scr = (c32*)(blk + b_cnt + b_cta + 2 * b_off + b_lt);
  std::vector<LongTask> lt_all;
  lt_all.reserve(nlt);
  for (int ph = 0; ph < 3; ++ph) lt_all.insert(lt_all.end(), lt[ph].begin(), lt[ph].end());
  cudaError_t e = cudaMemsetAsync(counters, 0, kBatchCounters * 4, st);
  if (e == cudaSuccess && !cta.empty())
    e = cudaMemcpyAsync(d_cta, cta.data(), cta.size() * sizeof(BatchTask), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && !off_in.empty()) {
    e = cudaMemcpyAsync(d_off_in, off_in.data(), off_in.size() * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_off_out, off_out.data(), off_out.size() * 8, cudaMemcpyHostToDevice, st);
  }
  if (e == cudaSuccess && nlt)
    e = cudaMemcpyAsync(d_lt, lt_all.data(), nlt * sizeof(LongTask), cudaMemcpyHostToDevice, st);
  // the kernels' shared-memory limits, raised to the largest seen so far
  const size_t smem_cta = 2 * (size_t)buf_cta * 8 + 2 * kBatchMaxG * 8;
  const size_t smem_long = (3 * (size_t)long_cap + 2 * kLongTab) * 8;
  if (e == cudaSuccess && !cta.empty() && smem_cta > reg->cta_smem_set) {
    e = set_smem(k_batch_cta, smem_cta);
    reg->cta_smem_set = smem_cta;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&reg->cta_per_sm, k_batch_cta, kCtaThreads, smem_cta);
  }
  if (e == cudaSuccess && nlt && smem_long > reg->long_smem_set) {
    e = set_smem(k_long_pass<1>, smem_long);
    if (e == cudaSuccess) e = set_smem(k_long_pass<2>, smem_long);
    if (e == cudaSuccess) e = set_smem(k_long_pass<3>, smem_long);
    reg->long_smem_set = smem_long;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&reg->long_per_sm, k_long_pass<2>, kLongThreads,
                                                  smem_long);
  }
  if (e == cudaSuccess && !cta.empty()) {
    BatchParams pt{};
    pt.in = (const c32*)in;
    pt.out = (c32*)out;
    pt.lens = reg->d_lens;
    pt.line_off = d_off_in;
    pt.line_off_out = d_off_out;
    pt.inverse = reg->direction == B2F_INVERSE ? 1u : 0u;
    pt.tw = reg->d_tw;
    pt.tasks = d_cta;
    pt.ntasks = (uint32_t)cta.size();
    pt.counter = counters;
    const unsigned grid = (unsigned)std::min<uint64_t>(
        (uint64_t)reg->nsm * std::max(reg->cta_per_sm, 1), cta.size());
    k_batch_cta<<<grid, kCtaThreads, smem_cta, st>>>(pt, buf_cta);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && nlt) {
    LongParams lp{};
    lp.in = (const c32*)in;
    lp.out = (c32*)out;
    lp.scratch = d_scr;
    lp.tw = reg->d_tw;
    lp.lens = reg->d_long_lens;
    lp.cap = long_cap;
    lp.inverse = reg->direction == B2F_INVERSE ? 1u : 0u;
    uint64_t first = 0;
    for (uint32_t ph = 0; ph < 3 && e == cudaSuccess; ++ph) {
      const uint64_t count = lt[ph].size();
      if (count) {
        lp.tasks = d_lt + first;
        lp.ntasks = (uint32_t)count;
        lp.phase = ph + 1;
        lp.counter = counters + 4 + ph;
        const unsigned grid = (unsigned)std::min<uint64_t>(
            (uint64_t)reg->nsm * std::max(reg->long_per_sm, 1), (count + kLongChunk - 1) / kLongChunk);
        if (ph == 0) k_long_pass<1><<<grid, kLongThreads, smem_long, st>>>(lp);
        else if (ph == 1) k_long_pass<2><<<grid, kLongThreads, smem_long, st>>>(lp);
        else k_long_pass<3><<<grid, kLongThreads, smem_long, st>>>(lp);
        e = cudaGetLastError();
      }
      first += count;
    }
  }
  cudaFreeAsync(blk, st);
  if (e != cudaSuccess)
    return done(fail(B2F_ERR_DEVICE, std::string("line batch launch failed: ") + cudaGetErrorString(e)));
  return done(B2F_OK);
}

}  // namespace b2f

using namespace b2f;

struct b2f_batch {
  BatchPlan* plan;
};

extern "C" {

b2f_status b2f_batch_new_ex(b2f_batch** out, const uint64_t* lengths, const uint64_t* offsets,
                            uint64_t nlines, int32_t direction, int32_t normalization,
                            int32_t device, uint32_t flags) {
  if (!out) return fail(B2F_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  BatchPlan* p = nullptr;
  b2f_status st = create_batch(lengths, offsets, nlines, direction, normalization, device, flags, &p);
  if (st) return st;
  *out = new b2f_batch{p};
  return B2F_OK;
}

b2f_status b2f_batch_new(b2f_batch** out, const uint64_t* lengths, const uint64_t* offsets,
                         uint64_t nlines, int32_t direction, int32_t normalization,
                         int32_t device) {
  return b2f_batch_new_ex(out, lengths, offsets, nlines, direction, normalization, device, 0);
}

void b2f_batch_free(b2f_batch* b) {
  if (!b) return;
  delete b->plan;
  delete b;
}

uint64_t b2f_batch_required_buffer_size_bytes(const b2f_batch* b) {
  return b ? b->plan->extent * 8 : 0;
}

b2f_status b2f_batch_execute(const b2f_batch* b, void* stream, const void* in, uint64_t in_bytes,
                             void* out, uint64_t out_bytes) {
  if (!b || !in || !out) return fail(B2F_ERR_INVALID_ARGUMENT, "null argument");
  const uint64_t need = b->plan->extent * 8;
  if (in_bytes < need || out_bytes < need)
    return fail(B2F_ERR_BUFFER_TOO_SMALL, "BufferViewTooSmall { required: " + std::to_string(need) + " }");
  return run_batch(*b->plan, (cudaStream_t)stream, in, out);
}

b2f_status b2f_batch_execute_parts(const b2f_batch* b, void* stream, const void* in,
                                   uint64_t in_bytes, void* out, uint64_t out_bytes,
                                   uint32_t parts, int32_t sequential) {
  if (!b || !in || !out) return fail(B2F_ERR_INVALID_ARGUMENT, "null argument");
  const uint64_t need = b->plan->extent * 8;
  if (in_bytes < need || out_bytes < need)
    return fail(B2F_ERR_BUFFER_TOO_SMALL, "BufferViewTooSmall { required: " + std::to_string(need) + " }");
  return run_batch(*b->plan, (cudaStream_t)stream, in, out, parts, sequential != 0);
}

b2f_status b2f_batch_execute_host(const b2f_batch* b, void* stream, const void* host_in,
                                  void* host_out, void* dev_in, void* dev_out, uint64_t bytes) {
  if (!b || !host_in || !host_out || !dev_in || !dev_out)
    return fail(B2F_ERR_INVALID_ARGUMENT, "null argument");
  const uint64_t need = b->plan->extent * 8;
  if (bytes < need)
    return fail(B2F_ERR_BUFFER_TOO_SMALL, "BufferViewTooSmall { required: " + std::to_string(need) + " }");
  return run_batch_host(*b->plan, (cudaStream_t)stream, host_in, host_out, dev_in, dev_out);
}

b2f_status b2f_batch_diagnostics_json(const b2f_batch* b, char* buf, uint64_t* len) {
  if (!b || !len) return fail(B2F_ERR_INVALID_ARGUMENT, "null argument");
  const std::string& j = b->plan->diag;
  const uint64_t cap = *len;
  *len = j.size();
  if (buf && cap > 0) {
    const uint64_t n = std::min<uint64_t>(cap - 1, j.size());
    std::memcpy(buf, j.data(), n);
    buf[n] = 0;
    if (n < j.size()) return fail(B2F_ERR_BUFFER_TOO_SMALL, "diagnostics buffer too small");
  }
  return B2F_OK;
}

}  // extern "C"
