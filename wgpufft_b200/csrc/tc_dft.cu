// Tensor-core DFT layer (the precision form): batched length-64 complex
// DFTs as real GEMMs on the 5th-generation tensor cores (tcgen05), in f32
// accuracy from split TF32 operands.
//
// The complex DFT y = F x of a line is the real product
//   [yr; yi] = A [xr; xi],  A = [[C, S], [-S, C]],  C = cos(2 pi r m / 64),
//   S = sin(2 pi r m / 64)                                   (128 x 128),
// so a tile of 32 lines is D (128 x 32) = A (128 x 128) * B^T with B the
// 32 x 128 matrix of the lines' [re; im] values: tcgen05.mma with M = 128,
// N = 32 per K-step of 8.  Each operand is split into a TF32 high part (low
// 13 bits cleared: exact) and the remainder, and three products
//   D = Ah Bh + Ah Bl + Al Bh
// accumulate in FP32 in tensor memory: the dropped Al Bl term and the
// TF32 truncation of the remainders are ~2^-21 of each term, so the result
// stays well inside the 2e-6 relative-L2 f32 tolerance (BF16 splits need
// six products for that accuracy, which would cost more tensor time than
// the HBM pass this layer replaces).
//
// Operands sit in shared memory in the K-major, no-swizzle canonical
// layout: 8-row x 16-byte core matrices, consecutive along K (LBO = 128 B),
// row groups 4096 B apart (SBO).  One thread issues a tile's 48 MMAs and
// commits them to the tile's mbarrier; waits on it are bounded (past the
// limit the kernel records an error, waits once more and stops).  The
// accumulator is read with tcgen05.ld (warp w: TMEM lanes 32 (w % 4).., one
// half of the lines per warpgroup), transposed through shared memory and
// stored coalesced.  The kernel is persistent and software-pipelined over
// two operand buffers, two 32-column accumulators and two mbarriers.
#include <cstdint>
#include <cstring>
#include <vector>

#include "hostfft.h"
#include "plan.h"

namespace b2f {

namespace {

constexpr uint32_t kTcR = 64, kTcM = 128, kTcK = 128, kTcN = 32;  // N: lines per tile
constexpr uint32_t kTcKC = kTcK / 4;                  // 16-byte chunks along K
constexpr uint32_t kTcABytes = kTcM * kTcK * 4;       // one split half of A: 64 KB
constexpr uint32_t kTcBBytes = kTcN * kTcK * 4;       // one split half of a B tile: 16 KB
constexpr uint32_t kTcSmem = 2 * kTcABytes + 4 * kTcBBytes;  // A halves + two B buffers: 192 KB
constexpr uint32_t kTcWaitLimit = 1u << 26;           // mbarrier polls before giving up
constexpr uint32_t kTcThreads = 256;                  // two warpgroups
constexpr uint32_t kTcPer = kTcN * kTcR / kTcThreads;   // complex values per thread and tile

__host__ __device__ inline uint32_t tc_off(uint32_t row, uint32_t k) {
  return (((row >> 3) * kTcKC + (k >> 2)) << 7) + ((row & 7) << 4) + ((k & 3) << 2);
}

__device__ inline uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ inline uint64_t tc_desc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((128u >> 4) & 0x3FFF) << 16;          // LBO: next core matrix along K
  d |= (uint64_t)(((kTcKC * 128u) >> 4) & 0x3FFF) << 32;  // SBO: next 8 rows
  d |= (uint64_t)1 << 46;                                // descriptor version (sm_100)
  return d;                                              // base offset 0, no swizzle
}

// kind::tf32, D in F32, A and B K-major, M = 128, N = 32
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((kTcN >> 3) << 17) |
                              ((kTcM >> 4) << 24);

__device__ inline float tf32_hi(float x) {
  return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u);
}

__device__ inline void tc_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(kTcIdesc), "r"(accumulate), "r"(0), "r"(0), "r"(0),
        "r"(0));
}

__device__ inline void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ inline void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}

__device__ inline void tc_ld16(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

// Bounded wait for phase `parity` of the mbarrier; false when it gave up.
__device__ inline bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (uint32_t it = 0; it < kTcWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Element j of thread tid within a tile: each group of 32 consecutive
// elements (a warp's) covers 8 lines x 4 consecutive positions, so the
// split stores of a warp hit 32 different banks (a core-matrix row is 16
// bytes of one line, rows of 8 lines are consecutive).
__device__ inline void tc_elem(uint32_t tid, uint32_t j, uint32_t& n, uint32_t& m) {
  const uint32_t e = tid + j * kTcThreads, g = e >> 5, lane = e & 31;
  n = (g & (kTcN / 8 - 1)) * 8 + (lane >> 2);
  m = (g / (kTcN / 8)) * 4 + (lane & 3);
}

// Loads of one tile into registers.
__device__ inline void tc_load(const float2* __restrict__ in, uint64_t line0, uint64_t nlines,
                               uint32_t tid, float2* reg) {
#pragma unroll
  for (uint32_t j = 0; j < kTcPer; ++j) {
    uint32_t n, m;
    tc_elem(tid, j, n, m);
    reg[j] = (line0 + n < nlines) ? in[(line0 + n) * kTcR + m] : make_float2(0.0f, 0.0f);
  }
}

// Splits the registers of a tile into the buffer's high and low operand halves.
__device__ inline void tc_split(const float2* reg, unsigned char* bh, unsigned char* bl,
                                uint32_t inverse, uint32_t tid) {
#pragma unroll
  for (uint32_t j = 0; j < kTcPer; ++j) {
    uint32_t n, m;
    tc_elem(tid, j, n, m);
    float2 v = reg[j];
    if (inverse) v.y = -v.y;
    const float hr = tf32_hi(v.x), hi = tf32_hi(v.y);
    *reinterpret_cast<float*>(bh + tc_off(n, m)) = hr;
    *reinterpret_cast<float*>(bl + tc_off(n, m)) = v.x - hr;
    *reinterpret_cast<float*>(bh + tc_off(n, kTcR + m)) = hi;
    *reinterpret_cast<float*>(bl + tc_off(n, kTcR + m)) = v.y - hi;
  }
}

// Persistent, software-pipelined: while the MMAs of tile i+1 run and the
// loads of tile i+2 are in flight, tile i's accumulator is read out and
// stored.  Two operand buffers (each the staging area of its tile's output
// once its MMAs are done), two TMEM accumulators, two mbarriers.
__global__ void __launch_bounds__(kTcThreads, 1)
    k_dft64_tc(const float2* __restrict__ in, float2* __restrict__ out, const float* __restrict__ atab,
               uint64_t nlines, float scale, uint32_t inverse, unsigned int* err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* sAh = sm;
  unsigned char* sAl = sm + kTcABytes;
  unsigned char* sB = sm + 2 * kTcABytes;  // buffer b: high half at b * 2 kTcBBytes, low half after it
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t s_taddr;
  __shared__ uint32_t s_fail;
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  {
    const uint4* src = reinterpret_cast<const uint4*>(atab);
    uint4* dst = reinterpret_cast<uint4*>(sm);
    for (uint32_t i = tid; i < 2 * kTcABytes / 16; i += kTcThreads) dst[i] = src[i];
  }
  const uint32_t mb0 = smem_u32(&mbar[0]), mb1 = smem_u32(&mbar[1]);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    s_fail = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&s_taddr)),
                 "r"(2 * kTcN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t taddr = s_taddr;
  const uint64_t ntiles = (nlines + kTcN - 1) / kTcN;
  const uint64_t step = gridDim.x;
  uint32_t parity[2] = {0, 0};
  bool pending[2] = {false, false};  // MMAs committed to mbar[b] and not yet waited for
  auto bufh = [&](uint32_t b) { return sB + b * 2 * kTcBBytes; };
  auto bufl = [&](uint32_t b) { return sB + b * 2 * kTcBBytes + kTcBBytes; };
  // split registers into buffer b and issue its MMAs into accumulator b
  auto launch_tile = [&](const float2* reg, uint32_t b) {
    tc_split(reg, bufh(b), bufl(b), inverse, tid);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      const uint32_t a[3] = {smem_u32(sAh), smem_u32(sAh), smem_u32(sAl)};
      const uint32_t bb[3] = {smem_u32(bufh(b)), smem_u32(bufl(b)), smem_u32(bufh(b))};
      const uint32_t d = taddr + b * kTcN;
#pragma unroll 1
      for (int prod = 0; prod < 3; ++prod)
#pragma unroll 1
        for (uint32_t s = 0; s < kTcK / 8; ++s)
          tc_mma(d, tc_desc(a[prod] + 256 * s), tc_desc(bb[prod] + 256 * s),
                 (prod | s) != 0 ? 1u : 0u);
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                       b ? mb1 : mb0)
                   : "memory");
    }
    pending[b] = true;
  };
  float2 reg[kTcPer];
  uint64_t t = blockIdx.x;
  if (t < ntiles) {
    tc_load(in, t * kTcN, nlines, tid, reg);
    launch_tile(reg, 0);
    if (t + step < ntiles) tc_load(in, (t + step) * kTcN, nlines, tid, reg);
  }
  for (uint32_t i = 0; t < ntiles; ++i, t += step) {
    const uint32_t cur = i & 1, nxt = cur ^ 1;
    // next tile: its registers were loaded during the previous round
    if (t + step < ntiles) {
      launch_tile(reg, nxt);
      if (t + 2 * step < ntiles) tc_load(in, (t + 2 * step) * kTcN, nlines, tid, reg);
    }
    // this tile's MMAs
    bool done = mbar_wait(cur ? mb1 : mb0, parity[cur]);
    if (!done) {
      if (tid == 0) atomicOr(err, 1u);
      s_fail = 1;
      done = mbar_wait(cur ? mb1 : mb0, parity[cur]);  // second bounded wait before moving on
    }
    // still pending after both waits: the drain below waits for it once more
    if (done) {
      parity[cur] ^= 1;
      pending[cur] = false;
    }
    tc_fence_after();
    __syncthreads();
    if (s_fail) break;
    // accumulator row r = 32 (warp % 4) + lane: output r (re, r < 64) or r - 64 (im);
    // warpgroup warp / 4 reads lines 16 (warp / 4) .. + 16
    uint32_t v[16];
    const uint32_t c0 = (warp >> 2) * 16;
    tc_ld16(taddr + ((32 * (warp & 3)) << 16) + cur * kTcN + c0, v);
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
    float* stage = reinterpret_cast<float*>(bufh(cur));  // kTcN x 129 floats
    const uint32_t r = 32 * (warp & 3) + lane;
#pragma unroll
    for (uint32_t n = 0; n < 16; ++n) stage[(c0 + n) * 129 + r] = __uint_as_float(v[n]);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint64_t line0 = t * kTcN;
#pragma unroll
    for (uint32_t j = 0; j < kTcPer; ++j) {
      const uint32_t e = tid + j * kTcThreads, n = e >> 6, m = e & 63;
      if (line0 + n < nlines) {
        float2 y = make_float2(stage[n * 129 + m] * scale, stage[n * 129 + kTcR + m] * scale);
        if (inverse) y.y = -y.y;
        out[(line0 + n) * kTcR + m] = y;
      }
    }
    __syncthreads();  // the staging area becomes an operand buffer again
  }
  // no MMA may still write tensor memory when it is freed: every committed
  // group is waited for (bounded); a group that never completes (a device
  // fault: each wait allows about a second) is recorded in bit 1 of the
  // error flag, which the host reports (b2f_plan_device_status), and the
  // columns are freed regardless, since a CTA that kept them would stall
  // every later allocation on its SM
  for (uint32_t b = 0; b < 2; ++b)
    if (pending[b] && !mbar_wait(b ? mb1 : mb0, parity[b]) && tid == 0) atomicOr(err, 2u);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr),
                 "r"(2 * kTcN)
                 : "memory");
}

}  // namespace

// The two split halves of A in the operand layout (host side; FP64 angles
// reduced exactly, rounded once).
std::vector<float> dft64_tc_table() {
  std::vector<float> t(2 * kTcM * kTcK, 0.0f);
  for (uint32_t r = 0; r < kTcR; ++r)
    for (uint32_t m = 0; m < kTcR; ++m) {
      const cd w = root_fwd((uint64_t)r * m, kTcR);  // cos - i sin
      const double c = w.real(), s = -w.imag();
      const double vals[2][2] = {{c, s}, {-s, c}};
      for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) {
          const double a = vals[i][j];
          const float x = (float)a;
          uint32_t bits;
          std::memcpy(&bits, &x, 4);
          bits &= 0xFFFFE000u;
          float hi;
          std::memcpy(&hi, &bits, 4);
          const float lo = (float)(a - (double)hi);
          const uint32_t row = r + i * kTcR, k = m + j * kTcR;
          t[tc_off(row, k) / 4] = hi;
          t[(kTcABytes + tc_off(row, k)) / 4] = lo;
        }
    }
  return t;
}

cudaError_t launch_dft64_tc(const void* in, void* out, const float* table, uint64_t nlines,
                            float scale, bool inverse, unsigned int* err, unsigned grid,
                            cudaStream_t st) {
  static bool attr_done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr_done[dev]) {
    const cudaError_t e =
        cudaFuncSetAttribute(k_dft64_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
    if (e != cudaSuccess) return e;
    attr_done[dev] = true;
  }
  k_dft64_tc<<<grid, kTcThreads, kTcSmem, st>>>(reinterpret_cast<const float2*>(in),
                                         reinterpret_cast<float2*>(out), table, nlines, scale,
                                         inverse ? 1u : 0u, err);
  return cudaGetLastError();
}

}  // namespace b2f
