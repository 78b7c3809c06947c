// Column tiles of power-of-two lines staged through the Tensor Memory
// Accelerator (TMA), f32.
//
// A column pass (lines of N <= 256 points whose points lie in_es elements
// apart, adjacent lines adjacent in memory) reads its data as G x N tiles:
// G adjacent columns, all N points.  The register kernel (regfft.cuh,
// k_pow2<float,16,true>) loads a tile with one 8-byte load per value and
// hides the latency only through the other CTAs of the SM.  Here each CTA is
// persistent: one thread issues cp.async.bulk.tensor for the CTA's next tile
// (a 4D tensor map over columns, points, middle and outer blocks of this
// GPU's buffer; no multicast) into the other of two shared-memory tile
// buffers while the CTA transforms the current one, with an mbarrier per
// buffer counting the transaction bytes.  The current buffer is read into
// registers, then reused as the stage-exchange area of the register FFT,
// so two buffers of G x LD values are all the shared memory a CTA needs.
//
// Opt-in (tuning tma_tiles = 1): measured against the plain-load register
// kernel on 2048 x 4096, 4096 x 2048, 8192 x 8192, 2^24 and 256^3, it is
// 0-13 % slower at 3 CTAs per SM (80 registers) and 3-16 % at 2 — these
// passes are bound by instruction issue (70-100 instructions a point), and
// staging adds a shared-memory read per value without removing a global one.
//
// Every mbarrier wait is bounded; a wait that gives up sets bit 2 of the
// pass's device flag, waits (bounded) for the copy the CTA still has in
// flight and ends the CTA's loop.  The host reads the flag through
// b2f_plan_device_status.
#include <cuda.h>

#include <mutex>

#include "kernels_impl.cuh"
#include "regfft.cuh"

namespace b2f {
namespace {

constexpr uint32_t kTileWaitLimit = 1u << 26;  // mbarrier polls before giving up
constexpr uint32_t kTileFlag = 4u;             // bit of the pass's device flag

__device__ inline bool tile_wait(uint32_t mbar, uint32_t parity) {
  for (uint32_t it = 0; it < kTileWaitLimit; ++it) {
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

// Tile t: its columns' first index, middle and outer block (the order of
// group_of: tiles fastest, then middle, then outer).
struct TileCoord {
  uint32_t x, z, w;
};
__device__ inline TileCoord tile_coord(const LineIO& io, uint32_t G, uint64_t t) {
  const uint64_t rest = t / io.tiles;
  const uint64_t tile = t - rest * io.tiles;
  TileCoord c;
  c.w = (uint32_t)(rest / io.mid_n);
  c.z = (uint32_t)(rest - (uint64_t)c.w * io.mid_n);
  c.x = (uint32_t)(tile * G);
  return c;
}

__device__ inline void tile_issue(const CUtensorMap* map, uint32_t dst, uint32_t mbar,
                                  uint32_t bytes, TileCoord c) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mbar), "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c.x), "r"(0), "r"(c.z), "r"(c.w), "r"(mbar)
      : "memory");
}

// First-stage inputs of a radix-R stage from a tile in TMA layout (point n
// of column c at n * G + c): element j + q*NR, j = t + u*TL.
template <int R, int E>
__device__ inline void tile_read(cpx<float> (&v)[E], const cpx<float>* T, uint32_t t, uint32_t TL,
                                 uint32_t NR, uint32_t G, uint32_t c) {
  constexpr int NB = E / R;
#pragma unroll
  for (int u = 0; u < NB; ++u)
#pragma unroll
    for (int q = 0; q < R; ++q) v[u * R + q] = T[(t + u * TL + q * NR) * G + c];
}
template <int E>
__device__ inline void tile_read_any(uint32_t R, cpx<float> (&v)[E], const cpx<float>* T,
                                     uint32_t t, uint32_t TL, uint32_t NR, uint32_t G,
                                     uint32_t c) {
  switch (R) {
    case 2: tile_read<2, E>(v, T, t, TL, NR, G, c); break;
    case 4: tile_read<4, E>(v, T, t, TL, NR, G, c); break;
    case 8: tile_read<8, E>(v, T, t, TL, NR, G, c); break;
    default: tile_read<16, E>(v, T, t, TL, NR, G, c); break;
  }
}

}  // namespace

// Persistent column-tile FFT: ntiles tiles of G columns x N points (N a power
// of two, 16 <= N <= 256, E = 16 values a thread, G * N / 16 threads).
// Dynamic shared memory: 1024 bytes of alignment slack, then two tile
// buffers of `buf` complex values each (buf a multiple of 128), each
// 1024-byte aligned.
__global__ void __launch_bounds__(256, 3)
    k_pow2_tma(const __grid_constant__ CUtensorMap map, const __grid_constant__ LinesParams p,
               uint64_t ntiles, uint32_t buf, unsigned int* flag) {
  constexpr int E = 16, PAD = 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t s_mbar[2];
  using C = cpx<float>;
  const uint32_t raw = (uint32_t)__cvta_generic_to_shared(smem_raw);
  C* const tiles = reinterpret_cast<C*>(smem_raw + (((raw + 1023u) & ~1023u) - raw));
  const uint32_t tid = threadIdx.x;
  const uint32_t N = p.N, G = p.G, LD = p.LD, TL = N / E;
  const uint32_t c = tid & (G - 1), t = tid >> (31 - __clz(G));
  const uint32_t bytes = G * N * (uint32_t)sizeof(C);
  const uint32_t mb0 = (uint32_t)__cvta_generic_to_shared(&s_mbar[0]);
  const uint32_t mb1 = (uint32_t)__cvta_generic_to_shared(&s_mbar[1]);
  const uint32_t sb0 = (uint32_t)__cvta_generic_to_shared(tiles);
  const uint32_t sb1 = sb0 + buf * (uint32_t)sizeof(C);
  const C* tw = (p.flags & PF_TW_TABLE) ? (const C*)p.tw : nullptr;
  const Schedule& sch = p.sch;
  const uint32_t last = sch.nst - 1;
  const float sc = (float)p.scale;
  if (tid == 0) {
    asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&map)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    if (blockIdx.x < ntiles) tile_issue(&map, sb0, mb0, bytes, tile_coord(p.io, G, blockIdx.x));
  }
  __syncthreads();
  uint32_t k = 0;
  for (uint64_t ti = blockIdx.x; ti < ntiles; ti += gridDim.x, ++k) {
    const uint32_t cur = k & 1;
    // the next tile into the other buffer: its last reader (the previous
    // tile's stage exchanges) finished before the barrier that ended it
    const uint64_t tn = ti + gridDim.x;
    if (tid == 0) {
      if (tn < ntiles) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        tile_issue(&map, cur ? sb0 : sb1, cur ? mb0 : mb1, bytes, tile_coord(p.io, G, tn));
      }
    }
    // every thread waits (bounded); the CTA goes on only if all saw the tile
    const bool landed = tile_wait(cur ? mb1 : mb0, (k >> 1) & 1);
    if (!__syncthreads_and(landed)) {
      if (tid == 0) {
        atomicOr(flag, kTileFlag);
        // the next tile's copy may still be landing: wait for it (bounded)
        if (tn < ntiles) tile_wait(cur ? mb0 : mb1, ((k + 1) >> 1) & 1);
      }
      break;
    }
    C* const T = tiles + (size_t)cur * buf;
    const Group g = group_of(p.io, G, ti);
    const bool valid = c < g.nvalid;
    // first-stage inputs: point j + q*NR of column c sits at (j + q*NR)*G + c
    C v[E];
    tile_read_any<E>(sch.st[0].R, v, T, t, TL, sch.st[0].NR, G, c);
    if (p.flags & PF_CONJ_IN) {
#pragma unroll
      for (int i = 0; i < E; ++i) v[i].im = -v[i].im;
    }
    __syncthreads();  // the tile is in registers: its buffer becomes the exchange area
    C* line = T + c * LD;
#pragma unroll 1
    for (uint32_t s = 0;; ++s) {
      const StageDesc& sd = sch.st[s];
      reg_compute_any<float, E, PAD>(sd.R, v, t, TL, sd.Ns, tw, sd.tw_off);
      if (s == last) break;
      reg_write_any<float, E, PAD>(sd.R, v, line, t, TL, sd.Ns);
      __syncthreads();
      reg_read_any<float, E, PAD>(sch.st[s + 1].R, v, line, t, TL, sch.st[s + 1].NR);
      __syncthreads();
    }
    if (valid) {
      const StageDesc& sl = sch.st[last];
      const uint64_t row = (p.flags & PF_TW_STORE) ? fdiv((uint32_t)(g.c0 + c), p.d_tw) : 0;
      reg_store_any<float, E>(sl.R, v, (C*)p.out, g.out0 + (int64_t)c * g.dl_out, p.io.out_es, t,
                              TL, sl.Ns, p.flags, sc, row, p);
    }
  }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library); null when unavailable.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_fn() {
  static std::once_flag once;
  static EncodeTiledFn fn = nullptr;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
    cudaGetLastError();
  });
  return fn;
}

bool tma_tile_shape_ok(const LinesParams& lp, uint64_t outer_n) {
  const LineIO& io = lp.io;
  const uint32_t N = lp.N, G = lp.G;
  if (N < 16 || N > 256 || (N & (N - 1)) || G < 4 || (G & (G - 1)) || G * (N / 16) > 256)
    return false;
  if (io.in_inner != 1 || io.out_inner != 1 || io.in_es <= 0) return false;
  // row strides of the 4D view: multiples of 16 bytes (even element counts)
  if ((io.in_es & 1) || (io.mid_n > 1 && (io.in_mid & 1)) || (outer_n > 1 && (io.in_outer & 1)))
    return false;
  return io.inner_n >= 1 && io.mid_n >= 1 && outer_n >= 1;
}

size_t tma_tile_buf(const LinesParams& lp) {
  const size_t b = (size_t)lp.G * lp.LD;
  return (b + 127) & ~(size_t)127;  // 1024-byte multiple (128 complex values)
}

// Encodes the pass's input view and launches the persistent tile kernel;
// returns false (nothing launched) when the view cannot be a tensor map
// (base address or strides not 16-byte aligned, no driver entry point).
bool launch_pow2_tma(const LinesParams& lp, uint64_t ntiles, uint64_t outer_n, unsigned threads,
                     unsigned grid, unsigned int* flag, cudaStream_t st, cudaError_t* err) {
  *err = cudaSuccess;
  EncodeTiledFn enc = encode_fn();
  if (!enc || ((uintptr_t)lp.in & 15)) return false;
  const LineIO& io = lp.io;
  const uint64_t es = sizeof(cpx<float>);
  cuuint64_t dims[4] = {io.inner_n, lp.N, io.mid_n, outer_n};
  cuuint64_t strides[3] = {(cuuint64_t)io.in_es * es,
                           (cuuint64_t)(io.mid_n > 1 ? io.in_mid : io.in_es * lp.N) * es,
                           (cuuint64_t)(outer_n > 1 ? io.in_outer : io.in_es * lp.N) * es};
  cuuint32_t box[4] = {lp.G, lp.N, 1, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUtensorMap map;
  if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<void*>(lp.in), dims, strides, box,
          estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  const uint32_t buf = (uint32_t)tma_tile_buf(lp);
  const size_t smem = 2 * (size_t)buf * es + 1024;
  static std::mutex mu;
  static size_t smem_set = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (smem > smem_set) {
      *err = cudaFuncSetAttribute(k_pow2_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem);
      if (*err != cudaSuccess) return true;
      smem_set = smem;
    }
  }
  k_pow2_tma<<<grid, threads, smem, st>>>(map, lp, ntiles, buf, flag);
  *err = cudaGetLastError();
  return true;
}

int tma_tile_ctas_per_sm(const LinesParams& lp, unsigned threads) {
  const size_t smem = 2 * tma_tile_buf(lp) * sizeof(cpx<float>) + 1024;
  int n = 0;
  cudaFuncSetAttribute(k_pow2_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_pow2_tma, threads, smem) != cudaSuccess)
    n = 0;
  cudaGetLastError();
  return n;
}

}  // namespace b2f
