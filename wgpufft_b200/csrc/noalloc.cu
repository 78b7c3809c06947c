// 1D complex f32 transforms for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: code running inside
// a CUDA graph that is being captured with allocations forbidden, plug-ins
// handed a fixed device-memory budget by their host application, and
// real-time paths that must not hit the allocator's locks or its
// synchronisation.  b2f_c2c_1d_f32_noalloc serves them: it plans on the host
// with no device tables (stage twiddles computed in-kernel) and, for lengths
// too long for one CTA, runs the two four-step passes through a fixed,
// statically allocated device scratch array instead of a plan workspace.
#include <cstring>
#include <memory>
#include <mutex>

#include "plan.h"

namespace b2f {

// Capacity of the static scratch: 32 MiB, i.e. 4,194,304 complex f32 points
// (n * batch) for the multi-pass route.  Every GPU that loads this library
// holds this array from module load until the process exits.
constexpr uint64_t kNoAllocScratchBytes = 32ull << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the scratch array per device, looked up once with that
// device current (the host-side symbol is not a device address).  The
// cached address belongs to the device's primary context: it stays valid
// while that context lives, i.e. until process exit unless the caller
// resets the device (cudaDeviceReset), which this entry point does not
// support.
static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[128] = {};

static b2f_status noalloc_scratch(int dev, void** out) {
  if (dev < 0 || dev >= 128) return fail(B2F_ERR_DEVICE, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(B2F_ERR_DEVICE, std::string("cudaGetSymbolAddress of the static scratch failed: ") +
                                      cudaGetErrorString(e));
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return B2F_OK;
}

static b2f_status noalloc_run(const Plan& plan, cudaStream_t st, const void* in, void* out,
                              void* const* ws) {
  void* bufs[2 + kNumWorkspaces] = {const_cast<void*>(in), out};
  for (int i = 0; i < kNumWorkspaces; ++i) bufs[2 + i] = ws[i];
  cudaError_t e = cudaSuccess;
  for (const Pass& p0 : plan.passes) {
    Pass p = p0;
    void* src = bufs[p.src];
    void* dst = bufs[p.dst];
    switch (p.kind) {
      case Pass::LINES:
        p.lines.in = src;
        p.lines.out = dst;
        e = launch_lines(plan.prec, p.lines, p.grid, p.threads, p.smem, st);
        break;
      case Pass::POW2:
        p.lines.in = src;
        p.lines.out = dst;
        e = launch_pow2(plan.prec, p.pow2_E, p.colmajor, p.lines, p.grid, p.threads, p.smem, st);
        break;
      case Pass::SCALE_COPY:
        e = launch_scale_copy(plan.prec, src, dst, p.copy_n, p.copy_scale, p.copy_conj, st);
        break;
      default:
        return fail(B2F_ERR_UNSUPPORTED_LENGTH, "route needs device tables (Rader/Bluestein)");
    }
    if (e != cudaSuccess) break;
  }
  if (e != cudaSuccess)
    return fail(B2F_ERR_DEVICE, std::string("kernel launch failed: ") + cudaGetErrorString(e));
  return B2F_OK;
}

}  // namespace b2f

using namespace b2f;

extern "C" b2f_status b2f_c2c_1d_f32_noalloc(void* stream, const void* in, uint64_t in_bytes,
                                             void* out, uint64_t out_bytes, uint64_t n,
                                             uint64_t batch, int32_t direction,
                                             int32_t normalization) {
  if (!in || !out) return fail(B2F_ERR_INVALID_ARGUMENT, "null buffer");
  Config cfg;
  cfg.shape = {n};
  cfg.axes = {0};
  cfg.batch = batch;
  cfg.direction = direction;
  cfg.normalization = normalization;
  cfg.precision = B2F_F32;
  cfg.tuning.twiddle_table = 0;  // stage twiddles computed in-kernel: no tables
  b2f_status st = validate_config(cfg);
  if (st) return st;
  if (!is_smooth13(n))
    return fail(B2F_ERR_UNSUPPORTED_LENGTH,
                "UnsupportedLength { len: " + std::to_string(n) +
                    " } (the allocation-free entry point takes 2,3,5,7,11,13-smooth lengths)");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(B2F_ERR_DEVICE, "no current device");
  // host-only planning (no device allocation) within this device's own
  // shared-memory limit (a device attribute query allocates nothing)
  int smem = 0;
  if (cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
      smem <= 0)
    return fail(B2F_ERR_DEVICE, "could not read the device's shared-memory limit");
  Plan* raw = nullptr;
  st = create_plan(cfg, B2F_C2C, -2, &raw, (size_t)smem);
  if (st) return st;
  std::unique_ptr<Plan> plan(raw);
  if (plan->table_bytes != 0)
    return fail(B2F_ERR_UNSUPPORTED_LENGTH, "route needs device tables");
  const uint64_t bytes = n * batch * 8;
  if (in_bytes < bytes || out_bytes < bytes)
    return fail(B2F_ERR_BUFFER_TOO_SMALL,
                "BufferViewTooSmall { required: " + std::to_string(bytes) + " }");
  uint64_t need = 0;
  for (uint64_t w : plan->ws_bytes) need += (w + 255) / 256 * 256;
  if (need > kNoAllocScratchBytes)
    return fail(B2F_ERR_WORKSPACE_TOO_SMALL,
                "WorkspaceTooSmall { required: " + std::to_string(need) +
                    ", limit: " + std::to_string(kNoAllocScratchBytes) +
                    " } (n * batch above the static scratch of the allocation-free entry point)");
  void* scratch = nullptr;
  void* ws[kNumWorkspaces] = {};
  if (need > 0) {
    st = noalloc_scratch(dev, &scratch);
    if (st) return st;
    uint64_t off = 0;
    for (int i = 0; i < kNumWorkspaces; ++i) {
      if (plan->ws_bytes[i] == 0) continue;
      ws[i] = (unsigned char*)scratch + off;
      off += (plan->ws_bytes[i] + 255) / 256 * 256;
    }
  }
  return noalloc_run(*plan, (cudaStream_t)stream, in, out, ws);
}
