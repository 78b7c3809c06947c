// Strided and offset caller views (b2f_plan_execute_logical_views): the
// crate's FftLogicalView / FftLogicalLayout execution
// (src/runtime/logical_io.rs:5-200, src/plan.rs:580-806).  A view places
// logical element i of batch b of an endpoint at element
//   element_offset + b * batch_stride + i * element_stride
// of the caller's buffer, in units of the endpoint's element (complex value
// of the plan's precision; a real value for the real side of R2C/C2R).
// Contiguous and offset-only views run the plan in place on the caller's
// memory; strided views gather the input into a staging buffer owned by the
// plan, run the plan, and scatter the output, each a coalesced-on-one-side
// copy kernel.
#include <cstring>
#include <string>

#include "plan.h"

namespace b2f {

struct ViewShape {
  uint64_t offset, stride, batch_stride, per_batch, batch;
  size_t elem;  // bytes of one element
  bool contiguous() const { return stride == 1 && (batch <= 1 || batch_stride == per_batch); }
};

template <class T>
__global__ void k_view_gather(T* __restrict__ dst, const T* __restrict__ src, uint64_t per_batch,
                              uint64_t total, uint64_t offset, uint64_t stride, uint64_t bstride) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = e / per_batch, i = e - b * per_batch;
    dst[e] = src[offset + b * bstride + i * stride];
  }
}

template <class T>
__global__ void k_view_scatter(T* __restrict__ dst, const T* __restrict__ src, uint64_t per_batch,
                               uint64_t total, uint64_t offset, uint64_t stride, uint64_t bstride) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = e / per_batch, i = e - b * per_batch;
    dst[offset + b * bstride + i * stride] = src[e];
  }
}

static cudaError_t view_copy(bool gather, void* dst, const void* src, const ViewShape& v,
                             cudaStream_t st) {
  const uint64_t total = v.per_batch * v.batch;
  if (total == 0) return cudaSuccess;
  const unsigned threads = 256;
  const unsigned grid = (unsigned)std::min<uint64_t>((total + threads - 1) / threads, 148ull * 16);
  switch (v.elem) {
#define B2F_VIEW_CASE(BYTES, T)                                                                   \
  case BYTES:                                                                                     \
    if (gather)                                                                                   \
      k_view_gather<T><<<grid, threads, 0, st>>>((T*)dst, (const T*)src, v.per_batch, total,      \
                                                 v.offset, v.stride, v.batch_stride);             \
    else                                                                                          \
      k_view_scatter<T><<<grid, threads, 0, st>>>((T*)dst, (const T*)src, v.per_batch, total,     \
                                                  v.offset, v.stride, v.batch_stride);            \
    break;
    B2F_VIEW_CASE(4, float)
    B2F_VIEW_CASE(8, float2)
    B2F_VIEW_CASE(16, float4)
#undef B2F_VIEW_CASE
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// FftLogicalLayout::validate / required_element_span
// (src/runtime/logical_io.rs:112-147) plus the view's size check.
static b2f_status bind_view(const b2f_logical_layout* layout, uint64_t per_batch, uint64_t batch,
                            size_t elem, uint64_t view_bytes, const char* role, ViewShape* out) {
  ViewShape v{0, 1, per_batch, per_batch, batch, elem};
  if (layout) {
    v.offset = layout->element_offset;
    v.stride = layout->element_stride;
    if (v.stride == 0) return fail(B2F_ERR_LAYOUT_ZERO_STRIDE, "BufferLayoutZeroStride");
  }
  const unsigned __int128 span = (unsigned __int128)v.stride * (per_batch - 1) + 1;
  const unsigned __int128 bs =
      (layout && layout->batch_stride) ? (unsigned __int128)layout->batch_stride : span;
  if (bs < span)
    return fail(B2F_ERR_LAYOUT_BATCH_STRIDE_TOO_SMALL,
                "BufferLayoutBatchStrideTooSmall { required: " + std::to_string((uint64_t)span) +
                    ", actual: " + std::to_string((uint64_t)bs) + " }");
  const unsigned __int128 need_elems = (unsigned __int128)v.offset + bs * (batch - 1) + span;
  const unsigned __int128 need_bytes = need_elems * elem;
  if (need_bytes >> 63)
    return fail(B2F_ERR_LAYOUT_TOO_LARGE, std::string("BufferLayoutTooLarge: the ") + role +
                                              " view's span does not fit 63 bits");
  if ((uint64_t)need_bytes > view_bytes)
    return fail(B2F_ERR_LAYOUT_OUT_OF_BOUNDS,
                std::string("BufferLayoutOutOfBounds { role: ") + role +
                    ", required_bytes: " + std::to_string((uint64_t)need_bytes) +
                    ", actual_bytes: " + std::to_string(view_bytes) + " }");
  v.batch_stride = (uint64_t)bs;
  *out = v;
  return B2F_OK;
}

static b2f_status staging(const Plan& plan, void** slot, uint64_t bytes) {
  std::lock_guard<std::mutex> lk(plan.copy_mu);
  if (*slot) return B2F_OK;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(plan.device);
  const cudaError_t e = cudaMalloc(slot, std::max<uint64_t>(bytes, 16));
  if (prev >= 0) cudaSetDevice(prev);
  if (e != cudaSuccess) {
    *slot = nullptr;
    cudaGetLastError();
    return fail(B2F_ERR_RESOURCE_ALLOCATION, "logical-view staging buffer allocation failed");
  }
  return B2F_OK;
}

}  // namespace b2f

using namespace b2f;

extern "C" b2f_status b2f_plan_execute_logical_views(const b2f_plan* handle, void* stream,
                                                     const void* in, uint64_t in_bytes,
                                                     const b2f_logical_layout* in_layout,
                                                     void* out, uint64_t out_bytes,
                                                     const b2f_logical_layout* out_layout) {
  if (!handle || !handle->plan) return fail(B2F_ERR_INVALID_ARGUMENT, "null plan");
  if (!in || !out) return fail(B2F_ERR_INVALID_ARGUMENT, "null buffer");
  const Plan& plan = *handle->plan;
  if (plan.device < 0) return fail(B2F_ERR_DEVICE, "plan was created for planning only (no device)");
  const Config& c = plan.cfg;
  const size_t cb = complex_bytes(plan.prec), rb = cb / 2;
  uint64_t logical = 1, packed = 1;
  for (size_t d = 0; d < c.shape.size(); ++d) {
    logical *= c.shape[d];
    packed *= d == 0 ? c.shape[0] / 2 + 1 : c.shape[d];
  }
  uint64_t in_n = logical, out_n = logical;
  size_t in_e = cb, out_e = cb;
  if (plan.kind == B2F_R2C) {
    in_e = rb;
    out_n = packed;
  } else if (plan.kind == B2F_C2R) {
    in_n = packed;
    out_e = rb;
  }
  ViewShape vi, vo;
  b2f_status s = bind_view(in_layout, in_n, c.batch, in_e, in_bytes, "input", &vi);
  if (s) return s;
  s = bind_view(out_layout, out_n, c.batch, out_e, out_bytes, "output", &vo);
  if (s) return s;
  cudaStream_t st = (cudaStream_t)stream;
  const char* src = (const char*)in + vi.offset * in_e;
  char* dst = (char*)out + vo.offset * out_e;
  if (vi.contiguous() && vo.contiguous())
    return execute_plan(plan, st, src, plan.in_bytes, dst, plan.out_bytes);
  // strided: stage the input and/or the output in plan-owned buffers
  if (!vi.contiguous() && (s = staging(plan, &plan.view_in, plan.in_bytes))) return s;
  if (!vo.contiguous() && (s = staging(plan, &plan.view_out, plan.out_bytes))) return s;
  return run_ordered(plan, st, [&]() -> b2f_status {
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != plan.device) cudaSetDevice(plan.device);
    const void* xin = src;
    cudaError_t e = cudaSuccess;
    if (!vi.contiguous()) {
      e = view_copy(true, plan.view_in, in, vi, st);
      xin = plan.view_in;
    }
    // one side is a staging buffer, so input and output never alias here
    void* xout = vo.contiguous() ? (void*)dst : plan.view_out;
    b2f_status r = B2F_OK;
    if (e == cudaSuccess) r = run_passes_unordered(plan, st, xin, xout);
    if (e == cudaSuccess && r == B2F_OK && !vo.contiguous())
      e = view_copy(false, out, plan.view_out, vo, st);
    if (prev >= 0 && prev != plan.device) cudaSetDevice(prev);
    if (e != cudaSuccess)
      return fail(B2F_ERR_DEVICE, std::string("logical-view copy failed: ") + cudaGetErrorString(e));
    return r;
  });
}
