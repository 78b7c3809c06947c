// extern "C" entry points of include/wgpufft_b200.h.
#include <cstring>
#include <string>

#include "plan.h"

using namespace b2f;

struct b2f_recorder {
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool capturing = false;
  b2f_status first_error = B2F_OK;
};

#define REQUIRE(cond, msg) \
  do {                     \
    if (!(cond)) return fail(B2F_ERR_INVALID_ARGUMENT, msg); \
  } while (0)

extern "C" {

b2f_status b2f_config_new(b2f_config** out, const uint64_t* shape, uint32_t rank) {
  REQUIRE(out, "null output handle");
  *out = nullptr;
  REQUIRE(shape || rank == 0, "null shape");
  auto* c = new b2f_config();
  c->cfg.shape.assign(shape, shape + rank);
  for (uint32_t i = 0; i < rank; ++i) c->cfg.axes.push_back(i);
  *out = c;
  return B2F_OK;
}

void b2f_config_free(b2f_config* cfg) { delete cfg; }

b2f_status b2f_config_set_axes(b2f_config* cfg, const uint32_t* axes, uint32_t count) {
  REQUIRE(cfg, "null config");
  REQUIRE(axes || count == 0, "null axes");
  cfg->cfg.axes.assign(axes, axes + count);
  return B2F_OK;
}

b2f_status b2f_config_set_batch(b2f_config* cfg, uint64_t batch) {
  REQUIRE(cfg, "null config");
  cfg->cfg.batch = batch;
  return B2F_OK;
}

b2f_status b2f_config_set_direction(b2f_config* cfg, int32_t direction) {
  REQUIRE(cfg, "null config");
  REQUIRE(direction == B2F_FORWARD || direction == B2F_INVERSE, "direction must be 0 or 1");
  cfg->cfg.direction = direction;
  return B2F_OK;
}

b2f_status b2f_config_set_normalization(b2f_config* cfg, int32_t normalization) {
  REQUIRE(cfg, "null config");
  REQUIRE(normalization >= 0 && normalization <= 3, "normalization must be 0..=3");
  cfg->cfg.normalization = normalization;
  return B2F_OK;
}

b2f_status b2f_config_set_precision(b2f_config* cfg, int32_t precision) {
  REQUIRE(cfg, "null config");
  REQUIRE(precision >= 0 && precision <= 2, "precision must be 0..=2");
  cfg->cfg.precision = precision;
  return B2F_OK;
}

static int64_t* tuning_field(Tuning& t, const std::string& k) {
  if (k == "workgroup_size") return &t.workgroup_size;
  if (k == "fused_workgroup_size") return &t.fused_workgroup_size;
  if (k == "rader_max_prime") return &t.rader_max_prime;
  if (k == "direct_max_prime") return &t.direct_max_prime;
  if (k == "large_route") return &t.large_route;
  if (k == "large_chunk_max_batches") return &t.large_chunk_max_batches;
  if (k == "grouped_batch") return &t.grouped_batch;
  if (k == "swap_to_2_stage_4_step") return &t.swap_to_2_stage_4_step;
  if (k == "swap_to_3_stage_4_step") return &t.swap_to_3_stage_4_step;
  if (k == "segmented_burst_depth") return &t.segmented_burst_depth;
  if (k == "max_storage_buffer_binding_size") return &t.max_storage_buffer_binding_size;
  if (k == "max_buffer_size") return &t.max_buffer_size;
  if (k == "fused_min_convolution_length") return &t.fused_min_convolution_length;
  if (k == "fuse_long_axes") return &t.fuse_long_axes;
  if (k == "fuse_small_volumes") return &t.fuse_small_volumes;
  if (k == "lines_per_block") return &t.lines_per_block;
  if (k == "threads_per_block") return &t.threads_per_block;
  if (k == "twiddle_table") return &t.twiddle_table;
  if (k == "tensor_cores") return &t.tensor_cores;
  if (k == "radix_order") return &t.radix_order;
  if (k == "tma_tiles") return &t.tma_tiles;
  return nullptr;
}

b2f_status b2f_config_set_tuning(b2f_config* cfg, const char* key, int64_t value) {
  REQUIRE(cfg && key, "null config or key");
  int64_t* f = tuning_field(cfg->cfg.tuning, key);
  if (!f) return fail(B2F_ERR_INVALID_ARGUMENT, std::string("unknown tuning key: ") + key);
  *f = value;
  return B2F_OK;
}

b2f_status b2f_config_get_tuning(const b2f_config* cfg, const char* key, int64_t* value) {
  REQUIRE(cfg && key && value, "null config, key or output");
  int64_t* f = tuning_field(const_cast<b2f_config*>(cfg)->cfg.tuning, key);
  if (!f) return fail(B2F_ERR_INVALID_ARGUMENT, std::string("unknown tuning key: ") + key);
  *value = *f;
  return B2F_OK;
}

b2f_status b2f_config_set_tuning_axes(b2f_config* cfg, const char* key, const uint32_t* axes,
                                      uint32_t count) {
  REQUIRE(cfg && key, "null config or key");
  REQUIRE(axes || count == 0, "null axes");
  const std::string k(key);
  if (k == "force_rader_axes") cfg->cfg.tuning.force_rader_axes.assign(axes, axes + count);
  else if (k == "force_bluestein_axes") cfg->cfg.tuning.force_bluestein_axes.assign(axes, axes + count);
  else return fail(B2F_ERR_INVALID_ARGUMENT, "unknown tuning axes key: " + k);
  return B2F_OK;
}

b2f_status b2f_config_validate(const b2f_config* cfg) {
  REQUIRE(cfg, "null config");
  return validate_config(cfg->cfg);
}

b2f_status b2f_config_required_buffer_size_bytes(const b2f_config* cfg, uint64_t* out) {
  REQUIRE(cfg && out, "null argument");
  b2f_status st = validate_config(cfg->cfg);
  if (st) return st;
  uint64_t total = cfg->cfg.batch;
  for (auto s : cfg->cfg.shape) total *= s;
  *out = total * (cfg->cfg.precision == B2F_F32 ? 8 : 16);
  return B2F_OK;
}

b2f_status b2f_config_scale(const b2f_config* cfg, float* out_f32, double* out_f64) {
  REQUIRE(cfg, "null config");
  b2f_status st = validate_config(cfg->cfg);
  if (st) return st;
  uint64_t logical = 1;
  for (auto s : cfg->cfg.shape) logical *= s;
  const bool inv = cfg->cfg.direction == B2F_INVERSE;
  const float lf = (float)logical;
  const double ld = (double)logical;
  float f = 1.0f;
  double d = 1.0;
  switch (cfg->cfg.normalization) {
    case B2F_NORM_FORWARD: f = inv ? 1.0f : 1.0f / lf; d = inv ? 1.0 : 1.0 / ld; break;
    case B2F_NORM_INVERSE: f = inv ? 1.0f / lf : 1.0f; d = inv ? 1.0 / ld : 1.0; break;
    case B2F_NORM_ORTHOGONAL: f = 1.0f / sqrtf(lf); d = 1.0 / sqrt(ld); break;
    default: break;
  }
  if (out_f32) *out_f32 = f;
  if (out_f64) *out_f64 = d;
  return B2F_OK;
}

static b2f_status make_plan(b2f_plan** out, const b2f_config* cfg, int32_t device, int32_t kind) {
  REQUIRE(out, "null output handle");
  *out = nullptr;
  REQUIRE(cfg, "null config");
  Plan* p = nullptr;
  b2f_status st = create_plan(cfg->cfg, kind, device, &p);
  if (st) return st;
  *out = new b2f_plan{p};
  return B2F_OK;
}

b2f_status b2f_plan_c2c(b2f_plan** out, const b2f_config* cfg, int32_t device) {
  return make_plan(out, cfg, device, B2F_C2C);
}
b2f_status b2f_plan_r2c(b2f_plan** out, const b2f_config* cfg, int32_t device) {
  return make_plan(out, cfg, device, B2F_R2C);
}
b2f_status b2f_plan_c2r(b2f_plan** out, const b2f_config* cfg, int32_t device) {
  return make_plan(out, cfg, device, B2F_C2R);
}

void b2f_plan_free(b2f_plan* plan) {
  if (!plan) return;
  delete plan->plan;
  delete plan;
}

int32_t b2f_plan_kind(const b2f_plan* plan) { return plan ? plan->plan->kind : -1; }

uint64_t b2f_plan_required_buffer_size_bytes(const b2f_plan* plan) {
  if (!plan) return 0;
  return std::max(plan->plan->in_bytes, plan->plan->out_bytes);
}
uint64_t b2f_plan_required_input_buffer_size_bytes(const b2f_plan* plan) {
  return plan ? plan->plan->in_bytes : 0;
}
uint64_t b2f_plan_required_output_buffer_size_bytes(const b2f_plan* plan) {
  return plan ? plan->plan->out_bytes : 0;
}
uint64_t b2f_plan_workspace_size_bytes(const b2f_plan* plan) {
  return plan ? plan->plan->workspace_total() : 0;
}
int32_t b2f_plan_supports_in_place(const b2f_plan* plan) {
  return plan ? (plan->plan->in_place_kernels ? 1 : 0) : 0;
}

b2f_status b2f_plan_execute_checked(const b2f_plan* plan, void* stream, const void* in,
                                    uint64_t in_bytes, void* out, uint64_t out_bytes) {
  REQUIRE(plan, "null plan");
  return execute_plan(*plan->plan, (cudaStream_t)stream, in, in_bytes, out, out_bytes);
}

b2f_status b2f_plan_execute_in_place(const b2f_plan* plan, void* stream, void* buffer,
                                     uint64_t bytes) {
  REQUIRE(plan, "null plan");
  return execute_plan_in_place(*plan->plan, (cudaStream_t)stream, buffer, bytes);
}

b2f_status b2f_plan_device_status(const b2f_plan* plan) {
  REQUIRE(plan, "null plan");
  const Plan& p = *plan->plan;
  if (p.device < 0) return B2F_OK;
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != p.device) cudaSetDevice(p.device);
  uint32_t flags = 0;
  cudaError_t e = cudaSuccess;
  for (const Pass& ps : p.passes) {
    if (ps.kind != Pass::TC_DFT64 && !ps.tma) continue;
    uint32_t v = 0;
    void* d = p.device_allocs[ps.kind == Pass::TC_DFT64 ? ps.tc_err : ps.tma_err];
    e = cudaMemcpy(&v, d, sizeof(v), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && v) e = cudaMemset(d, 0, sizeof(v));
    if (e != cudaSuccess) break;
    flags |= v;
  }
  if (prev >= 0 && prev != p.device) cudaSetDevice(prev);
  if (e != cudaSuccess) return fail(B2F_ERR_DEVICE, std::string("device status read failed: ") + cudaGetErrorString(e));
  if (flags & 4)
    return fail(B2F_ERR_DEVICE, "TMA column tiles: a bounded wait for a tile copy timed out");
  if (flags)
    return fail(B2F_ERR_DEVICE, std::string("tensor-core layer: a bounded wait for its matrix products timed out") +
                                    ((flags & 2) ? " (tensor memory freed with a product still pending)" : ""));
  return B2F_OK;
}

b2f_status b2f_plan_diagnostics_json(const b2f_plan* plan, char* buf, uint64_t* len) {
  REQUIRE(plan && len, "null argument");
  const std::string& j = plan->plan->diag_json;
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

b2f_status b2f_recorder_begin(b2f_recorder** out, void* stream) {
  REQUIRE(out, "null output handle");
  *out = nullptr;
  auto* r = new b2f_recorder();
  if (cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete r;
    return fail(B2F_ERR_DEVICE, "recorder stream creation failed");
  }
  (void)stream;  // the graph is ordered by the stream it is submitted on
  if (cudaStreamBeginCapture(r->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
    cudaStreamDestroy(r->stream);
    delete r;
    return fail(B2F_ERR_DEVICE, "stream capture could not start");
  }
  r->capturing = true;
  *out = r;
  return B2F_OK;
}

b2f_status b2f_plan_record(const b2f_plan* plan, b2f_recorder* rec, const void* in,
                           uint64_t in_bytes, void* out, uint64_t out_bytes) {
  REQUIRE(plan && rec, "null argument");
  REQUIRE(rec->capturing, "recorder is not capturing");
  b2f_status st = execute_plan(*plan->plan, rec->stream, in, in_bytes, out, out_bytes);
  if (st && !rec->first_error) rec->first_error = st;
  return st;
}

b2f_status b2f_plan_record_in_place(const b2f_plan* plan, b2f_recorder* rec, void* buffer,
                                    uint64_t bytes) {
  REQUIRE(plan && rec, "null argument");
  REQUIRE(rec->capturing, "recorder is not capturing");
  b2f_status st = execute_plan_in_place(*plan->plan, rec->stream, buffer, bytes);
  if (st && !rec->first_error) rec->first_error = st;
  return st;
}

b2f_status b2f_recorder_finish(b2f_recorder* rec) {
  REQUIRE(rec, "null recorder");
  REQUIRE(rec->capturing, "recorder is not capturing");
  rec->capturing = false;
  if (cudaStreamEndCapture(rec->stream, &rec->graph) != cudaSuccess || !rec->graph)
    return fail(B2F_ERR_DEVICE, "stream capture failed");
  if (rec->first_error) return fail(rec->first_error, "a recorded plan failed: " + last_error());
  if (cudaGraphInstantiate(&rec->exec, rec->graph, 0) != cudaSuccess)
    return fail(B2F_ERR_DEVICE, "graph instantiation failed");
  return B2F_OK;
}

b2f_status b2f_recorder_submit(b2f_recorder* rec, void* stream) {
  REQUIRE(rec, "null recorder");
  REQUIRE(rec->exec, "recorder has no finished graph");
  if (cudaGraphLaunch(rec->exec, (cudaStream_t)stream) != cudaSuccess)
    return fail(B2F_ERR_DEVICE, "graph launch failed");
  return B2F_OK;
}

void b2f_recorder_free(b2f_recorder* rec) {
  if (!rec) return;
  if (rec->capturing) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(rec->stream, &g);
    if (g) cudaGraphDestroy(g);
  }
  if (rec->exec) cudaGraphExecDestroy(rec->exec);
  if (rec->graph) cudaGraphDestroy(rec->graph);
  if (rec->stream) cudaStreamDestroy(rec->stream);
  delete rec;
}

const char* b2f_status_string(b2f_status s) {
  switch (s) {
    case B2F_OK: return "Ok";
    case B2F_ERR_ZERO_LENGTH: return "ZeroLength";
    case B2F_ERR_ZERO_BATCH: return "ZeroBatch";
    case B2F_ERR_LENGTH_TOO_LARGE: return "LengthTooLarge";
    case B2F_ERR_UNSUPPORTED_LENGTH: return "UnsupportedLength";
    case B2F_ERR_PRECISION_UNSUPPORTED: return "PrecisionUnsupported";
    case B2F_ERR_INVALID_TUNING: return "InvalidTuning";
    case B2F_ERR_EMPTY_AXES: return "EmptyAxes";
    case B2F_ERR_INVALID_AXIS: return "InvalidAxis";
    case B2F_ERR_DUPLICATE_AXIS: return "DuplicateAxis";
    case B2F_ERR_INVALID_REAL_DIRECTION: return "InvalidRealTransformDirection";
    case B2F_ERR_UNSUPPORTED_REAL_AXES: return "UnsupportedRealAxes";
    case B2F_ERR_BUFFER_TOO_SMALL: return "BufferViewTooSmall";
    case B2F_ERR_IN_PLACE_UNSUPPORTED: return "InPlaceUnsupported";
    case B2F_ERR_RESOURCE_ALLOCATION: return "GpuPlanResourceAllocationFailed";
    case B2F_ERR_INVALID_ARGUMENT: return "InvalidArgument";
    case B2F_ERR_DEVICE: return "DeviceError";
    case B2F_ERR_WORKSPACE_TOO_SMALL: return "WorkspaceTooSmall";
    case B2F_ERR_SNAPSHOT_JSON: return "SnapshotJson";
    case B2F_ERR_SNAPSHOT_SCHEMA: return "SnapshotSchemaMismatch";
    case B2F_ERR_SNAPSHOT_VERSION: return "SnapshotVersionMismatch";
    case B2F_ERR_SNAPSHOT_INTEGRITY: return "SnapshotIntegrity";
    case B2F_ERR_LAYOUT_ZERO_STRIDE: return "BufferLayoutZeroStride";
    case B2F_ERR_LAYOUT_BATCH_STRIDE_TOO_SMALL: return "BufferLayoutBatchStrideTooSmall";
    case B2F_ERR_LAYOUT_OUT_OF_BOUNDS: return "BufferLayoutOutOfBounds";
    case B2F_ERR_LAYOUT_TOO_LARGE: return "BufferLayoutTooLarge";
    default: return "Unknown";
  }
}

uint64_t b2f_last_error_message(char* buf, uint64_t len) {
  const std::string& e = last_error();
  if (buf && len > 0) {
    const uint64_t n = std::min<uint64_t>(len - 1, e.size());
    std::memcpy(buf, e.data(), n);
    buf[n] = 0;
  }
  return e.size();
}

const char* b2f_version(void) { return "wgpufft_b200 0.1.0 (sm_100a)"; }

}  // extern "C"
