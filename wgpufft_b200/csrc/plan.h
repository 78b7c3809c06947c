// Host-side plan objects of the C ABI: configuration, tuning, route
// selection and the pass list a plan executes.
#pragma once
#include <cstdint>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/wgpufft_b200.h"
#include "kernels.h"

namespace b2f {

// FftTuning (src/tuning.rs:35-80): the crate's knobs, plus the B200 launch
// knobs (0 = planner's choice).  Knobs that only exist to work around
// WebGPU binding limits are accepted, validated and reported but change
// nothing here (no binding limits exist on the CUDA side).
struct Tuning {
  int64_t workgroup_size = 64;
  int64_t fused_workgroup_size = 256;
  int64_t rader_max_prime = 8192;
  int64_t direct_max_prime = 127;
  std::vector<uint32_t> force_rader_axes;
  std::vector<uint32_t> force_bluestein_axes;
  int64_t large_route = 0;
  int64_t large_chunk_max_batches = 0;
  int64_t grouped_batch = 0;
  int64_t swap_to_2_stage_4_step = 0;
  int64_t swap_to_3_stage_4_step = 0;
  int64_t segmented_burst_depth = 2;
  int64_t max_storage_buffer_binding_size = 0;
  int64_t max_buffer_size = 0;
  int64_t fused_min_convolution_length = 128;
  int64_t fuse_long_axes = 1;
  int64_t fuse_small_volumes = 1;
  int64_t lines_per_block = 0;
  int64_t threads_per_block = 0;
  int64_t twiddle_table = 1;
  int64_t tensor_cores = 0;  // 1: length-64 f32 lines on the tcgen05 split-TF32 DFT layer
  int64_t radix_order = 0;   // stage order of the shared-memory engine: 0 = planner's (radix 16
                             // first, small odd radices last), 1 = reversed
  int64_t tma_tiles = 0;     // 1: f32 column-tile passes of <= 256 points staged by TMA
};

struct Config {
  std::vector<uint64_t> shape;
  std::vector<uint32_t> axes;
  uint64_t batch = 1;
  int32_t direction = B2F_FORWARD;
  int32_t normalization = B2F_NORM_INVERSE;
  int32_t precision = B2F_F32;
  Tuning tuning;
};

enum class AxisKind { Mixed, Rader, Bluestein };
enum class Route { DirectDft, MixedRadix, Rader, Bluestein, AxisSequence };

// Buffers a pass reads or writes.
enum BufId : int {
  BUF_IN = 0, BUF_OUT = 1, BUF_WS0 = 2, BUF_WS1 = 3, BUF_WS2 = 4, BUF_WS3 = 5, BUF_WS4 = 6, BUF_WS5 = 7
};
constexpr int kNumWorkspaces = 6;

struct Pass {
  enum Kind { LINES, POW2, RADER, BLUESTEIN, R2C, C2R, SCALE_COPY, BLUE_ELEM, REAL_ELEM, TC_DFT64,
              SMALL_VOLUME } kind = LINES;
  int pow2_E = 16;         // POW2: values per thread
  bool colmajor = false;   // POW2: adjacent lines first
  std::string label;  // stage label (diagnostics)
  std::string route;  // axis route of the stage
  int axis = -1;
  int src = BUF_IN, dst = BUF_OUT;
  unsigned grid = 0, threads = 0;
  size_t smem = 0;
  std::vector<uint32_t> radices;
  LinesParams lines{};
  RaderParams rader{};
  BluesteinParams blue{};
  RealParams real{};
  BlueElemParams belem{};
  RealElemParams relem{};
  SmallVolumeParams svol{};
  uint64_t copy_n = 0;
  double copy_scale = 1.0;
  bool copy_conj = false;
  // TC_DFT64: lines, their scale and direction, device_allocs indices of the
  // operand table and of the wait-timeout flag
  uint64_t tc_nlines = 0;
  float tc_scale = 1.0f;
  bool tc_inverse = false;
  size_t tc_table = 0, tc_err = 0;
  // R2C / C2R on the fixed-length register kernels (even N0, h = N0/2 a
  // power of two)
  bool real_fx = false;
  // POW2 column tiles staged by TMA (tmatile.cu): persistent grid, the
  // device_allocs index of the wait-timeout flag
  bool tma = false;
  unsigned tma_grid = 0;
  size_t tma_err = 0;
};

struct Plan {
  Config cfg;
  int32_t kind = B2F_C2C;
  Route route = Route::MixedRadix;
  Prec prec = PREC_F32;
  int device = 0;
  std::vector<AxisKind> axis_kinds;
  std::vector<std::vector<uint32_t>> axis_factors;  // crate-style factorisation per axis
  std::vector<uint64_t> packed_shape;
  std::vector<Pass> passes;
  std::vector<void*> device_allocs;
  uint64_t table_bytes = 0;
  void* ws[kNumWorkspaces] = {};
  uint64_t ws_bytes[kNumWorkspaces] = {};
  uint64_t workspace_total() const {
    uint64_t t = 0;
    for (auto b : ws_bytes) t += b;
    return t;
  }
  uint64_t in_bytes = 0, out_bytes = 0;
  bool in_place_kernels = true;  // false: in place copies the input first
  mutable std::mutex copy_mu;
  mutable void* inplace_copy = nullptr;
  // Executions of a plan with device state shared between them (workspace,
  // in-place copy buffer, tensor-core error flag) are ordered on the device:
  // each one waits for the previous one's completion event and records its
  // own (exec_mu makes the wait/record pair atomic across host threads).
  bool shared_state = false;
  mutable std::mutex exec_mu;
  mutable cudaEvent_t last_done = nullptr;
  mutable bool last_done_recorded = false;
  // staging buffers of executions through strided logical views (created
  // on first use under copy_mu, kept until the plan is freed)
  mutable void* view_in = nullptr;
  mutable void* view_out = nullptr;
  std::string diag_json;
  ~Plan();
};

b2f_status validate_config(const Config& cfg);
// Tensor-core DFT layer (tc_dft.cu): the split operand table and the launcher.
std::vector<float> dft64_tc_table();
cudaError_t launch_dft64_tc(const void* in, void* out, const float* table, uint64_t nlines,
                            float scale, bool inverse, unsigned int* err, unsigned grid,
                            cudaStream_t st);
// device -2 plans on the host only (no device memory is touched); its
// shared-memory budget is smem_budget when non-zero, else 232448 bytes.
b2f_status create_plan(const Config& cfg, int32_t kind, int device, Plan** out,
                       size_t smem_budget = 0);
b2f_status execute_plan(const Plan& plan, cudaStream_t st, const void* in, uint64_t in_bytes,
                        void* out, uint64_t out_bytes);
b2f_status execute_plan_in_place(const Plan& plan, cudaStream_t st, void* buf, uint64_t bytes);
// f() ordered after the plan's previous execution and before its next (the
// plan's completion event), whatever the plan's route.
b2f_status run_ordered(const Plan& plan, cudaStream_t st, const std::function<b2f_status()>& f);
// The plan's passes from in to out (sizes already checked), not ordered.
b2f_status run_passes_unordered(const Plan& plan, cudaStream_t st, const void* in, void* out);

// Thread-local error detail.
b2f_status fail(b2f_status code, const std::string& msg);
const std::string& last_error();

// Integer helpers shared with the tests through the C ABI diagnostics.
bool is_prime_u64(uint64_t n);
uint64_t primitive_root(uint64_t p);
bool is_smooth13(uint64_t n);
std::vector<uint32_t> factor_supported_length(uint64_t n);  // empty if unsupported
std::vector<uint32_t> stage_radices(uint64_t n);             // kernel schedule
AxisKind axis_kind_for(const Config& cfg, uint32_t axis);
Route select_route(const Config& cfg);
const char* route_name(Route r);
const char* axis_kind_name(AxisKind k);

}  // namespace b2f

// Opaque handles of the C ABI (shared by the translation units that use them).
struct b2f_config {
  b2f::Config cfg;
};
struct b2f_plan {
  b2f::Plan* plan;
};
