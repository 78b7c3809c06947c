// Planner and executor of the C ABI.
//
// Plan creation mirrors the crate's planner (src/runtime/c2c.rs:921-1275,
// src/runtime/axis_plan.rs:516-1144, src/runtime/real.rs:721-1340): validate
// the configuration, classify each axis (mixed radix, Rader, Bluestein),
// select the route, then turn every axis into passes over the buffers.  The
// pass ladder is B200-shaped rather than the crate's WebGPU ladder:
//   - a line that fits one CTA's shared memory runs in one pass (one HBM
//     read and one write) whatever its smooth length;
//   - a longer smooth line runs as a four-step pair of passes, the first
//     applying the W_N^{n2 k1} twiddle on store;
//   - a prime whose p-1 is 13-smooth runs Rader's convolution in one pass;
//     other lengths run Bluestein's chirp convolution in one pass;
//   - real transforms pack/unpack inside the axis-0 pass.
// All stage twiddles and convolution spectra are built once, in FP64 on the
// host, and rounded once to the working precision.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
#include <sstream>

#include "hostfft.h"
#include "plan.h"

namespace b2f {

// ---------------------------------------------------------------- errors
static thread_local std::string t_last_error;

b2f_status fail(b2f_status code, const std::string& msg) {
  t_last_error = msg;
  return code;
}
const std::string& last_error() { return t_last_error; }

// ------------------------------------------------------------- integers
bool is_prime_u64(uint64_t n) {
  if (n < 2) return false;
  if (n % 2 == 0) return n == 2;
  for (uint64_t d = 3; d <= n / d; d += 2)
    if (n % d == 0) return false;
  return true;
}

static uint64_t mod_pow(uint64_t b, uint64_t e, uint64_t m) {
  uint64_t r = 1;
  b %= m;
  while (e) {
    if (e & 1) r = (unsigned __int128)r * b % m;
    b = (unsigned __int128)b * b % m;
    e >>= 1;
  }
  return r;
}

// Smallest primitive root (src/runtime/axis_policy.rs:134-152).
uint64_t primitive_root(uint64_t p) {
  if (!is_prime_u64(p)) return 0;
  if (p == 2) return 1;
  const uint64_t phi = p - 1;
  std::vector<uint64_t> f;
  uint64_t n = phi;
  for (uint64_t d = 2; d <= n / d; d += (d == 2 ? 1 : 2))
    if (n % d == 0) {
      f.push_back(d);
      while (n % d == 0) n /= d;
    }
  if (n > 1) f.push_back(n);
  for (uint64_t g = 2; g < p; ++g) {
    bool ok = true;
    for (uint64_t q : f)
      if (mod_pow(g, phi / q, p) == 1) {
        ok = false;
        break;
      }
    if (ok) return g;
  }
  return 0;
}

bool is_smooth13(uint64_t n) {
  if (n == 0) return false;
  for (uint64_t r : {2, 3, 5, 7, 11, 13})
    while (n % r == 0) n /= r;
  return n == 1;
}

static bool is_smooth7(uint64_t n) {
  if (n == 0) return false;
  for (uint64_t r : {2, 3, 5, 7})
    while (n % r == 0) n /= r;
  return n == 1;
}

// factor_supported_length (src/runtime/mod.rs:34-57): greedy over
// 13, 11, 8, 7, 5, 4, 3, 2.
std::vector<uint32_t> factor_supported_length(uint64_t n) {
  static const uint32_t order[] = {13, 11, 8, 7, 5, 4, 3, 2};
  std::vector<uint32_t> f;
  if (n == 0) return f;
  while (n > 1) {
    bool found = false;
    for (uint32_t r : order)
      if (n % r == 0) {
        f.push_back(r);
        n /= r;
        found = true;
        break;
      }
    if (!found) return {};
  }
  return f;
}

// The kernel radix schedule: radix-16 stages for the power of two (then one
// 8, 4 or 2), 9 for pairs of threes, then the odd primes.
std::vector<uint32_t> stage_radices(uint64_t n) {
  std::vector<uint32_t> r;
  int e2 = 0;
  while (n % 2 == 0) {
    n /= 2;
    ++e2;
  }
  while (e2 >= 4) {
    r.push_back(16);
    e2 -= 4;
  }
  if (e2 == 3) r.push_back(8);
  if (e2 == 2) r.push_back(4);
  if (e2 == 1) r.push_back(2);
  for (uint32_t p : {13u, 11u, 7u, 5u}) {
    while (n % p == 0) {
      r.push_back(p);
      n /= p;
    }
  }
  int e3 = 0;
  while (n % 3 == 0) {
    n /= 3;
    ++e3;
  }
  while (e3 >= 2) {
    r.push_back(9);
    e3 -= 2;
  }
  if (e3 == 1) r.push_back(3);
  if (n != 1) return {};
  return r;
}

// axis_kind_for_len_with_rader_max (src/runtime/axis_policy.rs:72-80) with
// the forced-axis tuning of resolve_axis_kinds_for_axes_with_tuning (41-65).
AxisKind axis_kind_for(const Config& cfg, uint32_t axis) {
  const auto& t = cfg.tuning;
  if (std::find(t.force_rader_axes.begin(), t.force_rader_axes.end(), axis) != t.force_rader_axes.end())
    return AxisKind::Rader;
  if (std::find(t.force_bluestein_axes.begin(), t.force_bluestein_axes.end(), axis) !=
      t.force_bluestein_axes.end())
    return AxisKind::Bluestein;
  const uint64_t len = cfg.shape[axis];
  if (!factor_supported_length(len).empty() || len == 1) return AxisKind::Mixed;
  if (is_prime_u64(len) && (int64_t)len <= t.rader_max_prime) return AxisKind::Rader;
  return AxisKind::Bluestein;
}

// select_route (src/runtime/c2c.rs:7631-7650).
Route select_route(const Config& cfg) {
  uint64_t total = cfg.batch;
  for (auto s : cfg.shape) total *= s;
  if (total == 1) return Route::DirectDft;
  std::vector<AxisKind> k;
  for (auto a : cfg.axes) k.push_back(axis_kind_for(cfg, a));
  if (std::all_of(k.begin(), k.end(), [](AxisKind x) { return x == AxisKind::Mixed; }))
    return Route::MixedRadix;
  if (k.size() == 1 && k[0] == AxisKind::Rader) return Route::Rader;
  if (k.size() == 1 && k[0] == AxisKind::Bluestein) return Route::Bluestein;
  return Route::AxisSequence;
}

const char* route_name(Route r) {
  switch (r) {
    case Route::DirectDft: return "direct-dft";
    case Route::MixedRadix: return "mixed-radix";
    case Route::Rader: return "rader";
    case Route::Bluestein: return "bluestein";
    case Route::AxisSequence: return "axis-sequence";
  }
  return "?";
}

const char* axis_kind_name(AxisKind k) {
  switch (k) {
    case AxisKind::Mixed: return "mixed";
    case AxisKind::Rader: return "rader";
    case AxisKind::Bluestein: return "bluestein";
  }
  return "?";
}

// ------------------------------------------------------------ validation
static b2f_status invalid_tuning(const char* field, int64_t value, const char* kind,
                                 const char* reason) {
  std::ostringstream os;
  os << "InvalidTuning { kind: " << kind << ", field: " << field << ", value: " << value
     << ", reason: " << reason << " }";
  return fail(B2F_ERR_INVALID_TUNING, os.str());
}

static bool pow2(int64_t v) { return v > 0 && (v & (v - 1)) == 0; }

// FftTuning::validate_for_config (src/tuning.rs:280-355).
static b2f_status validate_tuning(const Config& cfg) {
  const Tuning& t = cfg.tuning;
  if (!pow2(t.workgroup_size))
    return invalid_tuning("workgroup_size", t.workgroup_size, "InvalidValue",
                          "must be a non-zero power of two");
  if (!pow2(t.fused_workgroup_size))
    return invalid_tuning("fused_workgroup_size", t.fused_workgroup_size, "InvalidValue",
                          "must be a non-zero power of two");
  if (t.rader_max_prime < 2)
    return invalid_tuning("rader_max_prime", t.rader_max_prime, "InvalidValue",
                          "must be at least 2");
  if (t.large_chunk_max_batches < 0)
    return invalid_tuning("large_chunk_max_batches", t.large_chunk_max_batches, "InvalidValue",
                          "must be greater than zero when provided");
  if (t.grouped_batch < 0)
    return invalid_tuning("grouped_batch", t.grouped_batch, "InvalidValue",
                          "must be greater than zero when provided");
  if (t.segmented_burst_depth < 1 || t.segmented_burst_depth > 3)
    return invalid_tuning("segmented_burst_depth", t.segmented_burst_depth, "InvalidValue",
                          "must be in the range 1..=3");
  if (t.max_storage_buffer_binding_size < 0)
    return invalid_tuning("max_storage_buffer_binding_size", t.max_storage_buffer_binding_size,
                          "InvalidValue", "must be greater than zero when provided");
  if (t.max_buffer_size < 0)
    return invalid_tuning("max_buffer_size", t.max_buffer_size, "InvalidValue",
                          "must be greater than zero when provided");
  if (t.swap_to_2_stage_4_step > 0 && t.swap_to_3_stage_4_step > 0 &&
      t.swap_to_2_stage_4_step > t.swap_to_3_stage_4_step)
    return invalid_tuning("swap_to_2_stage_4_step", t.swap_to_2_stage_4_step,
                          "ConflictingValues",
                          "must not exceed swap_to_3_stage_4_step when both thresholds are active");
  if (t.tensor_cores != 0 && t.tensor_cores != 1)
    return invalid_tuning("tensor_cores", t.tensor_cores, "InvalidValue", "must be 0 or 1");
  if (t.radix_order != 0 && t.radix_order != 1)
    return invalid_tuning("radix_order", t.radix_order, "InvalidValue", "must be 0 or 1");
  if (t.tma_tiles != 0 && t.tma_tiles != 1)
    return invalid_tuning("tma_tiles", t.tma_tiles, "InvalidValue", "must be 0 or 1");
  if (t.lines_per_block < 0)
    return invalid_tuning("lines_per_block", t.lines_per_block, "InvalidValue",
                          "must be zero (planner's choice) or positive");
  if (t.threads_per_block != 0 &&
      (!pow2(t.threads_per_block) || t.threads_per_block < 32 || t.threads_per_block > 512))
    return invalid_tuning("threads_per_block", t.threads_per_block, "DeviceLimit",
                          "must be zero or a power of two in 32..=512");
  for (auto a : t.force_rader_axes)
    if (std::find(t.force_bluestein_axes.begin(), t.force_bluestein_axes.end(), a) !=
        t.force_bluestein_axes.end())
      return invalid_tuning("force_rader_axes/force_bluestein_axes", a, "ConflictingAxes",
                            "the same axis cannot be forced to both Rader and Bluestein");
  for (int which = 0; which < 2; ++which) {
    const auto& axes = which == 0 ? t.force_rader_axes : t.force_bluestein_axes;
    const char* field = which == 0 ? "force_rader_axes" : "force_bluestein_axes";
    for (size_t i = 0; i < axes.size(); ++i) {
      const uint32_t a = axes[i];
      if (std::find(axes.begin(), axes.begin() + i, a) != axes.begin() + i)
        return invalid_tuning(field, a, "DuplicateAxis", "axis appears more than once");
      if (a >= cfg.shape.size())
        return invalid_tuning(field, a, "AxisOutOfRange",
                              "axis is outside the configured shape rank");
      if (std::find(cfg.axes.begin(), cfg.axes.end(), a) == cfg.axes.end())
        return invalid_tuning(field, a, "AxisNotSelected",
                              "axis is not present in FftConfig::axes");
      const uint64_t len = cfg.shape[a];
      if (which == 0 && (len < 3 || !is_prime_u64(len)))
        return invalid_tuning(field, a, "AxisAlgorithmIncompatible",
                              "forced Rader axes must have prime length at least 3");
      if (which == 1 && len < 2)
        return invalid_tuning(field, a, "AxisAlgorithmIncompatible",
                              "forced Bluestein axes must have length at least 2");
    }
  }
  return B2F_OK;
}

static bool total_len(const Config& cfg, uint64_t* out) {
  unsigned __int128 t = cfg.batch;
  for (auto s : cfg.shape) {
    t *= s;
    if (t > 0xFFFFFFFFull) {
      *out = 0;
      return false;
    }
  }
  *out = (uint64_t)t;
  return true;
}

// FftConfig::validate (src/config.rs:178-211).
b2f_status validate_config(const Config& cfg) {
  if (cfg.shape.empty() || std::find(cfg.shape.begin(), cfg.shape.end(), 0) != cfg.shape.end())
    return fail(B2F_ERR_ZERO_LENGTH, "ZeroLength: shape is empty or has a zero extent");
  if (cfg.batch == 0) return fail(B2F_ERR_ZERO_BATCH, "ZeroBatch");
  if (cfg.axes.empty()) return fail(B2F_ERR_EMPTY_AXES, "EmptyAxes");
  uint64_t total = 0;
  const bool fits = total_len(cfg, &total);
  std::vector<bool> seen(cfg.shape.size(), false);
  for (auto a : cfg.axes) {
    if (a >= cfg.shape.size())
      return fail(B2F_ERR_INVALID_AXIS, "InvalidAxis { axis: " + std::to_string(a) +
                                            ", rank: " + std::to_string(cfg.shape.size()) + " }");
    if (seen[a]) return fail(B2F_ERR_DUPLICATE_AXIS, "DuplicateAxis { axis: " + std::to_string(a) + " }");
    seen[a] = true;
    if (cfg.shape[a] == 1 && !(fits && total == 1))
      return fail(B2F_ERR_UNSUPPORTED_LENGTH, "UnsupportedLength { len: 1 }");
  }
  if (!fits) return fail(B2F_ERR_LENGTH_TOO_LARGE, "LengthTooLarge: total complex length exceeds u32::MAX");
  if (cfg.direction != B2F_FORWARD && cfg.direction != B2F_INVERSE)
    return fail(B2F_ERR_INVALID_ARGUMENT, "direction must be 0 (forward) or 1 (inverse)");
  if (cfg.normalization < 0 || cfg.normalization > 3)
    return fail(B2F_ERR_INVALID_ARGUMENT, "normalization must be 0..=3");
  if (cfg.precision < 0 || cfg.precision > 2)
    return fail(B2F_ERR_INVALID_ARGUMENT, "precision must be 0 (f32), 1 (f64) or 2 (df64)");
  return validate_tuning(cfg);
}

// FftConfig::scale / scale_f64 (src/config.rs:262-286): f32 plans use the
// f32-computed factor, exactly as the reference.
static double plan_scale(const Config& cfg, uint64_t logical) {
  const bool inv = cfg.direction == B2F_INVERSE;
  if (cfg.precision == B2F_F32) {
    const float len = (float)logical;
    float s = 1.0f;
    switch (cfg.normalization) {
      case B2F_NORM_FORWARD: s = inv ? 1.0f : 1.0f / len; break;
      case B2F_NORM_INVERSE: s = inv ? 1.0f / len : 1.0f; break;
      case B2F_NORM_ORTHOGONAL: s = 1.0f / sqrtf(len); break;
      default: break;
    }
    return (double)s;
  }
  const double len = (double)logical;
  switch (cfg.normalization) {
    case B2F_NORM_FORWARD: return inv ? 1.0 : 1.0 / len;
    case B2F_NORM_INVERSE: return inv ? 1.0 / len : 1.0;
    case B2F_NORM_ORTHOGONAL: return 1.0 / std::sqrt(len);
    default: return 1.0;
  }
}

// ------------------------------------------------------------ planning
struct Builder {
  Plan& plan;
  bool dry;           // planning only: no device allocations
  size_t smem_budget; // bytes of dynamic shared memory per CTA
  std::vector<std::pair<size_t, std::vector<unsigned char>>> pending;  // (alloc index, bytes)

  size_t cb() const { return complex_bytes(plan.prec); }
  int pad_shift() const { return plan.prec == PREC_F32 ? 4 : 3; }
  uint32_t ld_for(uint64_t n) const { return (uint32_t)(n + (n >> pad_shift()) + 1); }

  // Records that workspace buffer `id` must hold at least `bytes`.
  void need(int id, uint64_t bytes) {
    if (id >= BUF_WS0) {
      uint64_t& w = plan.ws_bytes[id - BUF_WS0];
      w = std::max(w, bytes);
    }
  }

  // Registers a device table; returns its index in plan.device_allocs.
  size_t add_table(std::vector<unsigned char>&& bytes) {
    plan.table_bytes += bytes.size();
    plan.device_allocs.push_back(nullptr);
    pending.emplace_back(plan.device_allocs.size() - 1, std::move(bytes));
    return plan.device_allocs.size() - 1;
  }

  std::vector<unsigned char> pack_complex(const std::vector<cd>& v) const {
    std::vector<unsigned char> out;
    if (plan.prec == PREC_F32) {
      out.resize(v.size() * 8);
      float* f = (float*)out.data();
      for (size_t i = 0; i < v.size(); ++i) {
        f[2 * i] = (float)v[i].real();
        f[2 * i + 1] = (float)v[i].imag();
      }
    } else if (plan.prec == PREC_F64) {
      out.resize(v.size() * 16);
      double* d = (double*)out.data();
      for (size_t i = 0; i < v.size(); ++i) {
        d[2 * i] = v[i].real();
        d[2 * i + 1] = v[i].imag();
      }
    } else {
      out.resize(v.size() * 16);
      float* f = (float*)out.data();
      auto split = [](double x, float* w) {
        const float hi = (float)x;
        w[0] = hi;
        w[1] = std::isfinite(hi) ? (float)(x - (double)hi) : 0.0f;
      };
      for (size_t i = 0; i < v.size(); ++i) {
        split(v[i].real(), f + 4 * i);
        split(v[i].imag(), f + 4 * i + 2);
      }
    }
    return out;
  }

  // Stage schedule of length n plus its twiddle table (FP64, rounded once).
  bool make_schedule(uint64_t n, Schedule& sch, std::vector<uint32_t>& radices,
                     std::vector<cd>& tw) {
    radices = stage_radices(n);
    if (radices.empty() && n != 1) return false;
    if (plan.cfg.tuning.radix_order == 1) std::reverse(radices.begin(), radices.end());
    if (radices.size() > FFT_MAX_STAGES) return false;
    std::memset(&sch, 0, sizeof(sch));
    sch.N = (uint32_t)n;
    sch.nst = (uint32_t)radices.size();
    uint64_t Ns = 1;
    for (size_t s = 0; s < radices.size(); ++s) {
      const uint32_t R = radices[s];
      StageDesc& d = sch.st[s];
      d.R = R;
      d.Ns = (uint32_t)Ns;
      d.NR = (uint32_t)(n / R);
      d.tw_off = (uint32_t)tw.size();
      d.dNs = make_fastdiv((uint32_t)Ns);
      d.dNR = make_fastdiv((uint32_t)(n / R));
      std::vector<cd> rt;
      fill_roots(rt, Ns * R);
      for (uint64_t k = 0; k < Ns; ++k)
        for (uint32_t q = 1; q < R; ++q) tw.push_back(rt[(q * k) % (Ns * R)]);
      Ns *= R;
    }
    return true;
  }

  // Lines per CTA and threads for a pass whose FFT length is nfft and whose
  // per-line shared memory is line_bytes.
  bool choose_launch(uint64_t nfft, size_t line_bytes, uint64_t inner_n, bool column_tiles,
                     uint32_t* G_out, uint32_t* T_out) {
    const uint64_t gmax_smem = smem_budget / line_bytes;
    if (gmax_smem == 0) return false;
    const uint64_t target = plan.prec == PREC_F32 ? 4096 : 2048;
    uint64_t G = std::max<uint64_t>(1, target / nfft);
    if (column_tiles) G = std::max<uint64_t>(G, plan.prec == PREC_F32 ? 8 : 4);
    if (plan.cfg.tuning.lines_per_block > 0) G = (uint64_t)plan.cfg.tuning.lines_per_block;
    G = std::min<uint64_t>(G, inner_n);
    G = std::min<uint64_t>(G, gmax_smem);
    G = std::max<uint64_t>(G, 1);
    uint64_t T = (G * nfft + 15) / 16;
    T = (T + 31) / 32 * 32;
    T = std::min<uint64_t>(std::max<uint64_t>(T, 32), 512);
    if (plan.cfg.tuning.threads_per_block > 0) T = (uint64_t)plan.cfg.tuning.threads_per_block;
    *G_out = (uint32_t)G;
    *T_out = (uint32_t)T;
    return true;
  }

  bool fits_one_cta(uint64_t nbuf) const { return 2 * (size_t)ld_for(nbuf) * cb() <= smem_budget; }

  static void fill_io_grid(LinesParams& lp, Pass& ps, uint64_t outer_n) {
    lp.io.tiles = (lp.io.inner_n + lp.G - 1) / lp.G;
    lp.dN = make_fastdiv(lp.N);
    lp.dG = make_fastdiv(lp.G);
    if (lp.io.tw_div == 0) lp.io.tw_div = 1;
    lp.d_tw = make_fastdiv(lp.io.tw_div);
    ps.grid = (unsigned)(outer_n * lp.io.mid_n * lp.io.tiles);
  }

  // Table pointers are patched after upload, by pass index and field.
  enum Field { F_LINES_TW, F_RADER_TW, F_BLUE_TW, F_REAL_TW, F_PERM_IN, F_PERM_OUT, F_RADER_BHAT,
               F_BLUE_BHAT, F_BELEM_BHAT, F_TWS_A, F_TWS_B, F_SVOL_TW, F_BLUE_CHIRP,
               F_BELEM_CHIRP, F_REAL_RTW, F_BELEM_PIN, F_BELEM_POUT, F_BELEM_X0 };
  struct Patch {
    size_t table, pass;
    Field field;
  };
  std::vector<Patch> patches;
  // The index the pass being built will take when pushed.
  size_t next_pass() const { return plan.passes.size(); }
  void set_table(size_t pass, Field f, size_t table) { patches.push_back({table, pass, f}); }

  // Stage twiddle table of a pass (when enabled): returns true if added.
  bool tw_table_for(uint32_t& flags, std::vector<cd>& tw, Field f) {
    if (plan.cfg.tuning.twiddle_table && !tw.empty()) {
      flags |= PF_TW_TABLE;
      set_table(next_pass(), f, add_table(pack_complex(tw)));
      return true;
    }
    return false;
  }

  void apply_patches() {
    for (const Patch& pa : patches) {
      Pass& ps = plan.passes[pa.pass];
      const void* ptr = plan.device_allocs[pa.table];
      switch (pa.field) {
        case F_LINES_TW: ps.lines.tw = ptr; break;
        case F_RADER_TW: ps.rader.L.tw = ptr; break;
        case F_BLUE_TW: ps.blue.L.tw = ptr; break;
        case F_REAL_TW: ps.real.tw = ptr; break;
        case F_PERM_IN: ps.rader.perm_in = (const uint32_t*)ptr; break;
        case F_PERM_OUT: ps.rader.perm_out = (const uint32_t*)ptr; break;
        case F_RADER_BHAT: ps.rader.bhat = ptr; break;
        case F_BLUE_BHAT: ps.blue.bhat = ptr; break;
        case F_BELEM_BHAT: ps.belem.bhat = ptr; break;
        case F_TWS_A: ps.lines.tws_a = ptr; break;
        case F_TWS_B: ps.lines.tws_b = ptr; break;
        case F_SVOL_TW: ps.svol.tw = ptr; break;
        case F_BLUE_CHIRP: ps.blue.chirp = ptr; break;
        case F_BELEM_CHIRP: ps.belem.chirp = ptr; break;
        case F_REAL_RTW: ps.real.rtw = ptr; break;
        case F_BELEM_PIN: ps.belem.perm_in = (const uint32_t*)ptr; break;
        case F_BELEM_POUT: ps.belem.perm_out = (const uint32_t*)ptr; break;
        case F_BELEM_X0: ps.belem.x0 = const_cast<void*>(ptr); break;
      }
    }
  }
};

// Register-resident power-of-two pass when the line and its IO pattern
// allow it (see regfft.cuh); returns false to fall back to the general
// shared-memory engine.
static bool try_pow2_pass(Builder& b, Pass& ps, uint64_t outer_n) {
  LinesParams& lp = ps.lines;
  const uint64_t N = lp.N;
  const bool f32 = b.plan.prec == PREC_F32;
  if (N < 16 || (N & (N - 1)) || N > (f32 ? 8192u : 4096u)) return false;
  // the register kernel runs radix-16 stages then one smaller one: a
  // reordered schedule or explicit launch shapes go to the shared-memory engine
  if (b.plan.cfg.tuning.lines_per_block > 0 || b.plan.cfg.tuning.threads_per_block > 0 ||
      b.plan.cfg.tuning.radix_order != 0)
    return false;
  const LineIO& io = lp.io;
  bool colmajor;
  if (io.inner_n > 1 && io.in_inner == 1 && io.out_inner == 1) {
    colmajor = true;
  } else if (io.in_es == 1) {
    colmajor = false;
    if (io.out_es != 1) lp.flags |= PF_STORE_SMEM;
  } else {
    return false;
  }
  // f32 column tiles of 1024 points and more hold 32 values a thread (more
  // adjacent columns per tile, longer row segments); every other line holds
  // 16 (64 registers for f32: 4096- and 8192-point lines as 256 or 512
  // threads, twice the resident warps of 32 values at 128 registers)
  int E = 16;
  if (f32 && colmajor && N >= 1024) E = 32;
  // CTAs stay at 256 threads, so that two or more of them share an SM and
  // one's loads overlap another's butterflies; column tiles of 8192-point
  // lines keep 512 threads (two columns, 16-byte rows) rather than one
  // 8-byte column, and contiguous 8192-point f32 lines take 512 threads
  const uint32_t maxT = ((colmajor && N > 4096) || (!colmajor && f32 && N == 8192)) ? 512 : 256;
  const uint32_t TL = (uint32_t)(N / E);
  if (TL == 0 || TL > maxT) return false;
  const uint32_t LD = (uint32_t)(N + (N >> 4) + 1);
  const uint64_t gmax_smem = b.smem_budget / ((size_t)LD * b.cb());
  uint64_t G;
  if (colmajor) {
    G = maxT / TL;
    uint64_t cap = 1;
    while (cap < io.inner_n) cap <<= 1;
    G = std::min<uint64_t>(G, cap);
    while (G > 1 && G > gmax_smem) G >>= 1;
  } else {
    G = std::max<uint64_t>(1, 256 / TL);
    G = std::min<uint64_t>(G, io.inner_n);
    G = std::min<uint64_t>(G, gmax_smem);
  }
  if (G == 0 || G > gmax_smem) return false;
  lp.G = (uint32_t)G;
  lp.LD = LD;
  ps.kind = Pass::POW2;
  ps.pow2_E = E;
  ps.colmajor = colmajor;
  ps.threads = (unsigned)(G * TL);
  ps.smem = (size_t)G * LD * b.cb();
  (void)outer_n;
  return true;
}

// One complex axis in one pass (mixed radix, line fits a CTA).
static b2f_status add_lines_pass(Builder& b, int axis, uint64_t N, const LineIO& io,
                                 uint64_t outer_n, uint32_t flags, double scale, int src, int dst,
                                 const std::string& label, const char* route) {
  Pass ps;
  ps.kind = Pass::LINES;
  ps.axis = axis;
  ps.src = src;
  ps.dst = dst;
  ps.label = label;
  ps.route = route;
  LinesParams& lp = ps.lines;
  lp.N = (uint32_t)N;
  lp.io = io;
  lp.flags = flags;
  lp.scale = scale;
  std::vector<cd> tw;
  if (!b.make_schedule(N, lp.sch, ps.radices, tw))
    return fail(B2F_ERR_UNSUPPORTED_LENGTH, "UnsupportedLength { len: " + std::to_string(N) + " }");
  if (!try_pow2_pass(b, ps, outer_n)) {
    lp.LD = b.ld_for(N);
    const bool tiles = io.in_inner == 1 || io.out_inner == 1;
    if (!b.choose_launch(N, 2 * (size_t)lp.LD * b.cb(), io.inner_n, tiles && io.inner_n > 1,
                         &lp.G, &ps.threads))
      return fail(B2F_ERR_UNSUPPORTED_LENGTH,
                  "line of " + std::to_string(N) + " points does not fit a CTA");
    ps.smem = 2 * (size_t)lp.G * lp.LD * b.cb();
  }
  b.tw_table_for(lp.flags, tw, Builder::F_LINES_TW);
  Builder::fill_io_grid(lp, ps, outer_n);
  // f32 column tiles of <= 256 points: staged by TMA into a persistent grid
  // of as many CTAs as the SMs hold (needs a device to size the grid)
  if (ps.kind == Pass::POW2 && ps.colmajor && ps.pow2_E == 16 && b.plan.prec == PREC_F32 &&
      b.plan.cfg.tuning.tma_tiles && b.plan.device >= 0 && tma_tile_shape_ok(lp, outer_n)) {
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b.plan.device) == cudaSuccess) {
      const int per_sm = tma_tile_ctas_per_sm(lp, ps.threads);
      if (per_sm > 0 && nsm > 0) {
        ps.tma = true;
        ps.tma_grid = (unsigned)std::min<uint64_t>(ps.grid, (uint64_t)nsm * per_sm);
        ps.tma_err = b.add_table(std::vector<unsigned char>(16, 0));
      }
    }
    cudaGetLastError();
  }
  b.plan.passes.push_back(ps);
  return B2F_OK;
}

static b2f_status add_rader_pass(Builder& b, int axis, uint64_t p, const LineIO& io,
                                 uint64_t outer_n, uint32_t flags, double scale, int src, int dst) {
  Pass ps;
  ps.kind = Pass::RADER;
  ps.axis = axis;
  ps.src = src;
  ps.dst = dst;
  ps.label = "rader-fused-workgroup-stage";
  ps.route = "rader";
  RaderParams& rp = ps.rader;
  LinesParams& lp = rp.L;
  lp.N = (uint32_t)p;
  lp.io = io;
  lp.flags = flags;
  lp.scale = scale;
  std::vector<cd> tw;
  if (!b.make_schedule(p - 1, lp.sch, ps.radices, tw))
    return fail(B2F_ERR_UNSUPPORTED_LENGTH, "Rader convolution length is not smooth");
  lp.LD = b.ld_for(p);
  const bool tiles = io.in_inner == 1 || io.out_inner == 1;
  if (!b.choose_launch(p - 1, 2 * (size_t)lp.LD * b.cb() + 2 * b.cb(), io.inner_n,
                       tiles && io.inner_n > 1, &lp.G, &ps.threads))
    return fail(B2F_ERR_UNSUPPORTED_LENGTH, "Rader line does not fit a CTA");
  ps.smem = (2 * (size_t)lp.G * lp.LD + 2 * lp.G) * b.cb();
  b.tw_table_for(lp.flags, tw, Builder::F_RADER_TW);
  Builder::fill_io_grid(lp, ps, outer_n);
  rp.dP1 = make_fastdiv((uint32_t)(p - 1));
  // tables: perm_in[q] = g^q, perm_out[n-1] = r with g^-r = n, spectrum of b
  const uint64_t g = primitive_root(p);
  const uint64_t ginv = mod_pow(g, p - 2, p);
  std::vector<uint32_t> pin(p - 1), pout(p - 1);
  uint64_t v = 1;
  for (uint64_t q = 0; q + 1 < p; ++q) {
    pin[q] = (uint32_t)v;
    v = v * g % p;
  }
  v = 1;
  std::vector<cd> bvec(p - 1);
  for (uint64_t r = 0; r + 1 < p; ++r) {
    pout[v - 1] = (uint32_t)r;
    bvec[r] = root_fwd(v, p);  // W_p^{g^-r}
    v = v * ginv % p;
  }
  host_fft_fwd(bvec);
  for (auto& x : bvec) x /= (double)(p - 1);
  std::vector<unsigned char> bin(pin.size() * 4), bout(pout.size() * 4);
  std::memcpy(bin.data(), pin.data(), bin.size());
  std::memcpy(bout.data(), pout.data(), bout.size());
  b.set_table(b.next_pass(), Builder::F_PERM_IN, b.add_table(std::move(bin)));
  b.set_table(b.next_pass(), Builder::F_PERM_OUT, b.add_table(std::move(bout)));
  b.set_table(b.next_pass(), Builder::F_RADER_BHAT, b.add_table(b.pack_complex(bvec)));
  b.plan.passes.push_back(ps);
  return B2F_OK;
}

// Estimated instructions per point of one shared-memory engine stage of
// radix R: about 10 for the shared-memory traffic, addressing and twiddle
// product, plus the codelet's arithmetic.
static double stage_cost(uint32_t R) {
  switch (R) {
    case 2: return 12.0;
    case 3: case 4: return 14.0;
    case 5: return 16.4;
    case 7: return 20.3;
    case 8: return 16.5;
    case 9: return 18.9;
    case 11: return 22.7;
    case 13: return 23.8;
    default: return 19.0;  // 16
  }
}

// The Bluestein convolution length of a length-n line: the first 7-smooth
// length >= 2n - 1, or, when that fits one CTA, the 7-smooth length up to
// 2.25 n that also fits and has the lowest estimated cost (length x the
// per-point cost of its stages): a few percent more points in radix-16/8
// stages often beat the first length's radix-7 stages.  Multi-pass
// convolutions (HBM-bound) keep the first length.
static uint64_t bluestein_length(const Builder& b, uint64_t n) {
  uint64_t m0 = 2 * n - 1;
  while (!is_smooth7(m0)) ++m0;
  if (!b.fits_one_cta(m0)) return m0;
  auto cost = [](uint64_t m) {
    double c = 0;
    for (uint32_t R : stage_radices(m)) c += stage_cost(R);
    return c * (double)m;
  };
  uint64_t best = m0;
  double best_c = cost(m0);
  for (uint64_t m = m0 + 1; m <= 9 * n / 4 && b.fits_one_cta(m); ++m) {
    if (!is_smooth7(m)) continue;
    const double c = cost(m);
    if (c < best_c) {
      best_c = c;
      best = m;
    }
  }
  return best;
}

static b2f_status add_bluestein_pass(Builder& b, int axis, uint64_t N, const LineIO& io,
                                     uint64_t outer_n, uint32_t flags, double scale, int src,
                                     int dst) {
  const uint64_t M = bluestein_length(b, N);
  Pass ps;
  ps.kind = Pass::BLUESTEIN;
  ps.axis = axis;
  ps.src = src;
  ps.dst = dst;
  ps.label = "bluestein-fused-workgroup-stage";
  ps.route = "bluestein";
  BluesteinParams& bp = ps.blue;
  LinesParams& lp = bp.L;
  lp.N = (uint32_t)N;
  lp.io = io;
  lp.flags = flags;
  lp.scale = scale;
  bp.M = (uint32_t)M;
  std::vector<cd> tw;
  if (!b.make_schedule(M, lp.sch, ps.radices, tw))
    return fail(B2F_ERR_UNSUPPORTED_LENGTH, "Bluestein convolution length is not smooth");
  lp.LD = b.ld_for(M);
  const bool tiles = io.in_inner == 1 || io.out_inner == 1;
  if (!b.choose_launch(M, 2 * (size_t)lp.LD * b.cb(), io.inner_n, tiles && io.inner_n > 1, &lp.G,
                       &ps.threads))
    return fail(B2F_ERR_UNSUPPORTED_LENGTH,
                "UnsupportedLength { len: " + std::to_string(N) +
                    " } (Bluestein convolution does not fit one CTA)");
  ps.smem = 2 * (size_t)lp.G * lp.LD * b.cb();
  b.tw_table_for(lp.flags, tw, Builder::F_BLUE_TW);
  Builder::fill_io_grid(lp, ps, outer_n);
  bp.dM = make_fastdiv((uint32_t)M);
  bp.dMN = make_fastdiv((uint32_t)(M - N));
  const std::vector<cd> bvec = chirp_spectrum(N, M);
  b.set_table(b.next_pass(), Builder::F_BLUE_BHAT, b.add_table(b.pack_complex(bvec)));
  b.set_table(b.next_pass(), Builder::F_BLUE_CHIRP, b.add_table(b.pack_complex(chirp_table(N))));
  b.plan.passes.push_back(ps);
  return B2F_OK;
}

// Splits a long smooth N = N1 * N2 with both factors fitting one CTA,
// balanced as far as the divisors allow.
static bool four_step_split(const Builder& b, uint64_t N, uint64_t* n1, uint64_t* n2) {
  uint64_t best = 0;
  double best_bal = 1e300;
  for (uint64_t d = 2; d * d <= N; ++d) {
    if (N % d) continue;
    for (uint64_t c : {d, N / d}) {
      const uint64_t e = N / c;
      if (!b.fits_one_cta(c) || !b.fits_one_cta(e)) continue;
      const double bal = std::fabs(std::log((double)c) - std::log((double)e));
      if (bal < best_bal) {
        best_bal = bal;
        best = c;
      }
    }
  }
  if (!best) return false;
  *n1 = best;
  *n2 = N / best;
  return true;
}

static b2f_status add_complex_axis(Builder& b, int axis, AxisKind kind, uint64_t N, uint64_t s,
                                   uint64_t O, bool first, bool last, double scale, int* cur,
                                   int out_buf, int ws_buf, bool inverse);

// Bluestein whose convolution length M does not fit one CTA: chirp
// pre-multiply into workspace lines of M points, FFT_M (four-step), the
// spectrum product, FFT_M again, chirp post-multiply into the output.
static b2f_status add_bluestein_large(Builder& b, int axis, uint64_t N, uint64_t s, uint64_t O,
                                      uint32_t flags, double scale, int src, int dst) {
  const uint64_t M = bluestein_length(b, N);
  const uint64_t nlines = s * O;
  b.need(BUF_WS2, nlines * M * b.cb());
  b.need(dst, N * s * O * b.cb());
  Pass pre;
  pre.kind = Pass::BLUE_ELEM;
  pre.axis = axis;
  pre.src = src;
  pre.dst = BUF_WS2;
  pre.label = "bluestein-forward-chirp-stage";
  pre.route = "bluestein";
  pre.belem = BlueElemParams{nullptr, nullptr, nullptr, (uint32_t)N, (uint32_t)M, BE_PRE,
                             flags & PF_CONJ_IN, s, nlines, 1.0, nullptr};
  const size_t chirp_tab = b.add_table(b.pack_complex(chirp_table(N)));
  b.set_table(b.next_pass(), Builder::F_BELEM_CHIRP, chirp_tab);
  b.plan.passes.push_back(pre);
  int cur = BUF_WS2;
  b2f_status st = add_complex_axis(b, axis, AxisKind::Mixed, M, 1, nlines, false, false, 1.0, &cur,
                                   BUF_WS2, BUF_WS3, false);
  if (st) return st;
  Pass mid = pre;
  mid.src = mid.dst = BUF_WS2;
  mid.label = "bluestein-spectrum-product-stage";
  mid.belem.mode = BE_MID;
  mid.belem.flags = 0;
  const std::vector<cd> bvec = chirp_spectrum(N, M);
  b.set_table(b.next_pass(), Builder::F_BELEM_BHAT, b.add_table(b.pack_complex(bvec)));
  b.plan.passes.push_back(mid);
  st = add_complex_axis(b, axis, AxisKind::Mixed, M, 1, nlines, false, false, 1.0, &cur, BUF_WS2,
                        BUF_WS3, false);
  if (st) return st;
  Pass post = pre;
  post.src = BUF_WS2;
  post.dst = dst;
  post.label = "bluestein-inverse-chirp-stage";
  post.belem.mode = BE_POST;
  post.belem.flags = flags & (PF_CONJ_OUT | PF_SCALE);
  post.belem.scale = scale;
  b.set_table(b.next_pass(), Builder::F_BELEM_CHIRP, chirp_tab);
  b.plan.passes.push_back(post);
  return B2F_OK;
}

// Rader for a prime p whose line does not fit one CTA, p - 1 smooth
// (src/runtime/rader_axis.rs:1270-1286 runs long primes as multipass Rader
// too): gather a[q] = x[g^q] into workspace lines of p - 1 points (x[0]
// kept), FFT_{p-1} (four-step), the spectrum product (X[0] = x[0] + A[0]
// kept), FFT_{p-1} again, and the scatter X[g^-r] = x[0] + conv[r].
static b2f_status add_rader_large(Builder& b, int axis, uint64_t p, uint64_t s, uint64_t O,
                                  uint32_t flags, double scale, int src, int dst) {
  const uint64_t M = p - 1;
  const uint64_t nlines = s * O;
  b.need(BUF_WS2, nlines * M * b.cb());
  b.need(dst, p * s * O * b.cb());
  const uint64_t g = primitive_root(p);
  const uint64_t ginv = mod_pow(g, p - 2, p);
  std::vector<uint32_t> pin(M), pout(M);
  std::vector<cd> bvec(M);
  uint64_t v = 1;
  for (uint64_t q = 0; q < M; ++q) {
    pin[q] = (uint32_t)v;
    v = v * g % p;
  }
  v = 1;
  for (uint64_t r = 0; r < M; ++r) {
    pout[v - 1] = (uint32_t)r;
    bvec[r] = root_fwd(v, p);  // W_p^{g^-r}
    v = v * ginv % p;
  }
  host_fft_fwd(bvec);
  for (auto& x : bvec) x /= (double)M;
  std::vector<unsigned char> bin(M * 4), bout(M * 4);
  std::memcpy(bin.data(), pin.data(), bin.size());
  std::memcpy(bout.data(), pout.data(), bout.size());
  const size_t t_in = b.add_table(std::move(bin)), t_out = b.add_table(std::move(bout));
  const size_t t_x0 = b.add_table(std::vector<unsigned char>(2 * nlines * b.cb(), 0));
  const size_t t_bhat = b.add_table(b.pack_complex(bvec));
  Pass pre;
  pre.kind = Pass::BLUE_ELEM;
  pre.axis = axis;
  pre.src = src;
  pre.dst = BUF_WS2;
  pre.label = "rader-gather-stage";
  pre.route = "rader";
  pre.belem = BlueElemParams{nullptr, nullptr, nullptr, (uint32_t)p, (uint32_t)M, BE_RADER_PRE,
                             flags & PF_CONJ_IN, s, nlines, 1.0, nullptr, nullptr, nullptr, nullptr};
  b.set_table(b.next_pass(), Builder::F_BELEM_PIN, t_in);
  b.set_table(b.next_pass(), Builder::F_BELEM_X0, t_x0);
  b.plan.passes.push_back(pre);
  int cur = BUF_WS2;
  b2f_status st = add_complex_axis(b, axis, AxisKind::Mixed, M, 1, nlines, false, false, 1.0, &cur,
                                   BUF_WS2, BUF_WS3, false);
  if (st) return st;
  Pass mid = pre;
  mid.src = mid.dst = BUF_WS2;
  mid.label = "rader-spectrum-product-stage";
  mid.belem.mode = BE_RADER_MID;
  mid.belem.flags = 0;
  b.set_table(b.next_pass(), Builder::F_BELEM_BHAT, t_bhat);
  b.set_table(b.next_pass(), Builder::F_BELEM_X0, t_x0);
  b.plan.passes.push_back(mid);
  st = add_complex_axis(b, axis, AxisKind::Mixed, M, 1, nlines, false, false, 1.0, &cur, BUF_WS2,
                        BUF_WS3, false);
  if (st) return st;
  Pass post = pre;
  post.src = BUF_WS2;
  post.dst = dst;
  post.label = "rader-scatter-stage";
  post.belem.mode = BE_RADER_POST;
  post.belem.flags = flags & (PF_CONJ_OUT | PF_SCALE);
  post.belem.scale = scale;
  b.set_table(b.next_pass(), Builder::F_BELEM_POUT, t_out);
  b.set_table(b.next_pass(), Builder::F_BELEM_X0, t_x0);
  b.plan.passes.push_back(post);
  return B2F_OK;
}

// One complex axis of a plan: N points, stride s (complex elements), O
// outer rows of N*s elements.  Appends one or two passes and returns the
// buffer that holds the result.
static b2f_status add_complex_axis(Builder& b, int axis, AxisKind kind, uint64_t N, uint64_t s,
                                   uint64_t O, bool first, bool last, double scale, int* cur,
                                   int out_buf, int ws_buf, bool inverse) {
  uint32_t flags = 0;
  if (inverse && first) flags |= PF_CONJ_IN;
  if (inverse && last) flags |= PF_CONJ_OUT;
  if (last && scale != 1.0) flags |= PF_SCALE;
  LineIO io{};
  uint64_t outer_n;
  if (s == 1) {
    io.inner_n = (uint32_t)O;
    io.mid_n = 1;
    io.in_es = io.out_es = 1;
    io.in_inner = io.out_inner = (int64_t)N;
    io.in_outer = io.out_outer = 0;
    outer_n = 1;
  } else {
    io.inner_n = (uint32_t)s;
    io.mid_n = 1;
    io.in_es = io.out_es = (int64_t)s;
    io.in_inner = io.out_inner = 1;
    io.in_outer = io.out_outer = (int64_t)(N * s);
    outer_n = O;
    flags |= PF_CFIRST_LOAD | PF_CFIRST_STORE;
  }
  const int src = *cur;
  if (N == 1) {
    Pass ps;
    ps.kind = Pass::SCALE_COPY;
    ps.axis = axis;
    ps.src = src;
    ps.dst = out_buf;
    ps.label = "direct-dft-stage";
    ps.route = "direct-dft";
    ps.copy_n = O * s;
    ps.copy_scale = (flags & PF_SCALE) ? scale : 1.0;
    ps.copy_conj = false;
    b.plan.passes.push_back(ps);
    *cur = out_buf;
    return B2F_OK;
  }
  if (kind == AxisKind::Rader) {
    // Rader needs p - 1 smooth and the line in one CTA; otherwise Bluestein
    // (src/runtime/rader_axis.rs:1260-1268 prefers Bluestein's register
    // kernel for non-smooth p - 1 the same way).
    if (is_smooth13(N - 1) && b.fits_one_cta(N)) {
      b2f_status st = add_rader_pass(b, axis, N, io, outer_n, flags, scale, src, out_buf);
      if (st == B2F_OK) {
        *cur = out_buf;
        return st;
      }
    } else if (is_smooth13(N - 1)) {
      // too long for one CTA: multipass Rader over p - 1 (half Bluestein's
      // convolution length)
      b2f_status st = add_rader_large(b, axis, N, s, O, flags, scale, src, out_buf);
      if (st == B2F_OK) *cur = out_buf;
      return st;
    }
    kind = AxisKind::Bluestein;
  }
  if (kind == AxisKind::Bluestein) {
    const uint64_t M = bluestein_length(b, N);
    b2f_status st;
    if (b.fits_one_cta(M))
      st = add_bluestein_pass(b, axis, N, io, outer_n, flags, scale, src, out_buf);
    else
      st = add_bluestein_large(b, axis, N, s, O, flags, scale, src, out_buf);
    if (st == B2F_OK) *cur = out_buf;
    return st;
  }
  const bool p2 = (N & (N - 1)) == 0;
  b.need(out_buf, N * s * O * b.cb());
  // A long strided axis in one pass holds G*N values per CTA, so only two
  // to four adjacent columns fit: rows of 16-32 bytes, strided far apart.
  // Split into two passes of about sqrt(N), each a tile of many adjacent
  // columns (rows of hundreds of bytes), once enough columns exist.
  const bool split_strided = s >= 16 && N >= 2048;
  if (b.fits_one_cta(N) && !split_strided) {
    b2f_status st = add_lines_pass(b, axis, N, io, outer_n, flags, scale, src, out_buf,
                                   p2 ? "fused-pow2-workgroup-stage" : "fused-smooth-workgroup-stage",
                                   "mixed");
    if (st == B2F_OK) *cur = out_buf;
    return st;
  }
  // four-step: n = N2*n1 + n2, k = k1 + N1*k2
  b.need(ws_buf, N * s * O * b.cb());
  b.need(out_buf, N * s * O * b.cb());
  uint64_t N1, N2;
  if (!four_step_split(b, N, &N1, &N2))
    return fail(B2F_ERR_UNSUPPORTED_LENGTH,
                "UnsupportedLength { len: " + std::to_string(N) + " } (no four-step split)");
  // Very long contiguous lines: the balanced split's column pass (N1 >=
  // 2048, stride N2) again holds only a few adjacent columns per CTA, so
  // such lines take three passes instead: columns of N1 <= 256 (wide
  // tiles), then each row of N2 = B*C as columns of B (stride C, C
  // adjacent columns) and rows of C stored transposed.
  uint64_t B3 = 0, C3 = 0;
  if (s == 1 && N > (1ull << 22)) {
    for (uint64_t d = 256; d >= 16; --d) {
      if (N % d || !b.fits_one_cta(d)) continue;
      uint64_t bb, cc;
      if (four_step_split(b, N / d, &bb, &cc) && cc >= 16) {
        N1 = d;
        N2 = N / d;
        B3 = bb;
        C3 = cc;
        break;
      }
    }
  }
  // W_M^{row * n} on the store of pass `idx` from two tables of about
  // sqrt(M) values each, split at a power of two L >= sqrt(M) (the
  // exponent splits with a shift)
  auto store_twiddles = [&](size_t idx, uint64_t M) {
    LinesParams& lp = b.plan.passes[idx].lines;
    lp.tw_store_M = M;
    if (!b.plan.cfg.tuning.twiddle_table) return;
    uint64_t L = 1;
    while (L * L < M) L <<= 1;
    std::vector<cd> ta, tb;
    for (uint64_t q = 0; q * L < M; ++q) ta.push_back(root_fwd(q * L, M));
    for (uint64_t q = 0; q < L; ++q) tb.push_back(root_fwd(q, M));
    b.set_table(idx, Builder::F_TWS_A, b.add_table(b.pack_complex(ta)));
    b.set_table(idx, Builder::F_TWS_B, b.add_table(b.pack_complex(tb)));
    lp.d_tws = make_fastdiv((uint32_t)L);
  };
  {
    // pass A: columns n1 (stride N2*s), W_N^{n2 k1} on store, src -> ws
    LineIO a{};
    a.inner_n = (uint32_t)(N2 * s);
    a.mid_n = 1;
    a.in_es = a.out_es = (int64_t)(N2 * s);
    a.in_inner = a.out_inner = 1;
    a.in_outer = a.out_outer = (int64_t)(N * s);
    a.tw_div = (uint32_t)s;
    uint32_t fa = PF_CFIRST_LOAD | PF_CFIRST_STORE | PF_TW_STORE;
    if (inverse && first) fa |= PF_CONJ_IN;
    const char* lab = p2 ? "smooth-axis-phase1-fused-pow2-stage" : "smooth-axis-phase1-fused-smooth-stage";
    const size_t pass_a = b.next_pass();
    b2f_status st = add_lines_pass(b, axis, N1, a, O, fa, 1.0, src, ws_buf, lab, "mixed");
    if (st) return st;
    store_twiddles(pass_a, N);
  }
  if (B3) {
    // pass B1: in each row k1 (N2 = B3*C3 points, n2 = m1*C3 + m2), the
    // columns m2 over m1 (stride C3), W_N2^{m2 j1} on store, in place on ws
    LineIO c1{};
    c1.inner_n = (uint32_t)C3;
    c1.mid_n = (uint32_t)N1;
    c1.in_es = c1.out_es = (int64_t)C3;
    c1.in_inner = c1.out_inner = 1;
    c1.in_mid = c1.out_mid = (int64_t)N2;
    c1.in_outer = c1.out_outer = (int64_t)N;
    c1.tw_div = 1;
    const size_t pass_b1 = b.next_pass();
    b2f_status st = add_lines_pass(b, axis, B3, c1, O, PF_CFIRST_LOAD | PF_CFIRST_STORE | PF_TW_STORE,
                                   1.0, ws_buf, ws_buf, "smooth-axis-phase2a-column-stage", "mixed");
    if (st) return st;
    store_twiddles(pass_b1, N2);
    // pass B2: rows m2 of C3 contiguous points for each (k1, j1), stored at
    // k1 + N1*(j1 + B3*j2); lines of adjacent k1 share each output row
    LineIO c2{};
    c2.inner_n = (uint32_t)N1;
    c2.mid_n = (uint32_t)B3;
    c2.in_es = 1;
    c2.out_es = (int64_t)(N1 * B3);
    c2.in_inner = (int64_t)N2;
    c2.out_inner = 1;
    c2.in_mid = (int64_t)C3;
    c2.out_mid = (int64_t)N1;
    c2.in_outer = c2.out_outer = (int64_t)N;
    uint32_t f2 = PF_CFIRST_STORE;
    if (inverse && last) f2 |= PF_CONJ_OUT;
    if (last && scale != 1.0) f2 |= PF_SCALE;
    st = add_lines_pass(b, axis, C3, c2, O, f2, scale, ws_buf, out_buf,
                        "smooth-axis-phase2b-row-stage", "mixed");
    if (st) return st;
    *cur = out_buf;
    return B2F_OK;
  }
  {
    // pass B: rows n2 of each k1, stored transposed at k1 + N1*k2, ws -> out
    LineIO r{};
    uint64_t outer_b;
    uint32_t fb = 0;
    if (s == 1) {
      r.inner_n = (uint32_t)N1;
      r.mid_n = 1;
      r.in_es = 1;
      r.out_es = (int64_t)N1;
      r.in_inner = (int64_t)N2;
      r.out_inner = 1;
      r.in_outer = r.out_outer = (int64_t)N;
      outer_b = O;
      fb = PF_CFIRST_STORE;
    } else {
      r.inner_n = (uint32_t)s;
      r.mid_n = (uint32_t)N1;
      r.in_es = (int64_t)s;
      r.out_es = (int64_t)(N1 * s);
      r.in_inner = r.out_inner = 1;
      r.in_mid = (int64_t)(N2 * s);
      r.out_mid = (int64_t)s;
      r.in_outer = r.out_outer = (int64_t)(N * s);
      outer_b = O;
      fb = PF_CFIRST_LOAD | PF_CFIRST_STORE;
    }
    if (inverse && last) fb |= PF_CONJ_OUT;
    if (last && scale != 1.0) fb |= PF_SCALE;
    const char* lab = p2 ? "smooth-axis-phase2-fused-pow2-stage" : "smooth-axis-phase2-fused-smooth-stage";
    b2f_status st = add_lines_pass(b, axis, N2, r, outer_b, fb, scale, ws_buf, out_buf, lab, "mixed");
    if (st) return st;
  }
  *cur = out_buf;
  return B2F_OK;
}

static b2f_status add_real_pass(Builder& b, bool r2c, uint64_t N0, uint64_t nlines, double scale,
                                bool do_scale, int src, int dst) {
  Pass ps;
  ps.kind = r2c ? Pass::R2C : Pass::C2R;
  ps.axis = 0;
  ps.src = src;
  ps.dst = dst;
  ps.route = "real";
  RealParams& rp = ps.real;
  rp.N0 = (uint32_t)N0;
  rp.h = (uint32_t)(N0 / 2);
  rp.nlines = nlines;
  rp.scale = scale;
  rp.flags = do_scale ? PF_SCALE : 0;
  const bool even = N0 % 2 == 0;
  const uint64_t nfft = even ? N0 / 2 : N0;
  const uint64_t nbuf = even ? (r2c ? N0 / 2 : N0 / 2 + 1) : N0;
  std::vector<cd> tw;
  if (!b.make_schedule(nfft, rp.sch, ps.radices, tw) || !b.fits_one_cta(nbuf))
    return fail(B2F_ERR_UNSUPPORTED_LENGTH,
                "UnsupportedLength { len: " + std::to_string(N0) +
                    " } (real axis-0 lines need an even length whose half is 13-smooth, or an odd 13-smooth length, within one CTA)");
  rp.LD = b.ld_for(nbuf);
  uint32_t G, T;
  const Tuning& tn = b.plan.cfg.tuning;
  const uint64_t h = N0 / 2;
  // even N0 with a power-of-two half of 16..4096 (f32, f64; the planner's
  // stage order, no explicit launch shape): the fixed-length register
  // kernels, h/16 threads a line, one buffer of LD = h + h/16 + 1 per line
  ps.real_fx = even && h >= 16 && h <= 4096 && (h & (h - 1)) == 0 &&
               (b.plan.prec == PREC_F32 || b.plan.prec == PREC_F64) && tn.radix_order == 0 &&
               tn.lines_per_block <= 0 && tn.threads_per_block <= 0;
  if (ps.real_fx) {
    const uint64_t TL = h / 16;
    rp.LD = (uint32_t)(h + h / 16 + 1);
    uint64_t g = std::max<uint64_t>(1, 256 / TL);
    g = std::min<uint64_t>(g, std::max<uint64_t>(nlines, 1));
    while (g > 1 && g * rp.LD * b.cb() > b.smem_budget) g >>= 1;
    if (g * rp.LD * b.cb() > b.smem_budget) ps.real_fx = false;
    G = (uint32_t)g;
    T = (uint32_t)(g * TL);
  }
  if (!ps.real_fx) {
    rp.LD = b.ld_for(nbuf);
    if (!b.choose_launch(nfft, 2 * (size_t)rp.LD * b.cb(), nlines, false, &G, &T))
      return fail(B2F_ERR_UNSUPPORTED_LENGTH, "real line does not fit a CTA");
  }
  rp.G = G;
  ps.threads = T;
  ps.smem = (ps.real_fx ? 1 : 2) * (size_t)G * rp.LD * b.cb();
  if (ps.real_fx) {
    std::vector<cd> rt(h);
    for (uint64_t k = 0; k < h; ++k) rt[k] = root_fwd(k, N0);
    b.set_table(b.next_pass(), Builder::F_REAL_RTW, b.add_table(b.pack_complex(rt)));
  }
  rp.dh = make_fastdiv(std::max<uint32_t>(rp.h, 1));
  rp.dG = make_fastdiv(G);
  rp.dN0 = make_fastdiv((uint32_t)N0);
  rp.dP = make_fastdiv((uint32_t)(N0 / 2 + 1));
  b.tw_table_for(rp.flags, tw, Builder::F_REAL_TW);
  ps.grid = (unsigned)((nlines + G - 1) / G);
  ps.label = r2c ? (even ? "r2c-packed-fused-stage" : "r2c-odd-fused-stage")
                 : (even ? "c2r-packed-fused-stage" : "c2r-odd-fused-stage");
  b.plan.passes.push_back(ps);
  return B2F_OK;
}

// Whether the fused axis-0 real pass can run N0 (even N0 with N0/2 13-smooth,
// or odd 13-smooth N0, within one CTA).
static bool real_fast_path(const Builder& b, uint64_t N0) {
  const bool even = N0 % 2 == 0;
  const uint64_t nfft = even ? N0 / 2 : N0;
  const uint64_t nbuf = even ? N0 / 2 + 1 : N0;
  return !stage_radices(nfft).empty() && b.fits_one_cta(nbuf) && N0 >= 2;
}

static Pass real_elem_pass(RealElemMode mode, uint64_t N0, uint64_t nlines, int src, int dst,
                           const char* label) {
  Pass ps;
  ps.kind = Pass::REAL_ELEM;
  ps.axis = 0;
  ps.src = src;
  ps.dst = dst;
  ps.label = label;
  ps.route = "real";
  ps.relem = RealElemParams{nullptr, nullptr, (uint32_t)N0, (uint32_t)(N0 / 2 + 1), mode, 0, nlines};
  return ps;
}

// R2C axis 0 for any N0: expand to complex lines, complex FFT (any route),
// keep the first N0/2+1 bins.
static b2f_status add_real_generic_r2c(Builder& b, uint64_t N0, uint64_t nlines, bool last,
                                       double scale) {
  b.need(BUF_WS4, N0 * nlines * b.cb());
  b.plan.passes.push_back(real_elem_pass(RE_EXPAND, N0, nlines, BUF_IN, BUF_WS4, "r2c-expand-stage"));
  int cur = BUF_WS4;
  b2f_status st = add_complex_axis(b, 0, axis_kind_for(b.plan.cfg, 0), N0, 1, nlines, true, last,
                                   scale, &cur, BUF_WS4, BUF_WS5, false);
  if (st) return st;
  b.plan.passes.push_back(real_elem_pass(RE_PACK, N0, nlines, BUF_WS4, BUF_OUT, "r2c-pack-stage"));
  return B2F_OK;
}

// C2R axis 0 for any N0: Hermitian mirror into complex lines, inverse
// complex FFT (any route), real part.
static b2f_status add_real_generic_c2r(Builder& b, uint64_t N0, uint64_t nlines, double scale,
                                       int src) {
  b.need(BUF_WS4, N0 * nlines * b.cb());
  b.plan.passes.push_back(real_elem_pass(RE_UNPACK, N0, nlines, src, BUF_WS4, "c2r-unpack-stage"));
  int cur = BUF_WS4;
  b2f_status st = add_complex_axis(b, 0, axis_kind_for(b.plan.cfg, 0), N0, 1, nlines, true, true,
                                   scale, &cur, BUF_WS4, BUF_WS5, true);
  if (st) return st;
  b.plan.passes.push_back(real_elem_pass(RE_TAKE_REAL, N0, nlines, BUF_WS4, BUF_OUT, "c2r-take-real-stage"));
  return B2F_OK;
}

// The small-volume route (src/runtime/small_volume.rs:223-272): an f32 C2C
// plan over every axis of a rank-2 or rank-3 volume of at most 4096 points
// whose axes are all 2,3,5,7,11,13-smooth, no forced Rader/Bluestein axis,
// the automatic large route and fuse_small_volumes on.  One pass, one CTA
// per volume.  Returns false when the configuration is not eligible.
static bool try_small_volume(Builder& b, double scale, bool inverse) {
  const Config& cfg = b.plan.cfg;
  const Tuning& t = cfg.tuning;
  const size_t rank = cfg.shape.size();
  if (b.plan.prec != PREC_F32 || rank < 2 || rank > (size_t)kSmallVolumeMaxRank) return false;
  std::vector<uint32_t> axes(cfg.axes.begin(), cfg.axes.end());
  std::sort(axes.begin(), axes.end());
  for (size_t i = 0; i < rank; ++i)
    if (axes.size() != rank || axes[i] != i) return false;
  if (!t.force_rader_axes.empty() || !t.force_bluestein_axes.empty() || t.large_route != 0 ||
      !t.fuse_small_volumes || t.lines_per_block > 0 || t.threads_per_block > 0)
    return false;
  uint64_t V = 1;
  for (auto n : cfg.shape) V *= n;
  if (V > kSmallVolumeMaxPoints) return false;
  Pass ps;
  ps.kind = Pass::SMALL_VOLUME;
  ps.label = "small-volume-stage";
  ps.route = "mixed-radix";
  ps.axis = -1;
  ps.src = BUF_IN;
  ps.dst = BUF_OUT;
  SmallVolumeParams& sv = ps.svol;
  sv.rank = (uint32_t)rank;
  sv.V = (uint32_t)V;
  sv.nvol = cfg.batch;
  sv.scale = scale;
  sv.flags = (inverse ? (PF_CONJ_IN | PF_CONJ_OUT) : 0u) | (scale != 1.0 ? PF_SCALE : 0u);
  std::vector<cd> tw;
  uint32_t buf = 0;
  uint64_t stride = 1;
  for (size_t a = 0; a < rank; ++a) {
    const uint64_t N = cfg.shape[a];
    std::vector<uint32_t> rad;
    std::vector<cd> tw_a;
    if (N < 2 || !b.make_schedule(N, sv.sch[a], rad, tw_a)) return false;
    for (uint32_t st = 0; st < sv.sch[a].nst; ++st) sv.sch[a].st[st].tw_off += (uint32_t)tw.size();
    tw.insert(tw.end(), tw_a.begin(), tw_a.end());
    sv.dims[a] = (uint32_t)N;
    sv.strides[a] = (uint32_t)stride;
    sv.dN[a] = make_fastdiv((uint32_t)N);
    sv.dS[a] = make_fastdiv((uint32_t)stride);
    sv.LD[a] = b.ld_for(N);
    buf = std::max<uint32_t>(buf, (uint32_t)(V / N) * sv.LD[a]);
    ps.radices.insert(ps.radices.end(), rad.begin(), rad.end());
    stride *= N;
  }
  sv.buf = buf;
  ps.smem = ((size_t)V + 2 * (size_t)buf) * b.cb();
  if (ps.smem > b.smem_budget) return false;
  ps.threads = 256;
  ps.grid = (unsigned)std::min<uint64_t>(cfg.batch, 0x7FFFFFFFull);
  if (cfg.batch > 0x7FFFFFFFull) return false;
  if (t.twiddle_table && !tw.empty()) {
    sv.flags |= PF_TW_TABLE;
    b.set_table(b.next_pass(), Builder::F_SVOL_TW, b.add_table(b.pack_complex(tw)));
  }
  b.plan.passes.push_back(ps);
  return true;
}

Plan::~Plan() {
  int prev = -1;
  cudaGetDevice(&prev);
  if (device >= 0) cudaSetDevice(device);
  for (void* p : device_allocs)
    if (p) cudaFree(p);
  for (void* p : ws)
    if (p) cudaFree(p);
  if (inplace_copy) cudaFree(inplace_copy);
  if (last_done) cudaEventDestroy(last_done);
  if (view_in) cudaFree(view_in);
  if (view_out) cudaFree(view_out);
  if (prev >= 0) cudaSetDevice(prev);
}

static std::string json_escape(const std::string& s) {
  std::string o;
  for (char c : s) {
    if (c == '"' || c == '\\') o += '\\';
    o += c;
  }
  return o;
}

static const char* prec_name(int p) { return p == 0 ? "f32" : p == 1 ? "f64" : "df64"; }

static void build_diagnostics(Plan& plan) {
  std::ostringstream os;
  const char* tr = plan.kind == B2F_C2C ? "c2c" : plan.kind == B2F_R2C ? "r2c" : "c2r";
  const char* cfmt = plan.prec == PREC_F32 ? "complex-f32" : plan.prec == PREC_F64 ? "complex-f64" : "complex-df64";
  const char* rfmt = plan.prec == PREC_F64 ? "real-f64" : "real-f32";
  os << "{\"transform\":\"" << tr << "\",\"route\":\"" << route_name(plan.route) << "\"";
  os << ",\"precision\":\"" << prec_name(plan.cfg.precision) << "\"";
  os << ",\"execution_kind\":\"normal\"";
  os << ",\"axis_kinds\":[";
  for (size_t i = 0; i < plan.axis_kinds.size(); ++i)
    os << (i ? "," : "") << "\"" << axis_kind_name(plan.axis_kinds[i]) << "\"";
  os << "],\"axis_factors\":[";
  for (size_t i = 0; i < plan.axis_factors.size(); ++i) {
    os << (i ? "," : "") << "[";
    for (size_t j = 0; j < plan.axis_factors[i].size(); ++j) os << (j ? "," : "") << plan.axis_factors[i][j];
    os << "]";
  }
  os << "],\"stages\":[";
  for (size_t i = 0; i < plan.passes.size(); ++i) {
    const Pass& p = plan.passes[i];
    const char* kind = p.kind == Pass::LINES ? "lines" : p.kind == Pass::POW2 ? (p.colmajor ? "register-pow2-columns" : "register-pow2-lines") : p.kind == Pass::RADER ? "rader"
                     : p.kind == Pass::BLUESTEIN ? "bluestein" : p.kind == Pass::R2C ? "r2c"
                     : p.kind == Pass::C2R ? "c2r" : p.kind == Pass::BLUE_ELEM ? "bluestein-elementwise"
                     : p.kind == Pass::REAL_ELEM ? "real-elementwise"
                     : p.kind == Pass::TC_DFT64 ? "tensor-core-dft"
                     : p.kind == Pass::SMALL_VOLUME ? "small-volume" : "scale-copy";
    uint32_t G = (p.kind == Pass::LINES || p.kind == Pass::POW2) ? p.lines.G : p.kind == Pass::RADER ? p.rader.L.G
               : p.kind == Pass::BLUESTEIN ? p.blue.L.G : (p.kind == Pass::R2C || p.kind == Pass::C2R) ? p.real.G : 0;
    os << (i ? "," : "") << "{\"label\":\"" << json_escape(p.label) << "\",\"kind\":\"" << kind
       << "\",\"route\":\"" << p.route << "\",\"axis\":" << p.axis << ",\"radices\":[";
    for (size_t j = 0; j < p.radices.size(); ++j) os << (j ? "," : "") << p.radices[j];
    os << "],\"grid\":" << p.grid << ",\"threads\":" << p.threads << ",\"lines_per_block\":" << G
       << ",\"smem_bytes\":" << p.smem << ",\"src\":" << p.src << ",\"dst\":" << p.dst;
    if (p.kind == Pass::BLUESTEIN) os << ",\"convolution_length\":" << p.blue.M;
    if (p.kind == Pass::RADER) os << ",\"convolution_length\":" << (p.rader.L.N - 1);
    if (p.tma) os << ",\"tma_tiles\":true,\"persistent_grid\":" << p.tma_grid;
    os << "}";
  }
  os << "],\"buffer_requirements\":[";
  os << "{\"role\":\"input\",\"required_bytes\":" << plan.in_bytes << ",\"format\":\""
     << (plan.kind == B2F_R2C ? rfmt : cfmt) << "\"}";
  os << ",{\"role\":\"output\",\"required_bytes\":" << plan.out_bytes << ",\"format\":\""
     << (plan.kind == B2F_C2R ? rfmt : cfmt) << "\"}";
  if (plan.workspace_total() > 0)
    os << ",{\"role\":\"workspace\",\"required_bytes\":" << plan.workspace_total()
       << ",\"format\":\"" << cfmt << "\"}";
  if (plan.table_bytes > 0)
    os << ",{\"role\":\"helper:twiddle-luts-total\",\"required_bytes\":" << plan.table_bytes
       << ",\"format\":\"" << cfmt << "\"}";
  os << "]";
  const Tuning& t = plan.cfg.tuning;
  std::ostringstream tj;
  tj << "{\"workgroup_size\":" << t.workgroup_size << ",\"fused_workgroup_size\":" << t.fused_workgroup_size
     << ",\"rader_max_prime\":" << t.rader_max_prime << ",\"direct_max_prime\":" << t.direct_max_prime
     << ",\"fused_min_convolution_length\":" << t.fused_min_convolution_length
     << ",\"fuse_long_axes\":" << (t.fuse_long_axes ? "true" : "false")
     << ",\"fuse_small_volumes\":" << (t.fuse_small_volumes ? "true" : "false")
     << ",\"lines_per_block\":" << t.lines_per_block << ",\"threads_per_block\":" << t.threads_per_block
     << ",\"twiddle_table\":" << (t.twiddle_table ? "true" : "false")
     << ",\"radix_order\":" << t.radix_order << ",\"tma_tiles\":" << t.tma_tiles
     << ",\"tensor_cores\":" << (t.tensor_cores ? "true" : "false") << "}";
  os << ",\"tuning\":{\"requested\":" << tj.str() << ",\"effective\":" << tj.str() << "}";
  os << ",\"supports_in_place\":" << (plan.in_place_kernels ? "true" : "false");
  os << ",\"device\":" << plan.device << "}";
  plan.diag_json = os.str();
}

b2f_status create_plan(const Config& cfg_in, int32_t kind, int device, Plan** out,
                       size_t smem_budget) {
  *out = nullptr;
  b2f_status st = validate_config(cfg_in);
  if (st) return st;
  const bool dry = device == -2;
  if (kind != B2F_C2C) {
    const bool want_inv = kind == B2F_C2R;
    if ((cfg_in.direction == B2F_INVERSE) != want_inv)
      return fail(B2F_ERR_INVALID_REAL_DIRECTION,
                  std::string("InvalidRealTransformDirection { transform: ") + (want_inv ? "c2r" : "r2c") +
                      ", expected: " + (want_inv ? "inverse" : "forward") + " }");
    for (size_t i = 0; i < cfg_in.axes.size() || i < cfg_in.shape.size(); ++i)
      if (cfg_in.axes.size() != cfg_in.shape.size() || cfg_in.axes[i] != i)
        return fail(B2F_ERR_UNSUPPORTED_REAL_AXES, "UnsupportedRealAxes: real transforms use every axis in order");
    if (cfg_in.precision == B2F_DF64)
      return fail(B2F_ERR_PRECISION_UNSUPPORTED,
                  "PrecisionUnsupported { requested: df64, route: real, reason: real-transforms-support-f32-and-f64 }");
  }
  int prev = -1;
  if (!dry) {
    cudaGetDevice(&prev);
    if (device < 0) device = prev < 0 ? 0 : prev;
    if (cudaSetDevice(device) != cudaSuccess)
      return fail(B2F_ERR_DEVICE, "cudaSetDevice failed: " + std::string(cudaGetErrorString(cudaGetLastError())));
  }
  std::unique_ptr<Plan> plan(new Plan());
  plan->cfg = cfg_in;
  plan->kind = kind;
  plan->device = dry ? -2 : device;
  plan->prec = (Prec)cfg_in.precision;
  const Config& cfg = plan->cfg;
  for (auto a : cfg.axes) {
    plan->axis_kinds.push_back(axis_kind_for(cfg, a));
    plan->axis_factors.push_back(factor_supported_length(cfg.shape[a]));
  }
  plan->route = select_route(cfg);
  Builder b{*plan, dry, 0, {}};
  if (dry) {
    b.smem_budget = smem_budget ? smem_budget : 232448;
  } else {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess)
      v = 48 * 1024;
    b.smem_budget = (size_t)v;
  }
  const size_t cbytes = complex_bytes(plan->prec);
  const size_t sbytes = plan->prec == PREC_F64 ? 8 : 4;
  uint64_t logical = 1;
  for (auto s : cfg.shape) logical *= s;
  const uint64_t total = logical * cfg.batch;
  const double scale = plan_scale(cfg, logical);
  const bool inverse = cfg.direction == B2F_INVERSE;
  const int rank = (int)cfg.shape.size();

  if (kind == B2F_C2C) {
    plan->in_bytes = plan->out_bytes = total * cbytes;
    int cur = BUF_IN;
    if (total == 1) {
      Pass ps;
      ps.kind = Pass::SCALE_COPY;
      ps.label = "direct-dft-stage";
      ps.route = "direct-dft";
      ps.src = BUF_IN;
      ps.dst = BUF_OUT;
      ps.copy_n = 1;
      ps.copy_scale = scale;
      plan->passes.push_back(ps);
    } else if (cfg.tuning.tensor_cores && plan->prec == PREC_F32 && cfg.axes.size() == 1 &&
               cfg.axes[0] == 0 && cfg.shape[0] == 64) {
      // the tensor-core DFT layer: every (contiguous) line of axis 0 in one pass
      Pass ps;
      ps.kind = Pass::TC_DFT64;
      ps.label = "tensor-core-dft64-split-tf32-stage";
      ps.route = "mixed-radix";
      ps.axis = 0;
      ps.src = BUF_IN;
      ps.dst = BUF_OUT;
      ps.radices = {64};
      ps.tc_nlines = total / 64;
      ps.tc_scale = (float)scale;
      ps.tc_inverse = inverse;
      ps.threads = 256;
      ps.smem = 192 * 1024;
      int nsm = 148;
      if (!dry) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
      ps.grid = (unsigned)std::min<uint64_t>((uint64_t)nsm, (ps.tc_nlines + 31) / 32);
      const std::vector<float> tab = dft64_tc_table();
      std::vector<unsigned char> tb(tab.size() * 4);
      std::memcpy(tb.data(), tab.data(), tb.size());
      ps.tc_table = b.add_table(std::move(tb));
      ps.tc_err = b.add_table(std::vector<unsigned char>(16, 0));
      plan->passes.push_back(ps);
    } else if (try_small_volume(b, scale, inverse)) {
      // every axis in one pass
    } else {
      for (size_t ai = 0; ai < cfg.axes.size(); ++ai) {
        const uint32_t a = cfg.axes[ai];
        uint64_t s = 1, O = cfg.batch;
        for (uint32_t d = 0; d < a; ++d) s *= cfg.shape[d];
        for (int d = a + 1; d < rank; ++d) O *= cfg.shape[d];
        st = add_complex_axis(b, (int)a, plan->axis_kinds[ai], cfg.shape[a], s, O, ai == 0,
                              ai + 1 == cfg.axes.size(), scale, &cur, BUF_OUT, BUF_WS0, inverse);
        if (st) return st;
      }
    }
  } else {
    const uint64_t N0 = cfg.shape[0];
    plan->packed_shape = cfg.shape;
    plan->packed_shape[0] = N0 / 2 + 1;
    uint64_t plog = 1;
    for (auto s : plan->packed_shape) plog *= s;
    const uint64_t ptotal = plog * cfg.batch;
    const uint64_t nlines = total / N0;
    plan->in_place_kernels = false;
    if (kind == B2F_R2C) {
      plan->in_bytes = total * sbytes;
      plan->out_bytes = ptotal * cbytes;
      if (real_fast_path(b, N0))
        st = add_real_pass(b, true, N0, nlines, scale, rank == 1 && scale != 1.0, BUF_IN, BUF_OUT);
      else
        st = add_real_generic_r2c(b, N0, nlines, rank == 1, scale);
      if (st) return st;
      int cur = BUF_OUT;
      for (int a = 1; a < rank; ++a) {
        uint64_t s = 1, O = cfg.batch;
        for (int d = 0; d < a; ++d) s *= plan->packed_shape[d];
        for (int d = a + 1; d < rank; ++d) O *= plan->packed_shape[d];
        st = add_complex_axis(b, a, axis_kind_for(cfg, a), cfg.shape[a], s, O, false, a == rank - 1,
                              scale, &cur, BUF_OUT, BUF_WS0, false);
        if (st) return st;
      }
    } else {
      plan->in_bytes = ptotal * cbytes;
      plan->out_bytes = total * sbytes;
      int cur = BUF_IN;
      for (int a = 1; a < rank; ++a) {
        uint64_t s = 1, O = cfg.batch;
        for (int d = 0; d < a; ++d) s *= plan->packed_shape[d];
        for (int d = a + 1; d < rank; ++d) O *= plan->packed_shape[d];
        st = add_complex_axis(b, a, axis_kind_for(cfg, a), cfg.shape[a], s, O, a == 1, a == rank - 1,
                              1.0, &cur, BUF_WS0, BUF_WS1, true);
        if (st) return st;
      }
      if (real_fast_path(b, N0))
        st = add_real_pass(b, false, N0, nlines, scale, scale != 1.0, cur, BUF_OUT);
      else
        st = add_real_generic_c2r(b, N0, nlines, scale, cur);
      if (st) return st;
    }
  }
  build_diagnostics(*plan);
  if (!dry) {
    // upload tables, allocate workspaces
    for (auto& pend : b.pending) {
      void* d = nullptr;
      if (cudaMalloc(&d, pend.second.size()) != cudaSuccess) {
        cudaGetLastError();
        if (prev >= 0) cudaSetDevice(prev);
        return fail(B2F_ERR_RESOURCE_ALLOCATION,
                    "GpuPlanResourceAllocationFailed: table of " + std::to_string(pend.second.size()) + " bytes");
      }
      plan->device_allocs[pend.first] = d;
      if (cudaMemcpy(d, pend.second.data(), pend.second.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        if (prev >= 0) cudaSetDevice(prev);
        return fail(B2F_ERR_DEVICE, "table upload failed");
      }
    }
    b.apply_patches();
    plan->shared_state = plan->workspace_total() > 0 || !plan->in_place_kernels;
    for (const Pass& ps : plan->passes)
      if (ps.kind == Pass::TC_DFT64) plan->shared_state = true;
    // every plan gets the event: executions through staged views share
    // device memory even when the plan's own route does not
    if (cudaEventCreateWithFlags(&plan->last_done, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      if (prev >= 0) cudaSetDevice(prev);
      return fail(B2F_ERR_DEVICE, "plan event creation failed");
    }
    for (int w = 0; w < kNumWorkspaces; ++w) {
      if (plan->ws_bytes[w] == 0) continue;
      if (cudaMalloc(&plan->ws[w], plan->ws_bytes[w]) != cudaSuccess) {
        cudaGetLastError();
        if (prev >= 0) cudaSetDevice(prev);
        return fail(B2F_ERR_RESOURCE_ALLOCATION,
                    "GpuPlanResourceAllocationFailed: workspace of " + std::to_string(plan->ws_bytes[w]) + " bytes");
      }
    }
    if (prev >= 0) cudaSetDevice(prev);
  }
  *out = plan.release();
  return B2F_OK;
}

// ------------------------------------------------------------ execution
static b2f_status run_passes(const Plan& plan, cudaStream_t st, const void* in, void* out) {
  if (plan.device < 0) return fail(B2F_ERR_DEVICE, "plan was created for planning only (no device)");
  void* bufs[2 + kNumWorkspaces] = {const_cast<void*>(in), out};
  for (int i = 0; i < kNumWorkspaces; ++i) bufs[2 + i] = plan.ws[i];
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != plan.device) cudaSetDevice(plan.device);
  // launches report through cudaGetLastError: clear what an unrelated
  // earlier call of this thread left there
  cudaGetLastError();
  cudaError_t e = cudaSuccess;
  for (const Pass& p0 : plan.passes) {
    Pass p = p0;  // launch parameters take the caller's pointers
    void* src = bufs[p.src];
    void* dst = bufs[p.dst];
    switch (p.kind) {
      case Pass::LINES:
        p.lines.in = src;
        p.lines.out = dst;
        e = launch_lines(plan.prec, p.lines, p.grid, p.threads, p.smem, st);
        break;
      case Pass::POW2: {
        p.lines.in = src;
        p.lines.out = dst;
        bool done = false;
        if (p.tma) {
          const uint64_t outer = p.grid / ((uint64_t)p.lines.io.tiles * p.lines.io.mid_n);
          done = launch_pow2_tma(p.lines, p.grid, outer, p.threads, p.tma_grid,
                                 (unsigned int*)plan.device_allocs[p.tma_err], st, &e);
        }
        if (!done) e = launch_pow2(plan.prec, p.pow2_E, p.colmajor, p.lines, p.grid, p.threads, p.smem, st);
        break;
      }
      case Pass::RADER:
        p.rader.L.in = src;
        p.rader.L.out = dst;
        e = launch_rader(plan.prec, p.rader, p.grid, p.threads, p.smem, st);
        break;
      case Pass::BLUESTEIN:
        p.blue.L.in = src;
        p.blue.L.out = dst;
        e = launch_bluestein(plan.prec, p.blue, p.grid, p.threads, p.smem, st);
        break;
      case Pass::R2C:
      case Pass::C2R:
        p.real.in = src;
        p.real.out = dst;
        if (p.real_fx)
          e = launch_real_fixed(plan.prec, p.kind == Pass::R2C, p.real, p.grid, p.threads, p.smem, st);
        else if (p.kind == Pass::R2C)
          e = launch_r2c(plan.prec, p.real, p.grid, p.threads, p.smem, st);
        else
          e = launch_c2r(plan.prec, p.real, p.grid, p.threads, p.smem, st);
        break;
      case Pass::SCALE_COPY:
        e = launch_scale_copy(plan.prec, src, dst, p.copy_n, p.copy_scale, p.copy_conj, st);
        break;
      case Pass::BLUE_ELEM:
        p.belem.in = src;
        p.belem.out = dst;
        e = launch_blue_elem(plan.prec, p.belem, st);
        break;
      case Pass::REAL_ELEM:
        p.relem.in = src;
        p.relem.out = dst;
        e = launch_real_elem(plan.prec, p.relem, st);
        break;
      case Pass::SMALL_VOLUME:
        p.svol.in = src;
        p.svol.out = dst;
        e = launch_small_volume(plan.prec, p.svol, p.threads, p.smem, st);
        break;
      case Pass::TC_DFT64:
        e = launch_dft64_tc(src, dst, (const float*)plan.device_allocs[p.tc_table], p.tc_nlines,
                            p.tc_scale, p.tc_inverse, (unsigned int*)plan.device_allocs[p.tc_err],
                            p.grid, st);
        break;
    }
    if (e != cudaSuccess) break;
  }
  if (prev >= 0 && prev != plan.device) cudaSetDevice(prev);
  if (e != cudaSuccess) return fail(B2F_ERR_DEVICE, std::string("kernel launch failed: ") + cudaGetErrorString(e));
  return B2F_OK;
}

// Runs f() ordered after the plan's previous execution when the plan holds
// device state that its executions share (Plan::shared_state): the stream
// waits for the previous execution's completion event and this execution
// records a new one.  Executions recorded into a CUDA graph (the stream is
// capturing) are ordered by the graph itself and skip the events.
template <class F>
static b2f_status ordered(const Plan& plan, cudaStream_t st, F&& f, bool force = false) {
  if (!(plan.shared_state || force) || !plan.last_done) return f();
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
    cudaGetLastError();
    return f();
  }
  if (cs != cudaStreamCaptureStatusNone) return f();
  std::lock_guard<std::mutex> lk(plan.exec_mu);
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != plan.device) cudaSetDevice(plan.device);
  if (plan.last_done_recorded && cudaStreamWaitEvent(st, plan.last_done, 0) != cudaSuccess) {
    if (prev >= 0 && prev != plan.device) cudaSetDevice(prev);
    return fail(B2F_ERR_DEVICE, "could not order the execution after the plan's previous one");
  }
  const b2f_status s = f();
  if (cudaEventRecord(plan.last_done, st) == cudaSuccess) plan.last_done_recorded = true;
  if (prev >= 0 && prev != plan.device) cudaSetDevice(prev);
  return s;
}

static b2f_status execute_in_place_impl(const Plan& plan, cudaStream_t st, void* buf);

b2f_status run_ordered(const Plan& plan, cudaStream_t st, const std::function<b2f_status()>& f) {
  return ordered(plan, st, f, true);
}

b2f_status run_passes_unordered(const Plan& plan, cudaStream_t st, const void* in, void* out) {
  return run_passes(plan, st, in, out);
}

b2f_status execute_plan(const Plan& plan, cudaStream_t st, const void* in, uint64_t in_bytes,
                        void* out, uint64_t out_bytes) {
  if (!in || !out) return fail(B2F_ERR_INVALID_ARGUMENT, "null buffer");
  if (in_bytes < plan.in_bytes)
    return fail(B2F_ERR_BUFFER_TOO_SMALL, "BufferViewTooSmall { role: input, required: " +
                                              std::to_string(plan.in_bytes) + ", actual: " + std::to_string(in_bytes) + " }");
  if (out_bytes < plan.out_bytes)
    return fail(B2F_ERR_BUFFER_TOO_SMALL, "BufferViewTooSmall { role: output, required: " +
                                              std::to_string(plan.out_bytes) + ", actual: " + std::to_string(out_bytes) + " }");
  if (in == out && !plan.in_place_kernels)
    return execute_plan_in_place(plan, st, out, std::max(in_bytes, out_bytes));
  return ordered(plan, st, [&] { return run_passes(plan, st, in, out); });
}

b2f_status execute_plan_in_place(const Plan& plan, cudaStream_t st, void* buf, uint64_t bytes) {
  if (!buf) return fail(B2F_ERR_INVALID_ARGUMENT, "null buffer");
  const uint64_t need = std::max(plan.in_bytes, plan.out_bytes);
  if (bytes < need)
    return fail(B2F_ERR_BUFFER_TOO_SMALL, "BufferViewTooSmall { role: buffer, required: " +
                                              std::to_string(need) + ", actual: " + std::to_string(bytes) + " }");
  return ordered(plan, st, [&] { return execute_in_place_impl(plan, st, buf); });
}

static b2f_status execute_in_place_impl(const Plan& plan, cudaStream_t st, void* buf) {
  if (plan.in_place_kernels) return run_passes(plan, st, buf, buf);
  // real transforms: copy the input first, like the crate's in-place copy
  // buffer (src/plan.rs:856-863), created on first use and kept.
  void* copy = nullptr;
  {
    std::lock_guard<std::mutex> lk(plan.copy_mu);
    if (!plan.inplace_copy) {
      int prev = -1;
      cudaGetDevice(&prev);
      cudaSetDevice(plan.device);
      const cudaError_t e = cudaMalloc(&plan.inplace_copy, plan.in_bytes);
      if (prev >= 0) cudaSetDevice(prev);
      if (e != cudaSuccess) {
        plan.inplace_copy = nullptr;
        cudaGetLastError();
        return fail(B2F_ERR_RESOURCE_ALLOCATION, "in-place copy buffer allocation failed");
      }
    }
    copy = plan.inplace_copy;
  }
  if (cudaMemcpyAsync(copy, buf, plan.in_bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return fail(B2F_ERR_DEVICE, "in-place input copy failed");
  return run_passes(plan, st, copy, buf);
}

}  // namespace b2f
