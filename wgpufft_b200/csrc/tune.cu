// Autotuner and persistent tuning snapshot (b2f_autotune,
// b2f_tuning_snapshot_*).
//
// The autotuner times candidate FftTuning values of one configuration on the
// device (the kernel-shape knobs this library honours: twiddle_table,
// radix_order, lines_per_block, threads_per_block), keeps the fastest candidate whose
// results match the default plan's within the precision's tolerance, and
// records it in a process-wide snapshot keyed by the configuration (shape,
// axes, batch, direction, normalisation, precision, transform kind).  The
// snapshot persists as versioned JSON with integrity checks in the manner
// of the crate's pipeline-cache snapshot (src/runtime/pipeline_cache.rs:
// 14-99, 160-260: schema and version checks, canonical ordering, duplicate
// and re-derived-key checks), plus the device it was tuned on and an FNV-1a
// checksum over the canonical entries, so a stale, edited or foreign file is
// rejected instead of applied.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "plan.h"

namespace b2f {
namespace {

constexpr const char* kSchema = "wgpufft_b200.tuning";
constexpr int64_t kVersion = 2;  // 2: entries carry radix_order

struct Entry {
  int64_t lines_per_block = 0, threads_per_block = 0, twiddle_table = 1, radix_order = 0;
  double best_us = 0, default_us = 0;
};

std::mutex g_mu;
std::map<std::string, Entry> g_entries;  // ordered by key: the canonical order
std::string g_device;                    // device the entries were tuned on

const char* kind_name(int32_t k) { return k == B2F_R2C ? "r2c" : (k == B2F_C2R ? "c2r" : "c2c"); }
const char* prec_name(int32_t p) { return p == B2F_F64 ? "f64" : (p == B2F_DF64 ? "df64" : "f32"); }
const char* dir_name(int32_t d) { return d == B2F_INVERSE ? "inverse" : "forward"; }
const char* norm_name(int32_t n) {
  switch (n) {
    case B2F_NORM_NONE: return "none";
    case B2F_NORM_FORWARD: return "forward";
    case B2F_NORM_ORTHOGONAL: return "orthogonal";
    default: return "inverse";
  }
}

template <class T>
std::string join(const std::vector<T>& v) {
  std::string s;
  for (size_t i = 0; i < v.size(); ++i) s += (i ? "," : "") + std::to_string(v[i]);
  return s;
}

// Canonical key of a configuration (everything but its tuning).
std::string config_key(const Config& c, int32_t kind) {
  std::ostringstream os;
  os << kind_name(kind) << "/" << prec_name(c.precision) << "/" << dir_name(c.direction) << "/"
     << norm_name(c.normalization) << "/shape=" << join(c.shape) << "/axes=" << join(c.axes)
     << "/batch=" << c.batch;
  return os.str();
}

bool parse_u64_list(const std::string& s, std::vector<uint64_t>& out) {
  out.clear();
  size_t i = 0;
  while (i < s.size()) {
    size_t j = s.find(',', i);
    if (j == std::string::npos) j = s.size();
    const std::string t = s.substr(i, j - i);
    if (t.empty() || t.find_first_not_of("0123456789") != std::string::npos || t.size() > 19)
      return false;
    out.push_back(std::stoull(t));
    i = j + 1;
  }
  return !out.empty();
}

// Inverse of config_key; false when the key is not one config_key writes.
bool parse_key(const std::string& key, Config& c, int32_t& kind) {
  std::vector<std::string> f;
  size_t i = 0;
  while (true) {
    size_t j = key.find('/', i);
    f.push_back(key.substr(i, j == std::string::npos ? std::string::npos : j - i));
    if (j == std::string::npos) break;
    i = j + 1;
  }
  if (f.size() != 7) return false;
  const char* kinds[] = {"c2c", "r2c", "c2r"};
  const char* precs[] = {"f32", "f64", "df64"};
  const char* norms[] = {"none", "forward", "inverse", "orthogonal"};
  kind = -1;
  for (int k = 0; k < 3; ++k)
    if (f[0] == kinds[k]) kind = k;
  c.precision = -1;
  for (int k = 0; k < 3; ++k)
    if (f[1] == precs[k]) c.precision = k;
  c.direction = f[2] == "forward" ? B2F_FORWARD : (f[2] == "inverse" ? B2F_INVERSE : -1);
  c.normalization = -1;
  for (int k = 0; k < 4; ++k)
    if (f[3] == norms[k]) c.normalization = k;
  if (kind < 0 || c.precision < 0 || c.direction < 0 || c.normalization < 0) return false;
  if (f[4].rfind("shape=", 0) != 0 || f[5].rfind("axes=", 0) != 0 || f[6].rfind("batch=", 0) != 0)
    return false;
  std::vector<uint64_t> axes, batch;
  if (!parse_u64_list(f[4].substr(6), c.shape) || !parse_u64_list(f[5].substr(5), axes) ||
      !parse_u64_list(f[6].substr(6), batch) || batch.size() != 1)
    return false;
  c.axes.clear();
  for (uint64_t a : axes) c.axes.push_back((uint32_t)a);
  c.batch = batch[0];
  return config_key(c, kind) == key;
}

uint64_t fnv1a(const std::string& s) {
  uint64_t h = 1469598103934665603ull;
  for (unsigned char ch : s) {
    h ^= ch;
    h *= 1099511628211ull;
  }
  return h;
}

std::string json_escape(const std::string& s) {
  std::string o;
  for (char ch : s) {
    if (ch == '"' || ch == '\\') o += '\\';
    o += ch;
  }
  return o;
}

std::string fmt_double(double v) {
  char b[64];
  std::snprintf(b, sizeof(b), "%.3f", v);
  return b;
}

// The canonical text of the entries array (also what the checksum covers).
std::string entries_json(const std::map<std::string, Entry>& m) {
  std::ostringstream os;
  os << "[";
  bool first = true;
  for (const auto& kv : m) {
    os << (first ? "" : ",") << "\n    {\"key\": \"" << json_escape(kv.first)
       << "\", \"lines_per_block\": " << kv.second.lines_per_block
       << ", \"threads_per_block\": " << kv.second.threads_per_block
       << ", \"twiddle_table\": " << kv.second.twiddle_table
       << ", \"radix_order\": " << kv.second.radix_order
       << ", \"best_us\": " << fmt_double(kv.second.best_us)
       << ", \"default_us\": " << fmt_double(kv.second.default_us) << "}";
    first = false;
  }
  os << (m.empty() ? "]" : "\n  ]");
  return os.str();
}

std::string checksum_hex(const std::string& s) {
  char b[32];
  std::snprintf(b, sizeof(b), "%016llx", (unsigned long long)fnv1a(s));
  return b;
}

std::string snapshot_json_locked() {
  const std::string entries = entries_json(g_entries);
  std::ostringstream os;
  // the checksum covers the device and the canonical entries
  os << "{\n  \"schema\": \"" << kSchema << "\",\n  \"version\": " << kVersion
     << ",\n  \"library\": \"" << json_escape(b2f_version()) << "\",\n  \"device\": \""
     << json_escape(g_device) << "\",\n  \"entries\": " << entries << ",\n  \"checksum\": \""
     << checksum_hex(g_device + "\n" + entries) << "\"\n}\n";
  return os.str();
}

// ------------------------------------------------------------ a small JSON reader
struct JVal {
  enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
  double num = 0;
  bool b = false;
  std::string str;
  std::vector<JVal> arr;
  std::vector<std::pair<std::string, JVal>> obj;
  const JVal* get(const std::string& k) const {
    for (const auto& kv : obj)
      if (kv.first == k) return &kv.second;
    return nullptr;
  }
};

struct JParser {
  const std::string& s;
  size_t i = 0;
  std::string err;
  explicit JParser(const std::string& t) : s(t) {}
  void ws() {
    while (i < s.size() && (s[i] == ' ' || s[i] == '\n' || s[i] == '\r' || s[i] == '\t')) ++i;
  }
  bool fail_at(const char* what) {
    if (err.empty()) err = std::string(what) + " at offset " + std::to_string(i);
    return false;
  }
  bool str(std::string& out) {
    if (i >= s.size() || s[i] != '"') return fail_at("expected a string");
    ++i;
    out.clear();
    while (i < s.size() && s[i] != '"') {
      char ch = s[i++];
      if (ch == '\\') {
        if (i >= s.size()) return fail_at("unterminated escape");
        const char e = s[i++];
        if (e == '"' || e == '\\' || e == '/') ch = e;
        else if (e == 'n') ch = '\n';
        else if (e == 't') ch = '\t';
        else return fail_at("unsupported escape");
      }
      out += ch;
    }
    if (i >= s.size()) return fail_at("unterminated string");
    ++i;
    return true;
  }
  bool value(JVal& v, int depth) {
    if (depth > 16) return fail_at("nesting too deep");
    ws();
    if (i >= s.size()) return fail_at("unexpected end");
    const char c = s[i];
    if (c == '{') {
      v.kind = JVal::OBJ;
      ++i;
      ws();
      if (i < s.size() && s[i] == '}') { ++i; return true; }
      while (true) {
        ws();
        std::string k;
        if (!str(k)) return false;
        ws();
        if (i >= s.size() || s[i] != ':') return fail_at("expected ':'");
        ++i;
        JVal sub;
        if (!value(sub, depth + 1)) return false;
        v.obj.emplace_back(k, std::move(sub));
        ws();
        if (i < s.size() && s[i] == ',') { ++i; continue; }
        if (i < s.size() && s[i] == '}') { ++i; return true; }
        return fail_at("expected ',' or '}'");
      }
    }
    if (c == '[') {
      v.kind = JVal::ARR;
      ++i;
      ws();
      if (i < s.size() && s[i] == ']') { ++i; return true; }
      while (true) {
        JVal sub;
        if (!value(sub, depth + 1)) return false;
        v.arr.push_back(std::move(sub));
        ws();
        if (i < s.size() && s[i] == ',') { ++i; continue; }
        if (i < s.size() && s[i] == ']') { ++i; return true; }
        return fail_at("expected ',' or ']'");
      }
    }
    if (c == '"') {
      v.kind = JVal::STR;
      return str(v.str);
    }
    if (s.compare(i, 4, "true") == 0) { v.kind = JVal::BOOL; v.b = true; i += 4; return true; }
    if (s.compare(i, 5, "false") == 0) { v.kind = JVal::BOOL; i += 5; return true; }
    if (s.compare(i, 4, "null") == 0) { v.kind = JVal::NUL; i += 4; return true; }
    const size_t st = i;
    while (i < s.size() && std::strchr("+-0123456789.eE", s[i])) ++i;
    if (st == i) return fail_at("unexpected character");
    v.kind = JVal::NUM;
    try {
      v.num = std::stod(s.substr(st, i - st));
    } catch (...) {
      return fail_at("bad number");
    }
    return true;
  }
};

bool as_int(const JVal* v, int64_t& out) {
  if (!v || v->kind != JVal::NUM || v->num != std::floor(v->num) || std::fabs(v->num) > 9e15)
    return false;
  out = (int64_t)v->num;
  return true;
}

// Parses and checks a snapshot document; on success fills m and dev.
b2f_status parse_snapshot(const std::string& text, std::map<std::string, Entry>& m, std::string& dev) {
  JParser p(text);
  JVal root;
  if (!p.value(root, 0)) return fail(B2F_ERR_SNAPSHOT_JSON, "invalid tuning snapshot JSON: " + p.err);
  p.ws();
  if (p.i != text.size()) return fail(B2F_ERR_SNAPSHOT_JSON, "invalid tuning snapshot JSON: trailing data");
  if (root.kind != JVal::OBJ) return fail(B2F_ERR_SNAPSHOT_JSON, "invalid tuning snapshot JSON: not an object");
  for (const auto& kv : root.obj)
    if (kv.first != "schema" && kv.first != "version" && kv.first != "library" &&
        kv.first != "device" && kv.first != "entries" && kv.first != "checksum")
      return fail(B2F_ERR_SNAPSHOT_JSON, "invalid tuning snapshot JSON: unknown field " + kv.first);
  const JVal* schema = root.get("schema");
  if (!schema || schema->kind != JVal::STR || schema->str != kSchema)
    return fail(B2F_ERR_SNAPSHOT_SCHEMA,
                std::string("tuning snapshot schema mismatch: expected \"") + kSchema + "\", got " +
                    (schema && schema->kind == JVal::STR ? "\"" + schema->str + "\"" : "none"));
  int64_t version = -1;
  if (!as_int(root.get("version"), version) || version != kVersion)
    return fail(B2F_ERR_SNAPSHOT_VERSION, "tuning snapshot version mismatch: expected " +
                                              std::to_string(kVersion) + ", got " +
                                              std::to_string(version));
  const JVal* device = root.get("device");
  const JVal* entries = root.get("entries");
  const JVal* checksum = root.get("checksum");
  if (!device || device->kind != JVal::STR || !entries || entries->kind != JVal::ARR || !checksum ||
      checksum->kind != JVal::STR)
    return fail(B2F_ERR_SNAPSHOT_JSON, "invalid tuning snapshot JSON: missing device, entries or checksum");
  m.clear();
  std::string prev;
  for (const JVal& e : entries->arr) {
    const JVal* key = e.get("key");
    if (e.kind != JVal::OBJ || !key || key->kind != JVal::STR)
      return fail(B2F_ERR_SNAPSHOT_INTEGRITY, "tuning snapshot integrity check failed: entry without a key");
    Config c;
    int32_t kind = 0;
    if (!parse_key(key->str, c, kind))
      return fail(B2F_ERR_SNAPSHOT_INTEGRITY,
                  "tuning snapshot integrity check failed: key is not canonical: " + key->str);
    if (!prev.empty() && key->str <= prev)
      return fail(B2F_ERR_SNAPSHOT_INTEGRITY,
                  "tuning snapshot integrity check failed: duplicate or unordered key " + key->str);
    prev = key->str;
    Entry en;
    if (!as_int(e.get("lines_per_block"), en.lines_per_block) ||
        !as_int(e.get("threads_per_block"), en.threads_per_block) ||
        !as_int(e.get("twiddle_table"), en.twiddle_table) ||
        !as_int(e.get("radix_order"), en.radix_order))
      return fail(B2F_ERR_SNAPSHOT_INTEGRITY,
                  "tuning snapshot integrity check failed: bad tuning values for " + key->str);
    const JVal* bu = e.get("best_us");
    const JVal* du = e.get("default_us");
    if (!bu || bu->kind != JVal::NUM || !du || du->kind != JVal::NUM)
      return fail(B2F_ERR_SNAPSHOT_INTEGRITY,
                  "tuning snapshot integrity check failed: missing timings for " + key->str);
    en.best_us = bu->num;
    en.default_us = du->num;
    c.tuning.lines_per_block = en.lines_per_block;
    c.tuning.threads_per_block = en.threads_per_block;
    c.tuning.twiddle_table = en.twiddle_table;
    c.tuning.radix_order = en.radix_order;
    if (en.twiddle_table != 0 && en.twiddle_table != 1)
      return fail(B2F_ERR_SNAPSHOT_INTEGRITY,
                  "tuning snapshot integrity check failed: twiddle_table must be 0 or 1 for " + key->str);
    if (validate_config(c) != B2F_OK)
      return fail(B2F_ERR_SNAPSHOT_INTEGRITY, "tuning snapshot integrity check failed: " + last_error());
    m[key->str] = en;
  }
  if (checksum->str != checksum_hex(device->str + "\n" + entries_json(m)))
    return fail(B2F_ERR_SNAPSHOT_INTEGRITY,
                "tuning snapshot integrity check failed: checksum does not match the entries");
  dev = device->str;
  return B2F_OK;
}

std::string device_name(int device) {
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return "unknown";
  return std::string(prop.name) + " sm_" + std::to_string(prop.major) + std::to_string(prop.minor);
}

// ------------------------------------------------------------------ autotuner
// Deterministic inputs in [-1, 1): f32 / f64 values, df64 as (hi, 0) pairs.
void fill_input(std::vector<unsigned char>& buf, int32_t precision) {
  uint64_t s = 0x9E3779B97F4A7C15ull;
  auto next = [&]() {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return (double)(s >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
  };
  if (precision == B2F_F64) {
    double* d = reinterpret_cast<double*>(buf.data());
    for (size_t i = 0; i < buf.size() / 8; ++i) d[i] = next();
  } else if (precision == B2F_DF64) {
    float* f = reinterpret_cast<float*>(buf.data());
    for (size_t i = 0; i + 1 < buf.size() / 4; i += 2) {
      f[i] = (float)next();
      f[i + 1] = 0.0f;
    }
  } else {
    float* f = reinterpret_cast<float*>(buf.data());
    for (size_t i = 0; i < buf.size() / 4; ++i) f[i] = (float)next();
  }
}

// Relative L2 distance of two outputs, read as the precision's values.
double rel_l2(const std::vector<unsigned char>& a, const std::vector<unsigned char>& b,
              int32_t precision) {
  double num = 0, den = 0;
  if (precision == B2F_F64) {
    const double* x = reinterpret_cast<const double*>(a.data());
    const double* y = reinterpret_cast<const double*>(b.data());
    for (size_t i = 0; i < a.size() / 8; ++i) {
      num += (x[i] - y[i]) * (x[i] - y[i]);
      den += y[i] * y[i];
    }
  } else if (precision == B2F_DF64) {
    const float* x = reinterpret_cast<const float*>(a.data());
    const float* y = reinterpret_cast<const float*>(b.data());
    for (size_t i = 0; i + 1 < a.size() / 4; i += 2) {
      const double u = (double)x[i] + (double)x[i + 1], v = (double)y[i] + (double)y[i + 1];
      num += (u - v) * (u - v);
      den += v * v;
    }
  } else {
    const float* x = reinterpret_cast<const float*>(a.data());
    const float* y = reinterpret_cast<const float*>(b.data());
    for (size_t i = 0; i < a.size() / 4; ++i) {
      num += ((double)x[i] - y[i]) * ((double)x[i] - y[i]);
      den += (double)y[i] * y[i];
    }
  }
  return den > 0 ? std::sqrt(num / den) : std::sqrt(num);
}

struct Candidate {
  int64_t lpb, tpb, tt, ro;
  double us = -1;
  double err = 0;
  bool ok = false;
  std::string why;
};

}  // namespace

// Runs the autotuner for one configuration; report receives a JSON object.
b2f_status autotune(const Config& base, int32_t kind, int device, uint32_t reps,
                    std::string& report) {
  b2f_status st = validate_config(base);
  if (st) return st;
  if (reps == 0) reps = 20;
  int prev = -1;
  cudaGetDevice(&prev);
  if (device < 0) device = prev < 0 ? 0 : prev;
  if (cudaSetDevice(device) != cudaSuccess) return fail(B2F_ERR_DEVICE, "cudaSetDevice failed");
  Plan* p0 = nullptr;
  st = create_plan(base, kind, device, &p0);
  if (st) {
    if (prev >= 0) cudaSetDevice(prev);
    return st;
  }
  const uint64_t in_bytes = p0->in_bytes, out_bytes = p0->out_bytes;
  void *din = nullptr, *dout = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  bool ok = cudaMalloc(&din, in_bytes) == cudaSuccess && cudaMalloc(&dout, out_bytes) == cudaSuccess &&
            cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess;
  std::vector<unsigned char> host_in(in_bytes), ref(out_bytes), got(out_bytes);
  auto cleanup = [&]() {
    cudaFree(din);
    cudaFree(dout);
    if (stream) cudaStreamDestroy(stream);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (prev >= 0) cudaSetDevice(prev);
  };
  if (!ok) {
    delete p0;
    cleanup();
    return fail(B2F_ERR_RESOURCE_ALLOCATION, "autotune buffer allocation failed");
  }
  fill_input(host_in, base.precision);
  cudaMemcpy(din, host_in.data(), in_bytes, cudaMemcpyHostToDevice);
  // times one plan: 2 warm-up runs, then reps runs between two events
  auto time_plan = [&](const Plan& plan, double& us, std::vector<unsigned char>& out) -> b2f_status {
    for (int w = 0; w < 2; ++w) {
      b2f_status s = execute_plan(plan, stream, din, in_bytes, dout, out_bytes);
      if (s) return s;
    }
    cudaEventRecord(e0, stream);
    for (uint32_t r = 0; r < reps; ++r) {
      b2f_status s = execute_plan(plan, stream, din, in_bytes, dout, out_bytes);
      if (s) return s;
    }
    cudaEventRecord(e1, stream);
    if (cudaStreamSynchronize(stream) != cudaSuccess)
      return fail(B2F_ERR_DEVICE, "autotune: stream synchronisation failed");
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    us = 1e3 * ms / reps;
    if (cudaMemcpy(out.data(), dout, out_bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
      return fail(B2F_ERR_DEVICE, "autotune: output copy failed");
    return B2F_OK;
  };
  double default_us = 0;
  st = time_plan(*p0, default_us, ref);
  delete p0;
  if (st) {
    cleanup();
    return st;
  }
  const double tol = base.precision == B2F_F32 ? 2e-6 : (base.precision == B2F_F64 ? 1e-13 : 1e-12);
  std::vector<Candidate> tried;
  Candidate best{base.tuning.lines_per_block, base.tuning.threads_per_block,
                 base.tuning.twiddle_table, base.tuning.radix_order, default_us, 0.0, true,
                 "default"};
  auto run = [&](int64_t lpb, int64_t tpb, int64_t tt, int64_t ro) {
    for (const auto& c : tried)
      if (c.lpb == lpb && c.tpb == tpb && c.tt == tt && c.ro == ro) return;
    Candidate c{lpb, tpb, tt, ro};
    Config cfg = base;
    cfg.tuning.lines_per_block = lpb;
    cfg.tuning.threads_per_block = tpb;
    cfg.tuning.twiddle_table = tt;
    cfg.tuning.radix_order = ro;
    Plan* pl = nullptr;
    if (create_plan(cfg, kind, device, &pl) != B2F_OK) {
      c.why = last_error();
    } else {
      double us = 0;
      if (time_plan(*pl, us, got) != B2F_OK) {
        c.why = last_error();
      } else {
        c.us = us;
        c.err = rel_l2(got, ref, base.precision);
        c.ok = c.err <= tol;
        if (!c.ok) c.why = "result differs from the default plan";
      }
      delete pl;
    }
    if (c.ok && c.us < best.us) best = c;
    tried.push_back(c);
  };
  // staged search: twiddle source, then radix order, then lines per block,
  // then threads per block
  for (int64_t tt : {1, 0}) run(0, 0, tt, 0);
  const int64_t tt_best = best.tt;
  run(0, 0, tt_best, 1);
  const int64_t ro_best = best.ro;
  for (int64_t lpb : {1, 2, 4, 8, 16}) run(lpb, 0, tt_best, ro_best);
  const int64_t lpb_best = best.lpb;
  for (int64_t tpb : {64, 128, 256, 512}) run(lpb_best, tpb, tt_best, ro_best);
  cudaGetLastError();
  cleanup();
  const std::string key = config_key(base, kind);
  {
    std::lock_guard<std::mutex> lk(g_mu);
    const std::string dev = device_name(device);
    if (!g_device.empty() && g_device != dev) g_entries.clear();
    g_device = dev;
    Entry& en = g_entries[key];
    en.lines_per_block = best.lpb;
    en.threads_per_block = best.tpb;
    en.twiddle_table = best.tt;
    en.radix_order = best.ro;
    en.best_us = best.us;
    en.default_us = default_us;
  }
  std::ostringstream os;
  os << "{\"key\":\"" << json_escape(key) << "\",\"default_us\":" << fmt_double(default_us)
     << ",\"best_us\":" << fmt_double(best.us) << ",\"best\":{\"lines_per_block\":" << best.lpb
     << ",\"threads_per_block\":" << best.tpb << ",\"twiddle_table\":" << best.tt
     << ",\"radix_order\":" << best.ro << "},\"candidates\":[";
  for (size_t i = 0; i < tried.size(); ++i) {
    const Candidate& c = tried[i];
    os << (i ? "," : "") << "{\"lines_per_block\":" << c.lpb << ",\"threads_per_block\":" << c.tpb
       << ",\"twiddle_table\":" << c.tt << ",\"radix_order\":" << c.ro << ",\"us\":" << fmt_double(c.us) << ",\"rel_l2\":" << c.err
       << ",\"ok\":" << (c.ok ? "true" : "false") << ",\"note\":\"" << json_escape(c.why) << "\"}";
  }
  os << "]}";
  report = os.str();
  return B2F_OK;
}

}  // namespace b2f

using namespace b2f;

static b2f_status copy_out(const std::string& s, char* buf, uint64_t* len) {
  const uint64_t cap = *len;
  *len = s.size();
  if (buf && cap > 0) {
    const uint64_t n = std::min<uint64_t>(cap - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
    if (n < s.size()) return fail(B2F_ERR_BUFFER_TOO_SMALL, "buffer too small");
  }
  return B2F_OK;
}

extern "C" {

b2f_status b2f_autotune(const b2f_config* cfg, int32_t kind, int32_t device, uint32_t reps,
                        char* report, uint64_t* len) {
  if (!cfg || !len) return fail(B2F_ERR_INVALID_ARGUMENT, "null argument");
  if (kind < B2F_C2C || kind > B2F_C2R) return fail(B2F_ERR_INVALID_ARGUMENT, "kind must be 0..=2");
  std::string rep;
  const b2f_status st = autotune(cfg->cfg, kind, device, reps, rep);
  if (st) return st;
  return copy_out(rep, report, len);
}

b2f_status b2f_tuning_snapshot_record(const b2f_config* cfg, int32_t kind, int64_t lines_per_block,
                                      int64_t threads_per_block, int64_t twiddle_table,
                                      int64_t radix_order, double best_us, double default_us) {
  if (!cfg) return fail(B2F_ERR_INVALID_ARGUMENT, "null config");
  if (kind < B2F_C2C || kind > B2F_C2R) return fail(B2F_ERR_INVALID_ARGUMENT, "kind must be 0..=2");
  Config c = cfg->cfg;
  c.tuning.lines_per_block = lines_per_block;
  c.tuning.threads_per_block = threads_per_block;
  c.tuning.twiddle_table = twiddle_table;
  c.tuning.radix_order = radix_order;
  if (twiddle_table != 0 && twiddle_table != 1)
    return fail(B2F_ERR_INVALID_TUNING, "InvalidTuning { field: twiddle_table }: must be 0 or 1");
  const b2f_status st = validate_config(c);
  if (st) return st;
  std::lock_guard<std::mutex> lk(g_mu);
  Entry& en = g_entries[config_key(c, kind)];
  en.lines_per_block = lines_per_block;
  en.threads_per_block = threads_per_block;
  en.twiddle_table = twiddle_table;
  en.radix_order = radix_order;
  en.best_us = best_us;
  en.default_us = default_us;
  return B2F_OK;
}

b2f_status b2f_tuning_snapshot_apply(b2f_config* cfg, int32_t kind, int32_t* found) {
  if (!cfg || !found) return fail(B2F_ERR_INVALID_ARGUMENT, "null argument");
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_entries.find(config_key(cfg->cfg, kind));
  *found = it != g_entries.end();
  if (*found) {
    cfg->cfg.tuning.lines_per_block = it->second.lines_per_block;
    cfg->cfg.tuning.threads_per_block = it->second.threads_per_block;
    cfg->cfg.tuning.twiddle_table = it->second.twiddle_table;
    cfg->cfg.tuning.radix_order = it->second.radix_order;
  }
  return B2F_OK;
}

b2f_status b2f_tuning_snapshot_json(char* buf, uint64_t* len) {
  if (!len) return fail(B2F_ERR_INVALID_ARGUMENT, "null argument");
  std::string s;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    s = snapshot_json_locked();
  }
  return copy_out(s, buf, len);
}

b2f_status b2f_tuning_snapshot_save(const char* path) {
  if (!path) return fail(B2F_ERR_INVALID_ARGUMENT, "null path");
  std::string s;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    s = snapshot_json_locked();
  }
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) return fail(B2F_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path + " for writing");
  f << s;
  if (!f) return fail(B2F_ERR_INVALID_ARGUMENT, std::string("cannot write ") + path);
  return B2F_OK;
}

b2f_status b2f_tuning_snapshot_load(const char* path, int32_t device) {
  if (!path) return fail(B2F_ERR_INVALID_ARGUMENT, "null path");
  std::ifstream f(path, std::ios::binary);
  if (!f) return fail(B2F_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
  std::stringstream ss;
  ss << f.rdbuf();
  std::map<std::string, Entry> m;
  std::string dev;
  const b2f_status st = parse_snapshot(ss.str(), m, dev);
  if (st) return st;
  // entries recorded by hand carry no device and apply anywhere
  if (device >= 0 && !m.empty() && !dev.empty()) {
    const std::string here = device_name(device);
    if (dev != here)
      return fail(B2F_ERR_SNAPSHOT_INTEGRITY, "tuning snapshot integrity check failed: tuned on \"" +
                                                  dev + "\", this device is \"" + here + "\"");
  }
  std::lock_guard<std::mutex> lk(g_mu);
  g_entries.swap(m);
  g_device = dev;
  return B2F_OK;
}

void b2f_tuning_snapshot_clear(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_entries.clear();
  g_device.clear();
}

}  // extern "C"
