// df64 backend canary (b2f_df64_canary): the counterpart of the crate's
// validate_df64_invariants (src/df64_canary.rs).  The df64 route is only as
// accurate as its error-free transforms (two-sum, quick-two-sum, the FMA
// two-product and the df64 add/multiply built from them), and a compiler
// that contracts or reassociates them keeps ordinary round trips plausible
// while breaking the last bits.  The canary evaluates every transform the
// df64 kernels use on adversarial inputs on the device, with the device
// functions of cplx.cuh, and compares each f32 word bit for bit with the
// same transforms evaluated on the host in IEEE single precision.
#include <cmath>
#include <cstring>
#include <sstream>

#include "plan.h"

namespace b2f {

constexpr int kCanaryCases = 4;
constexpr int kCanaryWords = 22;  // f32 words per case

// Adversarial inputs (the crate's canary_inputs, src/df64_canary.rs):
// cancellation at 2^24, ulp-level neighbours of 1, extreme exponents and
// mixed magnitudes; per case a = (x, y, z, w) and b = (x, y, z, w).
static void canary_inputs(float in[kCanaryCases][2][4]) {
  auto f = [](uint32_t bits) {
    float v;
    std::memcpy(&v, &bits, 4);
    return v;
  };
  const float c[kCanaryCases][2][4] = {
      {{16777216.0f, 1.0f, 16777216.0f, 4097.0f}, {-16777216.0f, 1.0f, 1.0f, 4097.0f}},
      {{1.0f, f(0x33800000u), 1.0000001f, 1.0000001f}, {-1.0f, f(0x33000000u), -1.0f, 0.9999999f}},
      {{1.0e36f, 1.0e28f, 1.0e20f, f(0x7b4097ceu)}, {1.0e-30f, 1.0e-37f, 1.0f, f(0x0da24260u)}},
      {{-12345.125f, 0.00012207031f, -33554432.0f, -17.25f},
       {0.03125763f, -1.0e-10f, 3.0f, 3.0000002f}},
  };
  std::memcpy(in, c, sizeof(c));
}

// ---- host restatement in IEEE single precision (explicit fmaf where the
// device uses a fused multiply-add, plain operations elsewhere)
struct hdf {
  float hi, lo;
};
static hdf h_two_sum(float a, float b) {
  const float s = a + b;
  const float bb = s - a;
  const float e = (a - (s - bb)) + (b - bb);
  return {s, e};
}
static hdf h_quick_two_sum(float a, float b) {
  const float s = a + b;
  return {s, b - (s - a)};
}
static hdf h_two_prod(float a, float b) {
  const float p = a * b;
  return {p, std::fmaf(a, b, -p)};
}
static hdf h_add(hdf a, hdf b) {
  const hdf s = h_two_sum(a.hi, b.hi);
  const hdf t = h_two_sum(a.lo, b.lo);
  float e = s.lo + t.hi;
  const hdf u = h_quick_two_sum(s.hi, e);
  e = u.lo + t.lo;
  return h_quick_two_sum(u.hi, e);
}
static hdf h_neg(hdf a) { return {-a.hi, -a.lo}; }
static hdf h_mul(hdf a, hdf b) {
  const float p = a.hi * b.hi;
  float e = std::fmaf(a.hi, b.hi, -p);
  e = std::fmaf(a.hi, b.lo, e);
  e = std::fmaf(a.lo, b.hi, e);
  return h_quick_two_sum(p, e);
}

static void host_words(const float a[4], const float b[4], uint32_t out[kCanaryWords]) {
  hdf w[kCanaryWords / 2];
  w[0] = h_two_sum(a[0], b[0]);
  w[1] = h_quick_two_sum(a[2], b[2]);
  w[2] = h_two_prod(a[3], b[3]);
  const hdf ad = {a[0], a[1]}, bd = {b[0], b[1]};
  w[3] = h_add(ad, bd);
  w[4] = h_mul(ad, bd);
  // complex values (re = (x, y), im = (z, w))
  const hdf are = {a[0], a[1]}, aim = {a[2], a[3]}, bre = {b[0], b[1]}, bim = {b[2], b[3]};
  w[5] = h_add(are, bre);
  w[6] = h_add(aim, bim);
  w[7] = h_add(h_mul(are, bre), h_neg(h_mul(aim, bim)));
  w[8] = h_add(h_mul(are, bim), h_mul(aim, bre));
  float big, tiny;
  const uint32_t bb = 0x7f7fffffu, tb = 0x00800000u;
  std::memcpy(&big, &bb, 4);
  std::memcpy(&tiny, &tb, 4);
  w[9] = h_two_prod(big, tiny);
  float c0, c1;
  const uint32_t cb0 = 0x3cf0f0f1u, cb1 = 0xaef0f0f1u, lb = 0x30800000u;
  std::memcpy(&c0, &cb0, 4);
  std::memcpy(&c1, &cb1, 4);
  float l0;
  std::memcpy(&l0, &lb, 4);
  w[10] = h_mul({1.0f, l0}, {c0, c1});
  for (int i = 0; i < kCanaryWords / 2; ++i) {
    std::memcpy(&out[2 * i], &w[i].hi, 4);
    std::memcpy(&out[2 * i + 1], &w[i].lo, 4);
  }
}

// ---- device side: the df64 route's own functions (cplx.cuh)
__global__ void k_df64_canary(const float4* __restrict__ in, uint32_t* __restrict__ out) {
  const int c = threadIdx.x;
  if (c >= kCanaryCases) return;
  const float4 a = in[2 * c], b = in[2 * c + 1];
  df w[kCanaryWords / 2];
  w[0] = df_two_sum(a.x, b.x);
  w[1] = df_quick_two_sum(a.z, b.z);
  {
    const float p = __fmul_rn(a.w, b.w);
    w[2] = {p, __fmaf_rn(a.w, b.w, -p)};
  }
  const df ad = {a.x, a.y}, bd = {b.x, b.y};
  w[3] = ad + bd;
  w[4] = ad * bd;
  const cdf ac = {{a.x, a.y}, {a.z, a.w}}, bc = {{b.x, b.y}, {b.z, b.w}};
  const cdf s = ac + bc;
  const cdf m = cmul(ac, bc);
  w[5] = s.re;
  w[6] = s.im;
  w[7] = m.re;
  w[8] = m.im;
  {
    const float big = __uint_as_float(0x7f7fffffu), tiny = __uint_as_float(0x00800000u);
    const float p = __fmul_rn(big, tiny);
    w[9] = {p, __fmaf_rn(big, tiny, -p)};
  }
  w[10] = df{1.0f, __uint_as_float(0x30800000u)} *
          df{__uint_as_float(0x3cf0f0f1u), __uint_as_float(0xaef0f0f1u)};
  for (int i = 0; i < kCanaryWords / 2; ++i) {
    out[c * kCanaryWords + 2 * i] = __float_as_uint(w[i].hi);
    out[c * kCanaryWords + 2 * i + 1] = __float_as_uint(w[i].lo);
  }
}

}  // namespace b2f

using namespace b2f;

extern "C" b2f_status b2f_df64_canary(int32_t device, uint32_t* words, uint64_t* exact_words) {
  float in[kCanaryCases][2][4];
  canary_inputs(in);
  uint32_t expect[kCanaryCases * kCanaryWords];
  for (int c = 0; c < kCanaryCases; ++c) host_words(in[c][0], in[c][1], expect + c * kCanaryWords);
  int prev = -1;
  cudaGetDevice(&prev);
  if (device >= 0 && cudaSetDevice(device) != cudaSuccess)
    return fail(B2F_ERR_DEVICE, "cudaSetDevice failed");
  void* d_in = nullptr;
  void* d_out = nullptr;
  uint32_t got[kCanaryCases * kCanaryWords];
  cudaError_t e = cudaMalloc(&d_in, sizeof(in));
  if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(got));
  if (e == cudaSuccess) e = cudaMemcpy(d_in, in, sizeof(in), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_df64_canary<<<1, 32>>>((const float4*)d_in, (uint32_t*)d_out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(got, d_out, sizeof(got), cudaMemcpyDeviceToHost);
  if (d_in) cudaFree(d_in);
  if (d_out) cudaFree(d_out);
  if (prev >= 0) cudaSetDevice(prev);
  if (e != cudaSuccess)
    return fail(B2F_ERR_DEVICE, std::string("df64 canary execution failed: ") + cudaGetErrorString(e));
  if (words) std::memcpy(words, got, sizeof(got));
  uint64_t exact = 0;
  for (int i = 0; i < kCanaryCases * kCanaryWords; ++i) {
    if (got[i] != expect[i]) {
      if (exact_words) *exact_words = exact;
      std::ostringstream os;
      os << std::hex << "InvariantMismatch { case: " << std::dec << i / kCanaryWords
         << ", word: " << i % kCanaryWords << ", actual: 0x" << std::hex << got[i]
         << ", expected: 0x" << expect[i]
         << " } (a compiler contraction or reassociation broke an error-free transform)";
      return fail(B2F_ERR_DEVICE, os.str());
    }
    ++exact;
  }
  if (exact_words) *exact_words = exact;
  return B2F_OK;
}
