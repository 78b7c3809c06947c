// Complex arithmetic for the three storage precisions of the transform path:
//   f32  : {float re, im}                     8 bytes, interleaved [re, im]
//   f64  : {double re, im}                   16 bytes, interleaved [re, im]
//   df64 : {float re_hi, re_lo, im_hi, im_lo} 16 bytes (an unevaluated
//          hi + lo pair of f32 words per component, the reference crate's
//          Df64 storage order, src/math/double_float.rs:57-66).
// The df64 operations are the error-free transforms (two-sum, quick-two-sum,
// two-product through a fused multiply-add) written with the _rn intrinsics,
// which the compiler never contracts or reassociates.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "dft_consts.h"

#define FFT_HD __host__ __device__ __forceinline__
#define FFT_D __device__ __forceinline__

// ---------------------------------------------------------------- df64 scalar
struct df {
  float hi, lo;
};

FFT_D df df_two_sum(float a, float b) {
  float s = __fadd_rn(a, b);
  float bb = __fsub_rn(s, a);
  float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  return {s, e};
}

FFT_D df df_quick_two_sum(float a, float b) {
  float s = __fadd_rn(a, b);
  float e = __fsub_rn(b, __fsub_rn(s, a));
  return {s, e};
}

FFT_D df operator+(df a, df b) {
  df s = df_two_sum(a.hi, b.hi);
  df t = df_two_sum(a.lo, b.lo);
  float e = __fadd_rn(s.lo, t.hi);
  df u = df_quick_two_sum(s.hi, e);
  e = __fadd_rn(u.lo, t.lo);
  return df_quick_two_sum(u.hi, e);
}

FFT_D df operator-(df a) { return {-a.hi, -a.lo}; }
FFT_D df operator-(df a, df b) { return a + (-b); }

FFT_D df operator*(df a, df b) {
  float p = __fmul_rn(a.hi, b.hi);
  float e = __fmaf_rn(a.hi, b.hi, -p);
  e = __fmaf_rn(a.hi, b.lo, e);
  e = __fmaf_rn(a.lo, b.hi, e);
  return df_quick_two_sum(p, e);
}

FFT_D df df_from_double(double v) {
  float hi = __double2float_rn(v);
  float lo = __double2float_rn(v - (double)hi);
  return {hi, lo};
}

FFT_D double df_to_double(df v) { return (double)v.hi + (double)v.lo; }

// Multiplication by a small exact power of two (scale factors, halves).
FFT_D df df_mul_f(df a, float f) {
  float p = __fmul_rn(a.hi, f);
  float e = __fmaf_rn(a.hi, f, -p);
  e = __fmaf_rn(a.lo, f, e);
  return df_quick_two_sum(p, e);
}

// ------------------------------------------------------------ scalar traits
template <class S>
struct Scalar;

template <>
struct Scalar<float> {
  static FFT_D float from_double(double v) { return (float)v; }
  static FFT_D float zero() { return 0.0f; }
  static FFT_D float mul_small(float a, double f) { return a * (float)f; }
};

template <>
struct Scalar<double> {
  static FFT_D double from_double(double v) { return v; }
  static FFT_D double zero() { return 0.0; }
  static FFT_D double mul_small(double a, double f) { return a * f; }
};

template <>
struct Scalar<df> {
  static FFT_D df from_double(double v) { return df_from_double(v); }
  static FFT_D df zero() { return {0.0f, 0.0f}; }
  static FFT_D df mul_small(df a, double f) { return a * df_from_double(f); }
};

// ------------------------------------------------------------------ complex
template <class S>
struct alignas(2 * sizeof(S)) cpx {
  S re, im;
};

using c32 = cpx<float>;
using c64 = cpx<double>;
using cdf = cpx<df>;

template <class S>
FFT_D cpx<S> operator+(cpx<S> a, cpx<S> b) {
  return {a.re + b.re, a.im + b.im};
}
template <class S>
FFT_D cpx<S> operator-(cpx<S> a, cpx<S> b) {
  return {a.re - b.re, a.im - b.im};
}
template <class S>
FFT_D cpx<S> cmul(cpx<S> a, cpx<S> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}

// a * conj(b)
template <class S>
FFT_D cpx<S> cmulc(cpx<S> a, cpx<S> b) {
  return {a.re * b.re + a.im * b.im, a.im * b.re - a.re * b.im};
}
template <class S>
FFT_D cpx<S> conj(cpx<S> a) {
  return {a.re, -a.im};
}
// i * a
template <class S>
FFT_D cpx<S> mul_i(cpx<S> a) {
  return {-a.im, a.re};
}
// -i * a
template <class S>
FFT_D cpx<S> mul_neg_i(cpx<S> a) {
  return {a.im, -a.re};
}
template <class S>
FFT_D cpx<S> cscale(cpx<S> a, S s) {
  return {a.re * s, a.im * s};
}
template <class S>
FFT_D cpx<S> czero() {
  return {Scalar<S>::zero(), Scalar<S>::zero()};
}
template <class S>
FFT_D cpx<S> cfrom(double re, double im) {
  return {Scalar<S>::from_double(re), Scalar<S>::from_double(im)};
}

// Scale factor in the working type (f32 scale is computed in f32 as the
// reference does, src/runtime/axis_plan.rs:451-483).
template <class S>
struct ScaleT {
  S s;
};

// Forward root of unity exp(-2*pi*i*m/R) as a compile-time constant pair.
template <class S, int R>
FFT_D cpx<S> root(int m) {
  return cfrom<S>(dft_cos(R, m), -dft_sin(R, m));
}

// --------------------------------------------------------------- twiddles
// exp(-2*pi*i*m/M) for 0 <= m < M in f32, with the angle reduced to the first
// octant in integers (m' = 8m against M, 2M, 4M), then sincospif on an
// argument in [0, 1/4]: the error stays near one ulp for every M.
FFT_D c32 twiddle_f32(uint64_t m, uint64_t M) {
  uint64_t t = 8 * m;                      // angle = (pi/4) * t / M
  bool neg_s = false, neg_c = false, swap = false;
  if (t > 4 * M) { t = 8 * M - t; neg_s = true; }   // angle -> 2pi - angle
  if (t > 2 * M) { t = 4 * M - t; neg_c = true; }   // angle -> pi - angle
  if (t > M) { t = 2 * M - t; swap = true; }        // angle -> pi/2 - angle
  float x;
  if (M <= (1ull << 22)) {
    x = __fdiv_rn((float)t, (float)(4 * M));
  } else {
    x = (float)((double)t / (double)(4 * M));
  }
  float s, c;
  sincospif(x, &s, &c);
  if (swap) { float u = s; s = c; c = u; }
  if (neg_c) c = -c;
  if (neg_s) s = -s;
  return {c, -s};
}

FFT_D c64 twiddle_f64(uint64_t m, uint64_t M) {
  uint64_t t = 8 * m;
  bool neg_s = false, neg_c = false, swap = false;
  if (t > 4 * M) { t = 8 * M - t; neg_s = true; }
  if (t > 2 * M) { t = 4 * M - t; neg_c = true; }
  if (t > M) { t = 2 * M - t; swap = true; }
  double x = (double)t / (double)(4 * M);
  double s, c;
  sincospi(x, &s, &c);
  if (swap) { double u = s; s = c; c = u; }
  if (neg_c) c = -c;
  if (neg_s) s = -s;
  return {c, -s};
}

template <class S>
FFT_D cpx<S> twiddle(uint64_t m, uint64_t M);
template <>
FFT_D c32 twiddle<float>(uint64_t m, uint64_t M) {
  return twiddle_f32(m, M);
}
template <>
FFT_D c64 twiddle<double>(uint64_t m, uint64_t M) {
  return twiddle_f64(m, M);
}
template <>
FFT_D cdf twiddle<df>(uint64_t m, uint64_t M) {
  c64 w = twiddle_f64(m, M);
  return {df_from_double(w.re), df_from_double(w.im)};
}

// ------------------------------------------------------------ fast division
// Unsigned 32-bit division by a runtime constant d, exact for n < 2^31:
// with l = ceil(log2 d) and mul = ceil(2^(31+l) / d) (< 2^32 when d is not a
// power of two), n / d = umulhi(n, mul) >> (l - 1).  Powers of two shift.
struct FastDiv {
  uint32_t d, mul, shift;
};

inline FastDiv make_fastdiv(uint32_t d) {
  FastDiv f{d, 0, 0};
  if (d == 0) return f;
  uint32_t l = 0;
  while ((1ull << l) < d) ++l;
  if ((d & (d - 1)) == 0) {
    f.mul = 0;
    f.shift = l;
    return f;
  }
  unsigned __int128 num = (unsigned __int128)1 << (31 + l);
  uint64_t m = (uint64_t)(num / d) + ((num % d) ? 1 : 0);
  f.mul = (uint32_t)m;
  f.shift = l - 1;
  return f;
}

FFT_D uint32_t fdiv(uint32_t n, const FastDiv& f) {
  if (f.mul == 0) return n >> f.shift;
  return __umulhi(n, f.mul) >> f.shift;
}

// W_M^m (m < M) from a two-level table, m = a*L + b: A[a] * B[b], A[a] =
// W_M^{aL} and B[b] = W_M^b each computed in FP64 and rounded once, so the
// product carries about one more rounding than a single table entry.
// m < 2^31 takes the fast division, larger m a 64-bit one.
template <class S>
FFT_D cpx<S> tw_two_level(const cpx<S>* __restrict__ A, const cpx<S>* __restrict__ B, uint64_t m,
                          const FastDiv& dL) {
  uint32_t a, b;
  if (m < 0x80000000ull) {
    a = fdiv((uint32_t)m, dL);
    b = (uint32_t)m - a * dL.d;
  } else {
    a = (uint32_t)(m / dL.d);
    b = (uint32_t)(m - (uint64_t)a * dL.d);
  }
  return cmul(A[a], B[b]);
}
