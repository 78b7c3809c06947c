// Forward DFT codelets of radix R on R values held in registers, generic over
// the scalar type (float, double, df).  Inverse transforms reuse them through
// conj(DFT(conj(x))) at the line's load and store, so every codelet, table
// and twiddle on the device is a forward one.
//
//   R = 2, 4, 8            : closed-form butterflies;
//   R = 3, 5, 7, 11, 13     : symmetric pairs, X[k] and X[R-k] from the sums
//                             and differences of x[j], x[R-j] (O(R^2/4)
//                             multiplies), the scheme the reference uses for
//                             its odd radices (src/runtime/axis_plan.rs:3079);
//   R = 9, 16              : two nested codelets R = A*B with the
//                             W_R^{n2 k1} twiddles between them as constants.
#pragma once
#include "cplx.cuh"

template <class S, int R>
FFT_D void dft(cpx<S>* v);

// Multiply by the compile-time root exp(-2 pi i m / R); the trivial cases
// (1, -i, -1, i and the eighth roots) fold into adds after unrolling.
template <class S, int R>
FFT_D cpx<S> mul_root(cpx<S> a, int m) {
  m %= R;
  if (m == 0) return a;
  if (4 * m == R) return mul_neg_i(a);
  if (2 * m == R) return {-a.re, -a.im};
  if (4 * m == 3 * R) return mul_i(a);
  if (8 * m == R) {  // (1 - i)/sqrt2
    const S h = Scalar<S>::from_double(0.70710678118654752440);
    return {(a.re + a.im) * h, (a.im - a.re) * h};
  }
  if (8 * m == 3 * R) {  // (-1 - i)/sqrt2
    const S h = Scalar<S>::from_double(0.70710678118654752440);
    return {(a.im - a.re) * h, -(a.re + a.im) * h};
  }
  return cmul(a, root<S, R>(m));
}

template <class S>
FFT_D void dft2(cpx<S>& a, cpx<S>& b) {
  cpx<S> t = a - b;
  a = a + b;
  b = t;
}

template <class S>
struct Dft2 {
  static FFT_D void run(cpx<S>* v) { dft2(v[0], v[1]); }
};

template <class S>
struct Dft4 {
  static FFT_D void run(cpx<S>* v) {
    cpx<S> a0 = v[0] + v[2], a1 = v[0] - v[2];
    cpx<S> a2 = v[1] + v[3], a3 = mul_neg_i(v[1] - v[3]);
    v[0] = a0 + a2;
    v[2] = a0 - a2;
    v[1] = a1 + a3;
    v[3] = a1 - a3;
  }
};

template <class S>
struct Dft8 {
  static FFT_D void run(cpx<S>* v) {
    cpx<S> e[4] = {v[0], v[2], v[4], v[6]};
    cpx<S> o[4] = {v[1], v[3], v[5], v[7]};
    Dft4<S>::run(e);
    Dft4<S>::run(o);
    o[1] = mul_root<S, 8>(o[1], 1);
    o[2] = mul_neg_i(o[2]);
    o[3] = mul_root<S, 8>(o[3], 3);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v[k] = e[k] + o[k];
      v[k + 4] = e[k] - o[k];
    }
  }
};

template <class S, int R>
struct DftOddPrime {
  static FFT_D void run(cpx<S>* v) {
    constexpr int H = (R - 1) / 2;
    cpx<S> s[H + 1], d[H + 1];
#pragma unroll
    for (int j = 1; j <= H; ++j) {
      s[j] = v[j] + v[R - j];
      d[j] = v[j] - v[R - j];
    }
    cpx<S> x0 = v[0];
    cpx<S> sum = x0;
#pragma unroll
    for (int j = 1; j <= H; ++j) sum = sum + s[j];
#pragma unroll
    for (int k = 1; k <= H; ++k) {
      cpx<S> a = x0, b = czero<S>();
#pragma unroll
      for (int j = 1; j <= H; ++j) {
        const S c = Scalar<S>::from_double(dft_cos(R, (j * k) % R));
        const S sn = Scalar<S>::from_double(dft_sin(R, (j * k) % R));
        a = a + cscale(s[j], c);
        b = b + cscale(d[j], sn);
      }
      // forward: X[k] = a - i b, X[R-k] = a + i b
      v[k] = {a.re + b.im, a.im - b.re};
      v[R - k] = {a.re - b.im, a.im + b.re};
    }
    v[0] = sum;
  }
};

// R = A * B: input n = B*n1 + n2, output k = k1 + A*k2.
template <class S, int A, int B>
struct DftComposite {
  static FFT_D void run(cpx<S>* v) {
    constexpr int R = A * B;
    cpx<S> t[R];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) {
      cpx<S> a[A];
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1) a[n1] = v[B * n1 + n2];
      dft<S, A>(a);
#pragma unroll
      for (int k1 = 0; k1 < A; ++k1) t[k1 * B + n2] = mul_root<S, R>(a[k1], n2 * k1);
    }
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
      dft<S, B>(t + k1 * B);
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = t[k1 * B + k2];
    }
  }
};

template <class S, int R>
FFT_D void dft(cpx<S>* v) {
  if constexpr (R == 1) {
  } else if constexpr (R == 2) {
    Dft2<S>::run(v);
  } else if constexpr (R == 4) {
    Dft4<S>::run(v);
  } else if constexpr (R == 8) {
    Dft8<S>::run(v);
  } else if constexpr (R == 3 || R == 5 || R == 7 || R == 11 || R == 13) {
    DftOddPrime<S, R>::run(v);
  } else if constexpr (R == 9) {
    DftComposite<S, 3, 3>::run(v);
  } else if constexpr (R == 16) {
    DftComposite<S, 4, 4>::run(v);
  } else {
    static_assert(R <= 16, "unsupported codelet radix");
  }
}
