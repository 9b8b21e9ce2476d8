// fb_device.cuh -- complex arithmetic and register butterflies for sm_100a.
//
// Every add, multiply and fused multiply-add below is written with the
// round-to-nearest intrinsics (__fadd_rn, __fmul_rn, __fmaf_rn and the double
// forms).  The compiler never contracts or reorders those, so a butterfly
// gives the same bits in every kernel that inlines it.  That is what keeps a
// batched or strided transform bit-for-bit equal to the same transform run on
// one contiguous line, the property FFTA's tests check with `==`
// (test/onedim/complex_forward.jl:27-33, test/twodim/complex_forward.jl:29-43).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fb {

// ------------------------------------------------------------ scalar ops
template <typename R> struct Sc;
template <> struct Sc<float> {
  typedef float2 C;
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
  static __device__ __forceinline__ C mk(float x, float y) { return make_float2(x, y); }
};
template <> struct Sc<double> {
  typedef double2 C;
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
  static __device__ __forceinline__ C mk(double x, double y) { return make_double2(x, y); }
};

template <typename R> using cplx = typename Sc<R>::C;

template <typename R> __device__ __forceinline__ cplx<R> cadd(cplx<R> a, cplx<R> b) {
  return Sc<R>::mk(Sc<R>::add(a.x, b.x), Sc<R>::add(a.y, b.y));
}
template <typename R> __device__ __forceinline__ cplx<R> csub(cplx<R> a, cplx<R> b) {
  return Sc<R>::mk(Sc<R>::sub(a.x, b.x), Sc<R>::sub(a.y, b.y));
}
// a * b
template <typename R> __device__ __forceinline__ cplx<R> cmul(cplx<R> a, cplx<R> b) {
  return Sc<R>::mk(Sc<R>::fma(a.x, b.x, -Sc<R>::mul(a.y, b.y)),
                   Sc<R>::fma(a.x, b.y, Sc<R>::mul(a.y, b.x)));
}
// a * conj(b)
template <typename R> __device__ __forceinline__ cplx<R> cmulc(cplx<R> a, cplx<R> b) {
  return Sc<R>::mk(Sc<R>::fma(a.x, b.x, Sc<R>::mul(a.y, b.y)),
                   Sc<R>::fma(a.y, b.x, -Sc<R>::mul(a.x, b.y)));
}
// Four-step twiddle of element i of a line whose first stage has radix `rad`,
// from a full table t(k) = w^(k*l) (l: the line's twiddle index).  With
// nb = L/rad the first stage's butterfly j holds i = j + r*nb; for rad >= 4
// and r = 4a + c the twiddle is t(i - c*nb) * t(c*nb) (c > 0): a butterfly
// needs the entries r = 0, 4, 8, ... of its own and the line's three steps
// t(nb), t(2nb), t(3nb), at the cost of one more rounding.  The specialised
// and the generic kernels both form exactly this product.
template <typename R, class Tab>
__device__ __forceinline__ cplx<R> tw_elem(const Tab& t, int i, int nb, int rad) {
  if (rad < 4) return t(i);
  const int c = (i / nb) & 3;
  const cplx<R> b = t(i - c * nb);
  return c == 0 ? b : cmul<R>(b, t(c * nb));
}
// a * w where w is a forward-direction root; DIR>0 uses conj(w).
template <typename R, int DIR> __device__ __forceinline__ cplx<R> ctw(cplx<R> a, cplx<R> w) {
  return DIR < 0 ? cmul<R>(a, w) : cmulc<R>(a, w);
}
template <typename R> __device__ __forceinline__ cplx<R> cscale(cplx<R> a, R s) {
  return Sc<R>::mk(Sc<R>::mul(a.x, s), Sc<R>::mul(a.y, s));
}
// a * (-i*dir)... rotation used by the forward (-i) and backward (+i) kernels:
// DIR<0 multiplies by -i, DIR>0 by +i.  Exact.
template <typename R, int DIR> __device__ __forceinline__ cplx<R> rot(cplx<R> a) {
  return DIR < 0 ? Sc<R>::mk(a.y, -a.x) : Sc<R>::mk(-a.y, a.x);
}

// Constants, each a decimal literal rounded once to the working type.
template <typename R> struct K;
template <> struct K<float> {
  static constexpr float r2 = 0.70710678118654752440f;   // sqrt(2)/2
  static constexpr float c8 = 0.92387953251128675613f;   // cos(pi/8)
  static constexpr float s8 = 0.38268343236508977173f;   // sin(pi/8)
  static constexpr float s3 = 0.86602540378443864676f;   // sin(2pi/3)
  static constexpr float c51 = 0.30901699437494742410f;  // cos(2pi/5)
  static constexpr float c52 = -0.80901699437494742410f; // cos(4pi/5)
  static constexpr float s51 = 0.95105651629515357212f;  // sin(2pi/5)
  static constexpr float s52 = 0.58778525229247312917f;  // sin(4pi/5)
  static constexpr float c91 = 0.76604444311897803520f;  // cos(2pi/9)
  static constexpr float s91 = 0.64278760968653932632f;  // sin(2pi/9)
  static constexpr float c92 = 0.17364817766693034885f;  // cos(4pi/9)
  static constexpr float s92 = 0.98480775301220805936f;  // sin(4pi/9)
  static constexpr float c94 = -0.93969262078590838405f; // cos(8pi/9)
  static constexpr float s94 = 0.34202014332566873304f;  // sin(8pi/9)
};
template <> struct K<double> {
  static constexpr double r2 = 0.70710678118654752440;
  static constexpr double c8 = 0.92387953251128675613;
  static constexpr double s8 = 0.38268343236508977173;
  static constexpr double s3 = 0.86602540378443864676;
  static constexpr double c51 = 0.30901699437494742410;
  static constexpr double c52 = -0.80901699437494742410;
  static constexpr double s51 = 0.95105651629515357212;
  static constexpr double s52 = 0.58778525229247312917;
  static constexpr double c91 = 0.76604444311897803520;
  static constexpr double s91 = 0.64278760968653932632;
  static constexpr double c92 = 0.17364817766693034885;
  static constexpr double s92 = 0.98480775301220805936;
  static constexpr double c94 = -0.93969262078590838405;
  static constexpr double s94 = 0.34202014332566873304;
};

// -------------------------------------------------------- butterflies
// In-place DFT of v[0..R) with X_k = sum_n v_n exp(DIR * 2 pi i n k / R),
// DIR = -1 forward, +1 backward.  Outputs in natural order.

template <typename R, int DIR> __device__ __forceinline__ void bf2(cplx<R>& a, cplx<R>& b) {
  cplx<R> t = a;
  a = cadd<R>(t, b);
  b = csub<R>(t, b);
}

template <typename R, int DIR> __device__ __forceinline__ void dft4(cplx<R>* v) {
  cplx<R> t0 = cadd<R>(v[0], v[2]);
  cplx<R> t1 = csub<R>(v[0], v[2]);
  cplx<R> t2 = cadd<R>(v[1], v[3]);
  cplx<R> t3 = rot<R, DIR>(csub<R>(v[1], v[3]));
  v[0] = cadd<R>(t0, t2);
  v[2] = csub<R>(t0, t2);
  v[1] = cadd<R>(t1, t3);
  v[3] = csub<R>(t1, t3);
}

// multiply by exp(DIR*2*pi*i*k/8), k = 1, 3
template <typename R, int DIR> __device__ __forceinline__ cplx<R> w8_1(cplx<R> a) {
  // forward: (x + y, y - x) / sqrt2 ; backward: (x - y, x + y) / sqrt2
  const R c = K<R>::r2;
  return DIR < 0 ? Sc<R>::mk(Sc<R>::mul(Sc<R>::add(a.x, a.y), c), Sc<R>::mul(Sc<R>::sub(a.y, a.x), c))
                 : Sc<R>::mk(Sc<R>::mul(Sc<R>::sub(a.x, a.y), c), Sc<R>::mul(Sc<R>::add(a.x, a.y), c));
}
template <typename R, int DIR> __device__ __forceinline__ cplx<R> w8_3(cplx<R> a) {
  // forward w8^3 = (-1 - i)/sqrt2 : (-x + y, -x - y)/sqrt2 ; backward (-1 + i)/sqrt2 : (-x - y, x - y)/sqrt2
  const R c = K<R>::r2;
  return DIR < 0 ? Sc<R>::mk(Sc<R>::mul(Sc<R>::sub(a.y, a.x), c), -Sc<R>::mul(Sc<R>::add(a.x, a.y), c))
                 : Sc<R>::mk(-Sc<R>::mul(Sc<R>::add(a.x, a.y), c), Sc<R>::mul(Sc<R>::sub(a.x, a.y), c));
}

template <typename R, int DIR> __device__ __forceinline__ void dft8(cplx<R>* v) {
  cplx<R> e[4] = {v[0], v[2], v[4], v[6]};
  cplx<R> o[4] = {v[1], v[3], v[5], v[7]};
  dft4<R, DIR>(e);
  dft4<R, DIR>(o);
  o[1] = w8_1<R, DIR>(o[1]);
  o[2] = rot<R, DIR>(o[2]);
  o[3] = w8_3<R, DIR>(o[3]);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = cadd<R>(e[k], o[k]);
    v[k + 4] = csub<R>(e[k], o[k]);
  }
}

// multiply by a root given as (c, s): forward uses (c - i s), backward (c + i s)
template <typename R, int DIR> __device__ __forceinline__ cplx<R> mulcs(cplx<R> a, R c, R s) {
  cplx<R> w = Sc<R>::mk(c, DIR < 0 ? -s : s);
  return cmul<R>(a, w);
}

template <typename R, int DIR> __device__ __forceinline__ void dft16(cplx<R>* v) {
  // n = 4 n1 + n2, k = k1 + 4 k2
  cplx<R> b[4][4];
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) {
    cplx<R> t[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
    dft4<R, DIR>(t);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) b[n2][k1] = t[k1];
  }
  const R c1 = K<R>::c8, s1 = K<R>::s8;
  // twiddles w16^(n2*k1)
  b[1][1] = mulcs<R, DIR>(b[1][1], c1, s1);        // w^1
  b[1][2] = w8_1<R, DIR>(b[1][2]);                 // w^2
  b[1][3] = mulcs<R, DIR>(b[1][3], s1, c1);        // w^3: (cos 3pi/8, sin 3pi/8) = (s1, c1)
  b[2][1] = w8_1<R, DIR>(b[2][1]);                 // w^2
  b[2][2] = rot<R, DIR>(b[2][2]);                  // w^4
  b[2][3] = w8_3<R, DIR>(b[2][3]);                 // w^6
  b[3][1] = mulcs<R, DIR>(b[3][1], s1, c1);        // w^3
  b[3][2] = w8_3<R, DIR>(b[3][2]);                 // w^6
  b[3][3] = mulcs<R, DIR>(b[3][3], -c1, -s1);      // w^9 = -w^1
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    cplx<R> t[4] = {b[0][k1], b[1][k1], b[2][k1], b[3][k1]};
    dft4<R, DIR>(t);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[k2];
  }
}

template <typename R, int DIR> __device__ __forceinline__ void dft3(cplx<R>* v) {
  cplx<R> t = cadd<R>(v[1], v[2]);
  cplx<R> d = csub<R>(v[1], v[2]);
  cplx<R> m = Sc<R>::mk(Sc<R>::fma(R(-0.5), t.x, v[0].x), Sc<R>::fma(R(-0.5), t.y, v[0].y));
  cplx<R> j = rot<R, DIR>(cscale<R>(d, K<R>::s3));
  v[0] = cadd<R>(v[0], t);
  v[1] = cadd<R>(m, j);
  v[2] = csub<R>(m, j);
}

// 9 = 3 x 3: n = 3 n1 + n2, k = k1 + 3 k2, inner twiddles w9^(n2 k1).
template <typename R, int DIR> __device__ __forceinline__ void dft9(cplx<R>* v) {
  cplx<R> b[3][3];
#pragma unroll
  for (int n2 = 0; n2 < 3; ++n2) {
    cplx<R> t[3] = {v[n2], v[3 + n2], v[6 + n2]};
    dft3<R, DIR>(t);
#pragma unroll
    for (int k1 = 0; k1 < 3; ++k1) b[n2][k1] = t[k1];
  }
  b[1][1] = mulcs<R, DIR>(b[1][1], K<R>::c91, K<R>::s91);  // w9^1
  b[1][2] = mulcs<R, DIR>(b[1][2], K<R>::c92, K<R>::s92);  // w9^2
  b[2][1] = mulcs<R, DIR>(b[2][1], K<R>::c92, K<R>::s92);  // w9^2
  b[2][2] = mulcs<R, DIR>(b[2][2], K<R>::c94, K<R>::s94);  // w9^4
#pragma unroll
  for (int k1 = 0; k1 < 3; ++k1) {
    cplx<R> t[3] = {b[0][k1], b[1][k1], b[2][k1]};
    dft3<R, DIR>(t);
#pragma unroll
    for (int k2 = 0; k2 < 3; ++k2) v[k1 + 3 * k2] = t[k2];
  }
}

template <typename R, int DIR> __device__ __forceinline__ void dft5(cplx<R>* v) {
  typedef Sc<R> S;
  cplx<R> a = cadd<R>(v[1], v[4]), b = cadd<R>(v[2], v[3]);
  cplx<R> c = csub<R>(v[1], v[4]), d = csub<R>(v[2], v[3]);
  const R c1 = K<R>::c51, c2 = K<R>::c52, s1 = K<R>::s51, s2 = K<R>::s52;
  cplx<R> m1 = S::mk(S::fma(c2, b.x, S::fma(c1, a.x, v[0].x)), S::fma(c2, b.y, S::fma(c1, a.y, v[0].y)));
  cplx<R> m2 = S::mk(S::fma(c1, b.x, S::fma(c2, a.x, v[0].x)), S::fma(c1, b.y, S::fma(c2, a.y, v[0].y)));
  cplx<R> n1 = S::mk(S::fma(s2, d.x, S::mul(s1, c.x)), S::fma(s2, d.y, S::mul(s1, c.y)));
  cplx<R> n2 = S::mk(S::fma(-s1, d.x, S::mul(s2, c.x)), S::fma(-s1, d.y, S::mul(s2, c.y)));
  v[0] = cadd<R>(v[0], cadd<R>(a, b));
  cplx<R> r1 = rot<R, DIR>(n1), r2 = rot<R, DIR>(n2);
  v[1] = cadd<R>(m1, r1);
  v[4] = csub<R>(m1, r1);
  v[2] = cadd<R>(m2, r2);
  v[3] = csub<R>(m2, r2);
}

// Odd prime P >= 7 through the symmetric-pair form.  cs[2*m], cs[2*m+1] hold
// cos(2 pi m / P), sin(2 pi m / P) for m < P (FP64-generated, rounded once).
// Primes up to 13 are fully unrolled; larger ones (rare: factors 17..71 of a
// length) keep the loops rolled to bound code size.
template <typename R, int DIR, int P>
__device__ __forceinline__ void dftp(cplx<R>* v, const R* __restrict__ cs) {
  typedef Sc<R> S;
  constexpr int H = (P - 1) / 2;
  constexpr bool UNROLL = P <= 13;
  cplx<R> a[H], b[H];
#pragma unroll
  for (int k = 0; k < H; ++k) {
    a[k] = cadd<R>(v[k + 1], v[P - 1 - k]);
    b[k] = csub<R>(v[k + 1], v[P - 1 - k]);
  }
  cplx<R> x0 = v[0];
  cplx<R> s = x0;
#pragma unroll
  for (int k = 0; k < H; ++k) s = cadd<R>(s, a[k]);
  v[0] = s;
  if constexpr (UNROLL) {
#pragma unroll
    for (int j = 1; j <= H; ++j) {
      cplx<R> A = x0, B = S::mk(R(0), R(0));
#pragma unroll
      for (int k = 1; k <= H; ++k) {
        const int m = (j * k) % P;
        const R c = cs[2 * m], sn = cs[2 * m + 1];
        A = S::mk(S::fma(c, a[k - 1].x, A.x), S::fma(c, a[k - 1].y, A.y));
        B = S::mk(S::fma(sn, b[k - 1].x, B.x), S::fma(sn, b[k - 1].y, B.y));
      }
      cplx<R> rb = rot<R, DIR>(B);
      v[j] = cadd<R>(A, rb);
      v[P - j] = csub<R>(A, rb);
    }
  } else {
#pragma unroll 1
    for (int j = 1; j <= H; ++j) {
      cplx<R> A = x0, B = S::mk(R(0), R(0));
      int m = 0;
#pragma unroll 1
      for (int k = 1; k <= H; ++k) {
        m += j;
        if (m >= P) m -= P;
        const R c = cs[2 * m], sn = cs[2 * m + 1];
        A = S::mk(S::fma(c, a[k - 1].x, A.x), S::fma(c, a[k - 1].y, A.y));
        B = S::mk(S::fma(sn, b[k - 1].x, B.x), S::fma(sn, b[k - 1].y, B.y));
      }
      cplx<R> rb = rot<R, DIR>(B);
      v[j] = cadd<R>(A, rb);
      v[P - j] = csub<R>(A, rb);
    }
  }
}

}  // namespace fb
