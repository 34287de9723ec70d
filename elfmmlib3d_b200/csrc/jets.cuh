// jets.cuh -- truncated multivariate Taylor arithmetic in three variables.
//
// A Jet<N> holds the Taylor coefficients c_a = d^a f / a! of a function of
// (x, y, z) about a point, for all multi-indices |a| <= N.  Products and
// compositions with smooth univariate functions are exact up to order N, so
// evaluating a closed-form expression on jets yields all of its partial
// derivatives up to order N in one pass.  The near-field kernels use this to
// differentiate the closed-form edge integrals of r and 1/r with respect to the
// target point.
#pragma once

#ifdef __CUDACC__
#define EFMM_HD __host__ __device__ __forceinline__
#else
#define EFMM_HD inline
#endif

namespace efmm {

// number of coefficients with total degree <= n
EFMM_HD constexpr int jet_size(int n) { return (n + 1) * (n + 2) * (n + 3) / 6; }

// linear index of multi-index (a,b,c): grouped by total degree, then by a
// descending, then b descending.
EFMM_HD constexpr int jidx(int a, int b, int c) {
  int n = a + b + c;
  int off = n * (n + 1) * (n + 2) / 6;
  int pos = 0;
  for (int ap = n; ap > a; --ap) pos += n - ap + 1;
  pos += (n - a) - b;
  return off + pos;
}

EFMM_HD constexpr int ifact(int n) { return n <= 1 ? 1 : n * ifact(n - 1); }

}  // namespace efmm
#include "jets_gen.cuh"
namespace efmm {

template <int N>
struct Jet {
  static constexpr int NC = jet_size(N);
  double c[NC];

  EFMM_HD static Jet constant(double v) {
    Jet j;
#pragma unroll
    for (int i = 0; i < NC; i++) j.c[i] = 0.0;
    j.c[0] = v;
    return j;
  }
  // v + (dx, dy, dz) . (X - X0): an affine function of the three variables
  EFMM_HD static Jet affine(double v, double dx, double dy, double dz) {
    Jet j = constant(v);
    if (N >= 1) {
      j.c[jidx(1, 0, 0)] = dx;
      j.c[jidx(0, 1, 0)] = dy;
      j.c[jidx(0, 0, 1)] = dz;
    }
    return j;
  }
  // partial derivative d^(a,b,c) f at the expansion point
  EFMM_HD double deriv(int a, int b, int cc) const {
    return c[jidx(a, b, cc)] * (double)(ifact(a) * ifact(b) * ifact(cc));
  }
};

template <int N>
EFMM_HD Jet<N> operator+(const Jet<N>& x, const Jet<N>& y) {
  Jet<N> z;
#pragma unroll
  for (int i = 0; i < Jet<N>::NC; i++) z.c[i] = x.c[i] + y.c[i];
  return z;
}
template <int N>
EFMM_HD Jet<N> operator-(const Jet<N>& x, const Jet<N>& y) {
  Jet<N> z;
#pragma unroll
  for (int i = 0; i < Jet<N>::NC; i++) z.c[i] = x.c[i] - y.c[i];
  return z;
}
template <int N>
EFMM_HD Jet<N> operator*(double s, const Jet<N>& x) {
  Jet<N> z;
#pragma unroll
  for (int i = 0; i < Jet<N>::NC; i++) z.c[i] = s * x.c[i];
  return z;
}
template <int N>
EFMM_HD Jet<N> operator+(const Jet<N>& x, double s) {
  Jet<N> z = x;
  z.c[0] += s;
  return z;
}

// Cauchy product truncated at order 3 (straight-line code from gen_jets.py)
EFMM_HD Jet<3> operator*(const Jet<3>& x, const Jet<3>& y) {
  Jet<3> z;
  jet3_mul(x.c, y.c, z.c);
  return z;
}

// f(x) where t[k] = f^(k)(x0)/k!, x0 = constant term of x
template <int N>
EFMM_HD Jet<N> compose(const Jet<N>& x, const double (&t)[N + 1]) {
  Jet<N> d = x;
  d.c[0] = 0.0;
  Jet<N> z = Jet<N>::constant(t[0]);
  Jet<N> p = d;
#pragma unroll
  for (int k = 1; k <= N; k++) {
#pragma unroll
    for (int i = 0; i < Jet<N>::NC; i++) z.c[i] += t[k] * p.c[i];
    if (k < N) p = p * d;
  }
  return z;
}

template <int N>
EFMM_HD Jet<N> jsqrt(const Jet<N>& x) {
  double x0 = x.c[0];
  double s = sqrt(x0);
  double t[N + 1];
  // d^k/dx^k sqrt(x) / k! = binom(1/2, k) x^(1/2-k)
  double coef = s, e = 0.5;
#pragma unroll
  for (int k = 0; k <= N; k++) {
    t[k] = coef;
    coef = coef * (e - k) / ((k + 1) * x0);
  }
  return compose<N>(x, t);
}

template <int N>
EFMM_HD Jet<N> jlog(const Jet<N>& x) {
  double x0 = x.c[0];
  double t[N + 1];
  t[0] = log(x0);
  double ip = 1.0 / x0, pw = ip;
#pragma unroll
  for (int k = 1; k <= N; k++) {
    t[k] = ((k & 1) ? 1.0 : -1.0) * pw / k;
    pw *= ip;
  }
  return compose<N>(x, t);
}

// log(1 + x), accurate when the constant term of x is small
template <int N>
EFMM_HD Jet<N> jlog1p(const Jet<N>& x) {
  double x0 = x.c[0];
  double t[N + 1];
  t[0] = log1p(x0);
  double ip = 1.0 / (1.0 + x0), pw = ip;
#pragma unroll
  for (int k = 1; k <= N; k++) {
    t[k] = ((k & 1) ? 1.0 : -1.0) * pw / k;
    pw *= ip;
  }
  return compose<N>(x, t);
}

template <int N>
EFMM_HD Jet<N> jinv(const Jet<N>& x) {
  double x0 = x.c[0];
  double ip = 1.0 / x0;
  double t[N + 1];
  double pw = ip;
#pragma unroll
  for (int k = 0; k <= N; k++) {
    t[k] = ((k & 1) ? -1.0 : 1.0) * pw;
    pw *= ip;
  }
  return compose<N>(x, t);
}

}  // namespace efmm
