// harmonics.cuh -- solid harmonics and translation operators for the Laplace
// far field.
//
// Basis (factorial normalisation, no Condon-Shortley phase):
//   Y_n^m(x) = (-1)^m r^n      P_n^m(cos t) e^{i m p} / (n+m)!   (regular)
//   T_n^m(x) = (-1)^m (n-m)!   P_n^m(cos t) e^{i m p} / r^{n+1}  (irregular)
// with the identities (all verified numerically in the tests)
//   1/|x-y|        = sum_{n,m} conj(Y_n^m(y)) T_n^m(x)          (|y| < |x|)
//   Y_n^m(a+b)     = sum_{k,l} Y_k^l(a) Y_{n-k}^{m-l}(b)
//   T_n^m(x-y)     = sum_{k,l} conj(Y_k^l(y)) T_{n+k}^{m+l}(x)
//   d_z Y_n^m = Y_{n-1}^m,  (d_x + i d_y) Y_n^m = Y_{n-1}^{m+1},
//   (d_x - i d_y) Y_n^m = -Y_{n-1}^{m-1},  Y_n^{-m} = (-1)^m conj(Y_n^m).
//
// Expansions (box centre c, box side s, scaled coordinates z = (x-c)/s):
//   multipole  phi(x) = (1/s) sum M_n^m T_n^m(z),  M_n^m = sum_i q_i conj(Y_n^m(z_i))
//   local      phi(x) =       sum L_n^m conj(Y_n^m(z))
// Sources are real, so only m >= 0 is stored; coefficient (n, m) lives at
// cidx(n, m) = n(n+1)/2 + m and every expansion is a real vector of length
// 2*ncoef(p) with interleaved (re, im).  All translations are level
// independent in these units (M2L carries an extra 1/s), so each translation
// is one real matrix per relative offset, applied as a dense contraction.
#pragma once
#include <math.h>
#include "tri_index.cuh"

namespace efmm {

struct cplx {
  double re, im;
};
EFMM_HD cplx cmul(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
EFMM_HD cplx cconj(cplx a) { return {a.re, -a.im}; }
EFMM_HD cplx cadd(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
EFMM_HD cplx cscale(double s, cplx a) { return {s * a.re, s * a.im}; }

EFMM_HD constexpr int ncoef(int p) { return (p + 1) * (p + 2) / 2; }
EFMM_HD constexpr int cidx(int n, int m) { return n * (n + 1) / 2 + m; }

// Regular harmonics Y_n^m(x), 0 <= m <= n <= p, into Y[cidx(n,m)].
EFMM_HD void regular_harmonics(int p, double x, double y, double z, cplx* Y) {
  double r2 = x * x + y * y + z * z;
  cplx w = {-0.5 * x, -0.5 * y};  // -(x+iy)/2
  cplx d = {1.0, 0.0};
  for (int m = 0; m <= p; m++) {
    if (m > 0) d = cscale(1.0 / m, cmul(d, w));  // Y_m^m = (-(x+iy)/2)^m / m!
    Y[cidx(m, m)] = d;
    cplx ym2 = {0.0, 0.0}, ym1 = d;
    for (int n = m + 1; n <= p; n++) {
      double a = (2.0 * n - 1.0) * z, b = r2;
      double inv = 1.0 / ((double)(n - m) * (double)(n + m));
      cplx yn = {(a * ym1.re - b * ym2.re) * inv, (a * ym1.im - b * ym2.im) * inv};
      Y[cidx(n, m)] = yn;
      ym2 = ym1;
      ym1 = yn;
    }
  }
}

// Irregular harmonics T_n^m(x), 0 <= m <= n <= N, into T[cidx(n,m)].
EFMM_HD void irregular_harmonics(int N, double x, double y, double z, cplx* T) {
  double r2 = x * x + y * y + z * z;
  double ir2 = 1.0 / r2;
  double ir = sqrt(ir2);
  cplx d = {ir, 0.0};
  for (int m = 0; m <= N; m++) {
    if (m > 0) {  // T_m^m = -(2m-1)(x+iy)/r^2 T_{m-1}^{m-1}
      double f = -(2.0 * m - 1.0) * ir2;
      d = cmul(d, {f * x, f * y});
    }
    T[cidx(m, m)] = d;
    cplx tm2 = {0.0, 0.0}, tm1 = d;
    for (int n = m + 1; n <= N; n++) {
      double a = (2.0 * n - 1.0) * z;
      double b = (double)(n - 1 + m) * (double)(n - 1 - m);
      cplx tn = {(a * tm1.re - b * tm2.re) * ir2, (a * tm1.im - b * tm2.im) * ir2};
      T[cidx(n, m)] = tn;
      tm2 = tm1;
      tm1 = tn;
    }
  }
}

// Harmonic table of the half-space kernel U(x) = z log(r + z) - r (z > 0 or
// off the negative z axis), the function whose derivatives give the B piece
// of Mindlin's image solution (src/mindlinpieces.f:29).  With the operators
// that make the irregular harmonics, T_n^m = (-d_z)^{n-m} (d_x + i d_y)^m (1/r),
// J_n^m = (-d_z)^{n-m} (d_x + i d_y)^m U.  Because d_z^2 U = 1/r,
// J_n^m = T_{n-2}^m for n - m >= 2; the two outer diagonals are
//   J_m^m     = (d_x + i d_y)^m U                = w^m G^m U,
//   J_{m+1}^m = -(d_x + i d_y)^m log(r + z)      = -w^m G^m log(r + z),
// w = x + iy, G = (1/r) d/dr at fixed z (radial functions only), with
// G U = -1/(r+z), G log(r+z) = 1/(r (r+z)) and G(r^-a (r+z)^-b) =
// -a r^-(a+2) (r+z)^-b - b r^-(a+1) (r+z)^-(b+1): positive coefficients
// with one overall sign, so the sums do not cancel.  Replacing T by J in
// the M2L coefficients gives the M2L operator of U.  0 <= m <= n <= N <= UH_MAX.
constexpr int UH_MAX = 120;
EFMM_HD void u_harmonics(int N, double x, double y, double z, cplx* J) {
  if (N >= 2) irregular_harmonics(N - 2, x, y, z, J);  // T_{n}^m into slot of n for now
  // shift the irregular table up by two degrees (n from N-2 down to 0)
  for (int n = N; n >= 2; n--)
    for (int m = 0; m <= n - 2; m++) J[cidx(n, m)] = J[cidx(n - 2, m)];
  const double r = sqrt(x * x + y * y + z * z);
  const double u = 1.0 / r, rho = r / (r + z);  // rho = v / u, v = 1/(r+z)
  // g_M = u^{2M-1} sum_b c_b rho^b (b = 1..M);  h_M = u^{2M} sum_b d_b rho^b
  double c[UH_MAX + 2], d[UH_MAX + 2];
  for (int b = 0; b <= N + 1 && b < UH_MAX + 2; b++) c[b] = d[b] = 0.0;
  c[1] = -1.0;
  d[1] = 1.0;
  cplx wm = {1.0, 0.0};
  const cplx w = {x, y};
  for (int M = 0; M <= N; M++) {
    double gM, hM;
    if (M == 0) {
      gM = z * log(r + z) - r;
      hM = log(r + z);
    } else {
      double sg = 0.0, sh = 0.0, rp = 1.0;
      for (int b = 1; b <= M; b++) {
        rp *= rho;
        sg += c[b] * rp;
        sh += d[b] * rp;
      }
      gM = sg * pow(u, 2 * M - 1);
      hM = sh * pow(u, 2 * M);
      // advance: c'_b = -(2M-1-b) c_b - (b-1) c_{b-1};  d'_b = -(2M-b) d_b - (b-1) d_{b-1}
      for (int b = M + 1; b >= 1; b--) {
        const double cb = b <= M ? c[b] : 0.0, db = b <= M ? d[b] : 0.0;
        c[b] = -(2.0 * M - 1.0 - b) * cb - (b - 1.0) * c[b - 1];
        d[b] = -(2.0 * M - b) * db - (b - 1.0) * d[b - 1];
      }
    }
    J[cidx(M, M)] = cscale(gM, wm);
    if (M + 1 <= N) J[cidx(M + 1, M)] = cscale(-hM, wm);
    wm = cmul(wm, w);
  }
}

// Access with negative orders through X_n^{-m} = (-1)^m conj(X_n^m).
EFMM_HD cplx hget(const cplx* X, int n, int m) {
  if (n < 0 || m > n || -m > n) return {0.0, 0.0};
  if (m >= 0) return X[cidx(n, m)];
  cplx v = X[cidx(n, -m)];
  return ((-m) & 1) ? cplx{-v.re, v.im} : cplx{v.re, -v.im};
}

// Gradient of Y_n^m dotted with a real vector d:
//   d.grad Y_n^m = d_z Y_{n-1}^m + (d_x - i d_y)/2 Y_{n-1}^{m+1} - (d_x + i d_y)/2 Y_{n-1}^{m-1}
EFMM_HD cplx dgrad_regular(const cplx* Y, int n, int m, double dx, double dy, double dz) {
  if (n == 0) return {0.0, 0.0};
  cplx a = hget(Y, n - 1, m), b = hget(Y, n - 1, m + 1), c = hget(Y, n - 1, m - 1);
  cplx r = cscale(dz, a);
  r = cadd(r, cmul({0.5 * dx, -0.5 * dy}, b));
  r = cadd(r, cmul({-0.5 * dx, -0.5 * dy}, c));
  return r;
}

// Real-matrix form of a complex operator out_n^m = sum_{k,l} A(n,m,k,l) in_k^l
// acting on m >= 0 storage of expansions of real fields (in_k^{-l} =
// (-1)^l conj(in_k^l)).  Row (n,m) re/im, column (k,l) re/im, given
// A = A(n,m,k,l) and Bm = A(n,m,k,-l) (Bm unused for l = 0).
EFMM_HD void real_block(cplx A, cplx Bm, int l, double* rr, double* ri, double* ir,
                        double* ii) {
  if (l == 0) {
    *rr = A.re; *ri = -A.im; *ir = A.im; *ii = A.re;
    return;
  }
  double sg = (l & 1) ? -1.0 : 1.0;
  cplx B = {sg * Bm.re, sg * Bm.im};
  *rr = A.re + B.re;
  *ri = -A.im + B.im;
  *ir = A.im + B.im;
  *ii = A.re - B.re;
}

// M2L coefficient A(n,m,k,l) = (-1)^n T_{n+k}^{m+l}(X), X = offset in box units,
// from a table T of irregular harmonics up to order 2p.
EFMM_HD cplx m2l_coef(const cplx* T, int n, int m, int k, int l) {
  cplx t = hget(T, n + k, m + l);
  return (n & 1) ? cplx{-t.re, -t.im} : t;
}
// M2M (child -> parent) A(n,m,k,l) = 2^-k conj(Y_{n-k}^{m-l}(d)), d = (c_child - c_parent)/s_parent
// L2L (parent -> child) A(k,l,n,m) = 2^-k conj(Y_{n-k}^{m-l}(d)) (rows k,l; columns n,m)
EFMM_HD cplx shift_coef(const cplx* Y, int nhi, int mhi, int nlo, int mlo, double scale_lo) {
  if (nlo > nhi) return {0.0, 0.0};
  cplx y = hget(Y, nhi - nlo, mhi - mlo);
  return {scale_lo * y.re, -scale_lo * y.im};
}

// 2 x 2 real block of the operator of `kind` (0 M2L, 1 M2M, 2 L2L) between
// output coefficient r = cidx(n,m) and input coefficient c = cidx(k,l), from
// the harmonics table of the offset (irregular up to 2p for M2L, regular up
// to p for the shifts).
EFMM_HD void op_entry(int kind, const cplx* tab, int r, int c, double* rr, double* ri, double* ir,
                      double* ii) {
  int n = 0;
  while ((n + 1) * (n + 2) / 2 <= r) n++;
  int m = r - n * (n + 1) / 2;
  int k = 0;
  while ((k + 1) * (k + 2) / 2 <= c) k++;
  int l = c - k * (k + 1) / 2;
  cplx A, B;
  if (kind == 0) {
    A = m2l_coef(tab, n, m, k, l);
    B = m2l_coef(tab, n, m, k, -l);
  } else if (kind == 1) {  // M2M: rows (n,m) parent, cols (k,l) child
    double sc = ldexp(1.0, -k);
    A = shift_coef(tab, n, m, k, l, sc);
    B = shift_coef(tab, n, m, k, -l, sc);
  } else {  // L2L: rows (n,m) child, cols (k,l) parent: 2^-n conj(Y_{k-n}^{l-m})
    double sc = ldexp(1.0, -n);
    A = shift_coef(tab, k, l, n, m, sc);
    B = shift_coef(tab, k, -l, n, m, sc);
  }
  real_block(A, B, l, rr, ri, ir, ii);
}

// Evaluate potential, gradient and Hessian of a local expansion at scaled
// point z (box side s).  L: 2*ncoef(p) interleaved.  Outputs are the physical
// derivatives (divided by s, s^2).  hess order: xx, yy, zz, xy, xz, yz.
EFMM_HD void local_eval(int p, const double* L, const cplx* Y, double s, double* pot,
                        double* grad, double* hess) {
  // sums S = sum_{n,m} C_n^m conj(Y_n^m(z)) for shifted coefficient sets:
  //   phi:  L_n^m            Dz: L_{n+1}^m        D+: -L_{n+1}^{m+1}
  //   Dzz:  L_{n+2}^m        D+Dz: -L_{n+2}^{m+1}  D+D+: L_{n+2}^{m+2}
  double phi = 0.0, dz = 0.0, dzz = 0.0;
  cplx dp = {0, 0}, dpz = {0, 0}, dpp = {0, 0};
  auto Lg = [&](int n, int m) -> cplx {
    if (n > p || m > n || -m > n) return cplx{0.0, 0.0};
    if (m >= 0) return cplx{L[2 * cidx(n, m)], L[2 * cidx(n, m) + 1]};
    double re = L[2 * cidx(n, -m)], im = L[2 * cidx(n, -m) + 1];
    return ((-m) & 1) ? cplx{-re, im} : cplx{re, -im};
  };
  for (int n = 0; n <= p; n++) {
    for (int m = -n; m <= n; m++) {
      cplx yc = cconj(hget(Y, n, m));
      cplx c0 = Lg(n, m);
      phi += c0.re * yc.re - c0.im * yc.im;
      if (n + 1 <= p) {
        cplx c1 = Lg(n + 1, m);
        dz += c1.re * yc.re - c1.im * yc.im;
        cplx c2 = Lg(n + 1, m + 1);
        dp = cadd(dp, cmul(cplx{-c2.re, -c2.im}, yc));
      }
      if (n + 2 <= p) {
        cplx c3 = Lg(n + 2, m);
        dzz += c3.re * yc.re - c3.im * yc.im;
        cplx c4 = Lg(n + 2, m + 1);
        dpz = cadd(dpz, cmul(cplx{-c4.re, -c4.im}, yc));
        cplx c5 = Lg(n + 2, m + 2);
        dpp = cadd(dpp, cmul(c5, yc));
      }
    }
  }
  double is = 1.0 / s, is2 = is * is;
  *pot = phi;
  grad[0] = dp.re * is;
  grad[1] = dp.im * is;
  grad[2] = dz * is;
  double hzz = dzz;
  hess[0] = 0.5 * (dpp.re - hzz) * is2;
  hess[1] = 0.5 * (-dpp.re - hzz) * is2;
  hess[2] = hzz * is2;
  hess[3] = 0.5 * dpp.im * is2;
  hess[4] = dpz.re * is2;
  hess[5] = dpz.im * is2;
}

// Expansion order from the tolerance: smallest j >= 2 with
// (sqrt(3)/2)^j / z1^(j+1) < eps (the decay model of src/l3dterms.f:42),
// z1 = 1.5 for adjacent-but-separated boxes.
inline int order_for_eps(double eps, double z1) {
  double z2 = sqrt(3.0) / 2.0, jf = z2, hf = 1.0 / (z1 * z1);
  for (int j = 2; j <= 1000; j++) {
    hf /= z1;
    jf *= z2;
    if (jf * hf < eps) return j;
  }
  return 1000;
}

// Per-offset truncated order for list-2 offset (i,j,k), |max| in {2,3}
// (src/l3dterms.f:144 l3dterms_list2): distance from the nearer box face.
inline int m2l_order(double eps, int i, int j, int k) {
  int a[3] = {abs(i), abs(j), abs(k)};
  // dominant axis first, the two others in the reference's order
  int ii, jj, kk;
  if (a[0] > 1) { ii = a[0]; jj = a[1]; kk = a[2]; }
  else if (a[1] > 1) { ii = a[1]; jj = a[0]; kk = a[2]; }
  else { ii = a[2]; if (a[0] >= a[1]) { jj = a[0]; kk = a[1]; } else { jj = a[1]; kk = a[0]; } }
  double dx = ii > 0 ? ii - 0.5 : 0.0, dy = jj > 0 ? jj - 0.5 : 0.0, dz = kk > 0 ? kk - 0.5 : 0.0;
  return order_for_eps(eps, sqrt(dx * dx + dy * dy + dz * dz));
}

}  // namespace efmm
