/*
 * oracle.c -- CPU FP64 oracle for the elastostatic triangle-layer FMM.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this file.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference arm may use it, and only as the checker (or as the
 * timed CPU stand-in for the reference, which cannot be compiled here: the
 * reference is Fortran 77/90 and no Fortran compiler exists on this image).
 *
 * What it restates (reference paths are relative to the elfmmlib3d tree):
 *
 *   - triangle frame            src/trilib.f:535-577, rotshift3d trilib.f:457
 *   - derivative tables         src/triahquad.f:680-1010 (triartable/triabtable):
 *       R(ix,iy,iz) = int_T d^{ix}_x d^{iy}_y d^{iz}_z (1/r) dT,  |a|<=2
 *       B(ix,iy,iz) = int_T d^{ix}_x d^{iy}_y d^{iz}_z (r)   dT,  |a|<=4
 *     derivatives taken w.r.t. the SOURCE point (x,y,z) at z=0, the target at
 *     (x0,y0,z0) (kernel list triahquad.f:127-200, triahfun :1016).  On-surface
 *     (self) values use the reference's iquad=0 convention: principal value for
 *     odd-in-z0 terms and Hadamard finite part for hypersingular ones.
 *     The reference evaluates these with closed-form edge formulas; the oracle
 *     integrates the kernel definitions numerically instead (Gauss rule on the
 *     triangle for far targets, polar quadrature about the projected target for
 *     near ones, with the radial finite part taken analytically when z0 = 0),
 *     so it is independent of both the reference's and the product's closed
 *     forms.
 *   - SLP/DLP assembly          src/elfmm3dtria.f:1689-2015 (elust3triadirecttarg_one)
 *                               src/elfmm3dtria.f:2368-2911 (eltst3triadirecttarg_one)
 *   - direct O(N^2) sum         src/elfmm3dtria.f:1483 (el3dtriadirecttarg)
 *   - oct-tree + lists          src/d3tstrcr.f:31-270 (d3tstrcr), :1249 (d3tallbem),
 *                               :1712/:1867 (d3tsepa1/0), :1596/:1682 (d3tcentc/f),
 *                               :702 (d3tlsts), :919 (d3tlst31), :1082 (d3tifint);
 *                               Mindlin root rule src/d3tstrcr_mindlin.f:1380-1383.
 *
 * Parity status: the reference publishes no golden vectors and cannot be built
 * here, so the oracle is pinned against the reference's documented integral
 * definitions (independent mpmath quadrature, tests/golden/make_golden.py), against
 * exact identities (rigid-body double layer on a closed surface) and against
 * the reference's own test recipe (direct sum, elfmm3dtria_dr.f:142-205).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Gauss-Legendre nodes on [0,1] (Newton on P_n)                             */
/* ------------------------------------------------------------------------ */
#define MAXGL 32
static double gl_x[MAXGL + 1][MAXGL], gl_w[MAXGL + 1][MAXGL];
static int gl_ready[MAXGL + 1];

static void gl_make(int n) {
  for (int i = 0; i < n; i++) {
    double x = cos(M_PI * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; it++) {
      double p0 = 1, p1 = x;
      for (int k = 2; k <= n; k++) {
        double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
        p0 = p1; p1 = p2;
      }
      double pn = (n == 1) ? x : p1;
      double pm = (n == 1) ? 1 : p0;
      double dp = n * (x * pn - pm) / (x * x - 1);
      double dx = pn / dp;
      x -= dx;
      if (fabs(dx) < 1e-16) break;
    }
    double p0 = 1, p1 = x;
    for (int k = 2; k <= n; k++) {
      double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
      p0 = p1; p1 = p2;
    }
    double dp = n * (x * p1 - p0) / (x * x - 1);
    gl_x[n][i] = 0.5 * (1 - x);
    gl_w[n][i] = 1.0 / ((1 - x * x) * dp * dp);
  }
  gl_ready[n] = 1;
}

static void gl_init(void) {
  for (int n = 1; n <= MAXGL; n++)
    if (!gl_ready[n]) gl_make(n);
}

/* ------------------------------------------------------------------------ */
/* triangle frame: vert1 -> origin, vert1->vert2 on +x, normal = +z           */
/* (trilib.f:457 rotshift3d, trilib.f:535 tri_ini)                            */
/* ------------------------------------------------------------------------ */
typedef struct {
  double rot[3][3]; /* rot[i][c]: column c = c-th local axis in global coords */
  double org[3];
  double v[3][2];   /* local 2d vertices */
} frame_t;

static void frame_init(const double *tri, frame_t *f) {
  const double *a = tri, *b = tri + 3, *c = tri + 6;
  double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  double l1 = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
  for (int i = 0; i < 3; i++) e1[i] /= l1;
  double v2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  double e3[3] = {e1[1] * v2[2] - e1[2] * v2[1], e1[2] * v2[0] - e1[0] * v2[2],
                  e1[0] * v2[1] - e1[1] * v2[0]};
  double l3 = sqrt(e3[0] * e3[0] + e3[1] * e3[1] + e3[2] * e3[2]);
  for (int i = 0; i < 3; i++) e3[i] /= l3;
  double e2[3] = {e3[1] * e1[2] - e3[2] * e1[1], e3[2] * e1[0] - e3[0] * e1[2],
                  e3[0] * e1[1] - e3[1] * e1[0]};
  for (int i = 0; i < 3; i++) {
    f->rot[i][0] = e1[i];
    f->rot[i][1] = e2[i];
    f->rot[i][2] = e3[i];
    f->org[i] = a[i];
  }
  f->v[0][0] = 0; f->v[0][1] = 0;
  f->v[1][0] = l1; f->v[1][1] = 0;
  f->v[2][0] = e1[0] * v2[0] + e1[1] * v2[1] + e1[2] * v2[2];
  f->v[2][1] = e2[0] * v2[0] + e2[1] * v2[1] + e2[2] * v2[2];
}

static void frame_fwd_pt(const frame_t *f, const double *x, double *y) {
  double t[3] = {x[0] - f->org[0], x[1] - f->org[1], x[2] - f->org[2]};
  for (int c = 0; c < 3; c++)
    y[c] = f->rot[0][c] * t[0] + f->rot[1][c] * t[1] + f->rot[2][c] * t[2];
}
static void frame_fwd_vec(const frame_t *f, const double *x, double *y) {
  for (int c = 0; c < 3; c++)
    y[c] = f->rot[0][c] * x[0] + f->rot[1][c] * x[1] + f->rot[2][c] * x[2];
}
static void frame_bak_vec(const frame_t *f, const double *x, double *y) {
  for (int i = 0; i < 3; i++)
    y[i] = f->rot[i][0] * x[0] + f->rot[i][1] * x[1] + f->rot[i][2] * x[2];
}
/* H_global = Rot H_local Rot^T  (trilib.f:766 rothess3d) */
static void frame_bak_mat(const frame_t *f, const double h[3][3], double out[3][3]) {
  double t[3][3];
  for (int i = 0; i < 3; i++)
    for (int k = 0; k < 3; k++)
      t[i][k] = f->rot[i][0] * h[0][k] + f->rot[i][1] * h[1][k] + f->rot[i][2] * h[2][k];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      out[i][j] = t[i][0] * f->rot[j][0] + t[i][1] * f->rot[j][1] + t[i][2] * f->rot[j][2];
}

/* ------------------------------------------------------------------------ */
/* pointwise kernel derivatives w.r.t. the source point                      */
/* d = source - target = (x-x0, y-y0, -z0)                                    */
/* rt[ix][iy][iz] = d^a (1/r), |a|<=2 ;  bt[..] = d^a r, |a|<=4              */
/* ------------------------------------------------------------------------ */
typedef struct { double r[3][3][3]; double b[5][5][5]; } tables_t;

static inline int kd(int a, int b) { return a == b; }

/* general index form: derivatives of radial functions */
static void point_tables(const double d[3], double w, int maxr, int maxb,
                         tables_t *acc) {
  double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  double r = sqrt(r2), ir = 1.0 / r, ir3 = ir * ir * ir, ir5 = ir3 * ir * ir,
         ir7 = ir5 * ir * ir;
  /* enumerate multi-indices via explicit index lists */
  for (int ix = 0; ix <= 4; ix++)
    for (int iy = 0; iy <= 4 - ix; iy++)
      for (int iz = 0; iz <= 4 - ix - iy; iz++) {
        int n = ix + iy + iz;
        int idx[4], k = 0;
        for (int q = 0; q < ix; q++) idx[k++] = 0;
        for (int q = 0; q < iy; q++) idx[k++] = 1;
        for (int q = 0; q < iz; q++) idx[k++] = 2;
        if (n <= maxb) {
          double v = 0;
          if (n == 0) v = r;
          else if (n == 1) v = d[idx[0]] * ir;
          else if (n == 2) {
            int i = idx[0], j = idx[1];
            v = kd(i, j) * ir - d[i] * d[j] * ir3;
          } else if (n == 3) {
            int i = idx[0], j = idx[1], l = idx[2];
            v = -(kd(i, j) * d[l] + kd(i, l) * d[j] + kd(j, l) * d[i]) * ir3 +
                3 * d[i] * d[j] * d[l] * ir5;
          } else {
            int i = idx[0], j = idx[1], l = idx[2], m = idx[3];
            v = -(kd(i, j) * kd(l, m) + kd(i, l) * kd(j, m) + kd(i, m) * kd(j, l)) * ir3 +
                3 * (kd(i, j) * d[l] * d[m] + kd(i, l) * d[j] * d[m] + kd(i, m) * d[j] * d[l] +
                     kd(j, l) * d[i] * d[m] + kd(j, m) * d[i] * d[l] + kd(l, m) * d[i] * d[j]) * ir5 -
                15 * d[i] * d[j] * d[l] * d[m] * ir7;
          }
          acc->b[ix][iy][iz] += w * v;
        }
        if (n <= maxr) {
          double v = 0;
          if (n == 0) v = ir;
          else if (n == 1) v = -d[idx[0]] * ir3;
          else {
            int i = idx[0], j = idx[1];
            v = 3 * d[i] * d[j] * ir5 - kd(i, j) * ir3;
          }
          acc->r[ix][iy][iz] += w * v;
        }
      }
}

/* homogeneity degree -k of each kernel family */
static inline int degk_b(int n) { return n - 1; }
static inline int degk_r(int n) { return n + 1; }

/* in-plane (h=0) fan contribution: kernel value at v (in-plane, target at
 * origin) times radial finite part weight */
static void fan_point_h0(const double v[2], double wt, int maxr, int maxb,
                         tables_t *acc) {
  double L = sqrt(v[0] * v[0] + v[1] * v[1]);
  double d[3] = {v[0], v[1], 0.0};
  tables_t tmp;
  memset(&tmp, 0, sizeof(tmp));
  point_tables(d, 1.0, maxr, maxb, &tmp);
  for (int ix = 0; ix <= 4; ix++)
    for (int iy = 0; iy <= 4 - ix; iy++)
      for (int iz = 0; iz <= 4 - ix - iy; iz++) {
        int n = ix + iy + iz;
        if (n <= maxb) {
          int k = degk_b(n);
          double c = (k == 2) ? log(L) : 1.0 / (2 - k);
          acc->b[ix][iy][iz] += wt * c * tmp.b[ix][iy][iz];
        }
        if (n <= maxr) {
          int k = degk_r(n);
          double c = (k == 2) ? log(L) : 1.0 / (2 - k);
          acc->r[ix][iy][iz] += wt * c * tmp.r[ix][iy][iz];
        }
      }
}

static void tables_zero(tables_t *t) { memset(t, 0, sizeof(*t)); }

/* breakpoints for a graded panel set on [0,1] clustered at point c */
static int graded_breaks(double c, double scale, double *bk, int maxb) {
  /* scale: length scale of the near-singular feature */
  int n = 0;
  bk[n++] = 0.0;
  double lo[40], hi[40];
  int nlo = 0, nhi = 0;
  if (scale < 1e-300) scale = 1e-300;
  for (double s = scale; s < 1.0 && nlo < 38; s *= 3.0) {
    if (c - s > 0) lo[nlo++] = c - s;
    if (c + s < 1) hi[nhi++] = c + s;
  }
  for (int i = nlo - 1; i >= 0; i--)
    if (lo[i] > bk[n - 1] && n < maxb - 2) bk[n++] = lo[i];
  if (c > 0 && c < 1 && n < maxb - 2) bk[n++] = c;
  for (int i = 0; i < nhi; i++)
    if (hi[i] > bk[n - 1] && n < maxb - 1) bk[n++] = hi[i];
  if (bk[n - 1] < 1.0) bk[n++] = 1.0;
  return n;
}

/* Gauss rule (collapsed 12x12) on a planar sub-triangle tv = (x1,y1,x2,y2,x3,y3) */
static void gauss_tri(const double *tv, double x0, double y0, double z0, int n,
                      int maxr, int maxb, tables_t *out) {
  double area2 = (tv[2] - tv[0]) * (tv[5] - tv[1]) - (tv[4] - tv[0]) * (tv[3] - tv[1]);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      double u = gl_x[n][i], t = gl_x[n][j];
      double a = u, b = (1 - u) * t;
      double w = gl_w[n][i] * gl_w[n][j] * (1 - u) * fabs(area2);
      double px = tv[0] + a * (tv[2] - tv[0]) + b * (tv[4] - tv[0]);
      double py = tv[1] + a * (tv[3] - tv[1]) + b * (tv[5] - tv[1]);
      double d[3] = {px - x0, py - y0, -z0};
      point_tables(d, w, maxr, maxb, out);
    }
}

/* adaptive 4-way subdivision until each piece is well separated from the
 * target (distance to the piece's centroid > 3 piece diameters) */
static void adapt_tri(const double *tv, double x0, double y0, double z0, int depth,
                      int maxr, int maxb, tables_t *out) {
  double cx = (tv[0] + tv[2] + tv[4]) / 3, cy = (tv[1] + tv[3] + tv[5]) / 3;
  double diam = 0;
  for (int i = 0; i < 3; i++) {
    int j = (i + 1) % 3;
    double l = hypot(tv[2 * j] - tv[2 * i], tv[2 * j + 1] - tv[2 * i + 1]);
    if (l > diam) diam = l;
  }
  double dist = sqrt((x0 - cx) * (x0 - cx) + (y0 - cy) * (y0 - cy) + z0 * z0);
  if (dist > 3.0 * diam || depth >= 40) {
    gauss_tri(tv, x0, y0, z0, 12, maxr, maxb, out);
    return;
  }
  double m01[2] = {(tv[0] + tv[2]) / 2, (tv[1] + tv[3]) / 2};
  double m12[2] = {(tv[2] + tv[4]) / 2, (tv[3] + tv[5]) / 2};
  double m20[2] = {(tv[4] + tv[0]) / 2, (tv[5] + tv[1]) / 2};
  double c0[6] = {tv[0], tv[1], m01[0], m01[1], m20[0], m20[1]};
  double c1[6] = {m01[0], m01[1], tv[2], tv[3], m12[0], m12[1]};
  double c2[6] = {m20[0], m20[1], m12[0], m12[1], tv[4], tv[5]};
  double c3[6] = {m12[0], m12[1], m20[0], m20[1], m01[0], m01[1]};
  adapt_tri(c0, x0, y0, z0, depth + 1, maxr, maxb, out);
  adapt_tri(c1, x0, y0, z0, depth + 1, maxr, maxb, out);
  adapt_tri(c2, x0, y0, z0, depth + 1, maxr, maxb, out);
  adapt_tri(c3, x0, y0, z0, depth + 1, maxr, maxb, out);
}

/* integrate the tables over the triangle (local 2d vertices v[3][2]) for the
 * target (x0,y0,z0).  self: force z0=0 (iquad=0 convention). */
void oracle_tables(const double v[3][2], double x0, double y0, double z0,
                   int self, int maxr, int maxb, tables_t *out) {
  gl_init();
  tables_zero(out);
  if (self) z0 = 0.0;
  double cx = (v[0][0] + v[1][0] + v[2][0]) / 3, cy = (v[0][1] + v[1][1] + v[2][1]) / 3;
  double diam = 0;
  for (int i = 0; i < 3; i++) {
    int j = (i + 1) % 3;
    double l = hypot(v[j][0] - v[i][0], v[j][1] - v[i][1]);
    if (l > diam) diam = l;
  }
  double dist = sqrt((x0 - cx) * (x0 - cx) + (y0 - cy) * (y0 - cy) + z0 * z0);
  double area2 = (v[1][0] - v[0][0]) * (v[2][1] - v[0][1]) -
                 (v[2][0] - v[0][0]) * (v[1][1] - v[0][1]);
  int inside = 0;
  {
    /* barycentric test of the projected target against the (CCW) triangle */
    double w0 = (v[1][0] - x0) * (v[2][1] - y0) - (v[2][0] - x0) * (v[1][1] - y0);
    double w1 = (v[2][0] - x0) * (v[0][1] - y0) - (v[0][0] - x0) * (v[2][1] - y0);
    double w2 = (v[0][0] - x0) * (v[1][1] - y0) - (v[1][0] - x0) * (v[0][1] - y0);
    inside = (w0 >= 0 && w1 >= 0 && w2 >= 0) || (w0 <= 0 && w1 <= 0 && w2 <= 0);
  }
  if (self) inside = 1;
  if (!self && !inside && dist <= 4.0 * diam) {
    /* projected target outside: the integrand is smooth on the triangle; use
     * adaptive 4-way subdivision with a Gauss rule on each piece */
    double tv[6] = {v[0][0], v[0][1], v[1][0], v[1][1], v[2][0], v[2][1]};
    adapt_tri(tv, x0, y0, z0, 0, maxr, maxb, out);
    return;
  }
  double hjump = 0.0; /* side of a near-coplanar interior target */
  if (!self && inside && z0 != 0.0 && fabs(z0) < 1e-8 * diam) {
    hjump = z0 > 0 ? 1.0 : -1.0;
    z0 = 0.0;
  }
  if (!self && dist > 4.0 * diam) {
    /* collapsed Gauss-Legendre (Duffy) on the triangle; the order falls with
     * distance (error ~ (diam/dist)^(2n), below 1e-15 in every band) */
    int n = dist > 100.0 * diam ? 5 : (dist > 25.0 * diam ? 7 : (dist > 10.0 * diam ? 10 : 20));
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        double u = gl_x[n][i], t = gl_x[n][j];
        double a = u, b = (1 - u) * t;
        double w = gl_w[n][i] * gl_w[n][j] * (1 - u) * fabs(area2);
        double px = v[0][0] + a * (v[1][0] - v[0][0]) + b * (v[2][0] - v[0][0]);
        double py = v[0][1] + a * (v[1][1] - v[0][1]) + b * (v[2][1] - v[0][1]);
        double d[3] = {px - x0, py - y0, -z0};
        point_tables(d, w, maxr, maxb, out);
      }
    return;
  }
  /* polar quadrature: fan triangles (P, A, B) for each edge */
  const int NG = 20;
  for (int e = 0; e < 3; e++) {
    double A[2] = {v[e][0] - x0, v[e][1] - y0};
    double B[2] = {v[(e + 1) % 3][0] - x0, v[(e + 1) % 3][1] - y0};
    double E[2] = {B[0] - A[0], B[1] - A[1]};
    double fan2 = A[0] * B[1] - A[1] * B[0]; /* 2*signed fan area */
    if (fan2 == 0.0 && z0 == 0.0) continue;
    double l2 = E[0] * E[0] + E[1] * E[1];
    double tperp = -(A[0] * E[0] + A[1] * E[1]) / l2; /* foot of perpendicular */
    double tc = tperp < 0 ? 0 : (tperp > 1 ? 1 : tperp);
    double Q[2] = {A[0] + tc * E[0], A[1] + tc * E[1]};
    double dseg = sqrt(Q[0] * Q[0] + Q[1] * Q[1]); /* distance P to segment */
    double tsc = dseg / sqrt(l2);
    double hsc = fabs(z0) / sqrt(l2);
    double tsc2 = tsc > hsc ? tsc : hsc;
    if (tsc2 <= 0) tsc2 = 1e-8;
    double bk[64];
    int nb = graded_breaks(tc, tsc2 > 1 ? 1 : tsc2, bk, 64);
    for (int p = 0; p + 1 < nb; p++) {
      double ta = bk[p], tb = bk[p + 1];
      if (tb <= ta) continue;
      for (int q = 0; q < NG; q++) {
        double t = ta + (tb - ta) * gl_x[NG][q];
        double wt = (tb - ta) * gl_w[NG][q];
        double V[2] = {A[0] + t * E[0], A[1] + t * E[1]};
        double L = sqrt(V[0] * V[0] + V[1] * V[1]);
        if (z0 == 0.0) {
          fan_point_h0(V, wt * fan2, maxr, maxb, out);
        } else {
          /* radial integral over s in [0,1], graded at s ~ |z0|/L */
          double s0 = fabs(z0) / L;
          double sb[64];
          int ns = graded_breaks(0.0, s0 > 1 ? 1 : s0, sb, 64);
          for (int r = 0; r + 1 < ns; r++) {
            double sa = sb[r], sbb = sb[r + 1];
            if (sbb <= sa) continue;
            for (int u = 0; u < NG; u++) {
              double s = sa + (sbb - sa) * gl_x[NG][u];
              double ws = (sbb - sa) * gl_w[NG][u];
              double d[3] = {s * V[0], s * V[1], -z0};
              point_tables(d, wt * ws * s * fan2, maxr, maxb, out);
            }
          }
        }
      }
    }
  }
  /* one-sided limits for an interior target at z0 -> 0+/-: the solid angle
   * int z0/r^3 -> +/-2 pi, and d^3/dz^3 int r = 2*solid angle - z0*(...)    */
  if (hjump != 0.0) {
    out->r[0][0][1] += hjump * 2 * M_PI;
    if (maxb >= 3) out->b[0][0][3] += hjump * 4 * M_PI;
  }
}

/* ------------------------------------------------------------------------ */
/* SLP / DLP assembly for one (triangle, target) pair                        */
/* elfmm3dtria.f:1689 (SLP) and :2368 (DLP)                                  */
/* ------------------------------------------------------------------------ */
#define B3(t, a, b, c) ((t)->b[a][b][c])
#define R3(t, a, b, c) ((t)->r[a][b][c])

static double Bidx(const tables_t *t, int n, const int *ix) {
  int c[3] = {0, 0, 0};
  for (int q = 0; q < n; q++) c[ix[q]]++;
  return t->b[c[0]][c[1]][c[2]];
}
static double Ridx(const tables_t *t, int n, const int *ix) {
  int c[3] = {0, 0, 0};
  for (int q = 0; q < n; q++) c[ix[q]]++;
  return t->r[c[0]][c[1]][c[2]];
}

/* single layer: u (3), strain (3x3) at target; sigma global (3) */
void oracle_slp_one(double rlam, double rmu, const double *tri, const double *sigma,
                    int self, const double *target, int ifstrain, double *u,
                    double *strain) {
  frame_t f;
  frame_init(tri, &f);
  double xl[3], sl[3];
  frame_fwd_pt(&f, target, xl);
  frame_fwd_vec(&f, sigma, sl);
  double c1 = (rlam + rmu) / (rlam + 2 * rmu);
  tables_t t;
  oracle_tables(f.v, xl[0], xl[1], xl[2], self, ifstrain ? 1 : 0, ifstrain ? 3 : 2, &t);
  double ul[3] = {0, 0, 0}, el[3][3];
  memset(el, 0, sizeof(el));
  for (int k = 0; k < 3; k++) {
    for (int i = 0; i < 3; i++) {
      int ik[2] = {i, k};
      double val = -c1 * Bidx(&t, 2, ik) + (i == k ? 2 * t.r[0][0][0] : 0.0);
      ul[i] += sl[k] * val;
    }
    if (ifstrain) {
      double m[3][3];
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
          int ijk[3] = {i, j, k};
          m[i][j] = -c1 * Bidx(&t, 3, ijk) + (i == k ? 2 * Ridx(&t, 1, &j) : 0.0);
        }
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) el[i][j] += sl[k] * 0.5 * (m[i][j] + m[j][i]);
    }
  }
  double ug[3];
  frame_bak_vec(&f, ul, ug);
  for (int i = 0; i < 3; i++) u[i] = ug[i] / (2 * rmu);
  if (ifstrain) {
    double eg[3][3];
    frame_bak_mat(&f, el, eg);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) strain[3 * j + i] = -eg[i][j] / (2 * rmu);
  }
}

/* double layer (normal = local +z of the triangle frame) */
void oracle_dlp_one(double rlam, double rmu, const double *tri, const double *sigma,
                    int self, const double *target, int ifstrain, double *u,
                    double *strain) {
  frame_t f;
  frame_init(tri, &f);
  double xl[3], sl[3];
  frame_fwd_pt(&f, target, xl);
  frame_fwd_vec(&f, sigma, sl);
  double c1 = (rlam + rmu) / (rlam + 2 * rmu);
  tables_t t;
  oracle_tables(f.v, xl[0], xl[1], xl[2], self, ifstrain ? 2 : 1, ifstrain ? 4 : 3, &t);
  /* U(i,k,m) = -c1 B(i+k+m) + 2 d_ik R(m) */
  double U[3][3][3];
  for (int i = 0; i < 3; i++)
    for (int k = 0; k < 3; k++)
      for (int m = 0; m < 3; m++) {
        int ikm[3] = {i, k, m};
        U[i][k][m] = -c1 * Bidx(&t, 3, ikm) + (i == k ? 2 * Ridx(&t, 1, &m) : 0.0);
      }
  /* T(a,k) = lam d_k3 sum_l U(l,a,l) + mu (U(k,a,3) + U(3,a,k)) */
  double ul[3] = {0, 0, 0};
  for (int a = 0; a < 3; a++)
    for (int k = 0; k < 3; k++) {
      double T = rmu * (U[k][a][2] + U[2][a][k]);
      if (k == 2) T += rlam * (U[0][a][0] + U[1][a][1] + U[2][a][2]);
      ul[a] += sl[k] * T;
    }
  double ug[3];
  frame_bak_vec(&f, ul, ug);
  for (int i = 0; i < 3; i++) u[i] = ug[i] / (2 * rmu);
  if (ifstrain) {
    double el[3][3];
    memset(el, 0, sizeof(el));
    for (int k = 0; k < 3; k++) {
      double S[3][3];
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
          /* D(i,k,j,m) = -c1 B(i+k+j+m) + 2 d_ik R(j+m) */
#define DD(i_, k_, j_, m_)                                                    \
  (-c1 * Bidx(&t, 4, (int[4]){i_, k_, j_, m_}) +                              \
   ((i_) == (k_) ? 2 * Ridx(&t, 2, (int[2]){j_, m_}) : 0.0))
          double s = rmu * (DD(k, a, 2, b) + DD(2, a, k, b));
          if (k == 2) s += rlam * (DD(0, a, 0, b) + DD(1, a, 1, b) + DD(2, a, 2, b));
          S[a][b] = s;
#undef DD
        }
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) el[a][b] += sl[k] * 0.5 * (S[a][b] + S[b][a]);
    }
    double eg[3][3];
    frame_bak_mat(&f, el, eg);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) strain[3 * j + i] = -eg[i][j] / (2 * rmu);
  }
}

/* raw tables for tests (flattened: r[27], b[125]) */
void oracle_tables_flat(const double *tri, const double *target, int self,
                        double *rflat, double *bflat) {
  frame_t f;
  frame_init(tri, &f);
  double xl[3];
  frame_fwd_pt(&f, target, xl);
  tables_t t;
  oracle_tables(f.v, xl[0], xl[1], xl[2], self, 2, 4, &t);
  memcpy(rflat, t.r, sizeof(t.r));
  memcpy(bflat, t.b, sizeof(t.b));
}

void oracle_frame(const double *tri, double *rot9, double *v6) {
  frame_t f;
  frame_init(tri, &f);
  for (int i = 0; i < 3; i++)
    for (int c = 0; c < 3; c++) rot9[3 * i + c] = f.rot[i][c];
  for (int i = 0; i < 3; i++) {
    v6[2 * i] = f.v[i][0];
    v6[2 * i + 1] = f.v[i][1];
  }
}

/* ------------------------------------------------------------------------ */
/* direct sum (el3dtriadirecttarg, elfmm3dtria.f:1483)                       */
/* arrays column-major as in Fortran: tri(3,3,n), sigma(3,n), pt(3,m)...      */
/* evaluation points: the n centroids `source` (self pairs: i == j) and the   */
/* ntarg targets.  Computes only rows [row0,row1) of the sources and          */
/* [trow0,trow1) of the targets (for bounded oracle runs).                    */
/* ------------------------------------------------------------------------ */
void oracle_direct(double rlam, double rmu, int n, const double *tri,
                   const double *source, int ifsingle, const double *sigma_sl,
                   int ifdouble, const double *sigma_dl, int ifptfrc, double *ptfrc,
                   int ifstrain, double *strain, int ntarg, const double *target,
                   int ifptfrctarg, double *ptfrctarg, int ifstraintarg,
                   double *straintarg, int row0, int row1, int trow0, int trow1) {
  gl_init();
  int tot = (row1 - row0) + (trow1 - trow0);
#pragma omp parallel for schedule(dynamic, 1)
  for (int q = 0; q < tot; q++) {
    int istarg = q >= (row1 - row0);
    int j = istarg ? trow0 + (q - (row1 - row0)) : row0 + q;
    const double *x = istarg ? target + 3 * j : source + 3 * j;
    int ifs = istarg ? ifstraintarg : ifstrain;
    int ifp = istarg ? ifptfrctarg : ifptfrc;
    if (!ifs && !ifp) continue;
    double uacc[3] = {0, 0, 0}, eacc[9];
    memset(eacc, 0, sizeof(eacc));
    for (int i = 0; i < n; i++) {
      int self = (!istarg && i == j);
      double u0[3], e0[9];
      if (ifsingle) {
        oracle_slp_one(rlam, rmu, tri + 9 * i, sigma_sl + 3 * i, self, x, ifs, u0, e0);
        for (int c = 0; c < 3; c++) uacc[c] += u0[c];
        if (ifs)
          for (int c = 0; c < 9; c++) eacc[c] += e0[c];
      }
      if (ifdouble) {
        oracle_dlp_one(rlam, rmu, tri + 9 * i, sigma_dl + 3 * i, self, x, ifs, u0, e0);
        for (int c = 0; c < 3; c++) uacc[c] += u0[c];
        if (ifs)
          for (int c = 0; c < 9; c++) eacc[c] += e0[c];
      }
    }
    double *pu = istarg ? ptfrctarg : ptfrc;
    double *pe = istarg ? straintarg : strain;
    if (ifp)
      for (int c = 0; c < 3; c++) pu[3 * j + c] = uacc[c];
    if (ifs)
      for (int c = 0; c < 9; c++) pe[9 * j + c] = eacc[c];
  }
}

/* ------------------------------------------------------------------------ */
/* oct-tree (d3tstrcr.f) -- bit-exact restatement                            */
/* ------------------------------------------------------------------------ */
typedef struct {
  int nboxes, nlev;
  int *boxes;      /* 20 ints per box, 1-based values exactly as d3tallbem   */
  int *iz, *iztarg;/* 1-based permutations                                    */
  int laddr[2 * 200];
  double center[3], size;
  /* lists 1..5 in CSR (1-based box ids), per box in insertion order         */
  int *lstart[6], *litems[6], lcount[6];
} otree_t;

static void d3t_centf(const double *c0, double size, int level, int i, int j, int k,
                      double *c) {
  /* d3tstrcr.f:1682 d3tcentf -- same expression order */
  double side = size / (double)(1 << level);
  double side2 = side / 2;
  double x0 = c0[0] - size / 2, y0 = c0[1] - size / 2, z0 = c0[2] - size / 2;
  c[0] = x0 + (i - 1) * side + side2;
  c[1] = y0 + (j - 1) * side + side2;
  c[2] = z0 + (k - 1) * side + side2;
}

/* stable partition of iz[0..n) by coordinate `dim` against thresh: <= first */
static int d3t_sepa0(const double *z, int *iz, int n, int dim, double thresh,
                     int *iwork) {
  int i1 = 0, i2 = 0;
  for (int i = 0; i < n; i++) {
    int j = iz[i];
    if (z[3 * (j - 1) + dim] > thresh) iwork[i2++] = j;
    else iz[i1++] = j;
  }
  for (int i = 0; i < i2; i++) iz[i1 + i] = iwork[i];
  return i1;
}

static void d3t_sepa1(const double *cent, const double *z, int *iz, int n, int *iwork,
                      int *is, int *ns) {
  int n1234 = 0, n5678, n12 = 0, n34, n56 = 0, n78, n1 = 0, n2, n3 = 0, n4, n5 = 0, n6,
      n7 = 0, n8;
  n1234 = d3t_sepa0(z, iz, n, 2, cent[2], iwork);
  n5678 = n - n1234;
  if (n1234) n12 = d3t_sepa0(z, iz, n1234, 1, cent[1], iwork);
  n34 = n1234 - n12;
  if (n5678) n56 = d3t_sepa0(z, iz + n1234, n5678, 1, cent[1], iwork);
  n78 = n5678 - n56;
  if (n12) n1 = d3t_sepa0(z, iz, n12, 0, cent[0], iwork);
  n2 = n12 - n1;
  if (n34) n3 = d3t_sepa0(z, iz + n12, n34, 0, cent[0], iwork);
  n4 = n34 - n3;
  if (n56) n5 = d3t_sepa0(z, iz + n1234, n56, 0, cent[0], iwork);
  n6 = n56 - n5;
  if (n78) n7 = d3t_sepa0(z, iz + n1234 + n56, n78, 0, cent[0], iwork);
  n8 = n78 - n7;
  int nn[8] = {n1, n2, n3, n4, n5, n6, n7, n8};
  is[0] = 1;
  ns[0] = nn[0];
  for (int i = 1; i < 8; i++) {
    is[i] = is[i - 1] + ns[i - 1];
    ns[i] = nn[i];
  }
}

#define BX(ib, f) boxes[20 * ((ib) - 1) + ((f) - 1)]

/* d3tallbem (d3tstrcr.f:1249); mindlin != 0 applies d3tstrcr_mindlin.f:1380 */
static int d3t_allbem(const double *z, int n, int nbox, const double *zt, int nt,
                      int mindlin, int *boxes, int maxboxes, int *nboxes_out,
                      int *iz, int *izt, int *laddr, int *nlev_out, double *c0,
                      double *size_out) {
  double xmin = z[0], xmax = z[0], ymin = z[1], ymax = z[1], zmin = z[2], zmax = z[2];
  for (int i = 0; i < n; i++) {
    const double *p = z + 3 * i;
    if (p[0] < xmin) xmin = p[0];
    if (p[0] > xmax) xmax = p[0];
    if (p[1] < ymin) ymin = p[1];
    if (p[1] > ymax) ymax = p[1];
    if (p[2] < zmin) zmin = p[2];
    if (p[2] > zmax) zmax = p[2];
  }
  for (int i = 0; i < nt; i++) {
    const double *p = zt + 3 * i;
    if (p[0] < xmin) xmin = p[0];
    if (p[0] > xmax) xmax = p[0];
    if (p[1] < ymin) ymin = p[1];
    if (p[1] > ymax) ymax = p[1];
    if (p[2] < zmin) zmin = p[2];
    if (p[2] > zmax) zmax = p[2];
  }
  double size = xmax - xmin, sizey = ymax - ymin, sizez = zmax - zmin;
  if (sizey > size) size = sizey;
  if (sizez > size) size = sizez;
  c0[0] = (xmin + xmax) / 2;
  c0[1] = (ymin + ymax) / 2;
  c0[2] = (zmin + zmax) / 2;
  if (mindlin) {
    double distz = fabs(zmin) > fabs(zmax) ? fabs(zmin) : fabs(zmax);
    c0[2] = 0;
    double sz = 2 * distz;
    if (sz > size) size = sz;
  }
  *size_out = size;
  for (int f = 1; f <= 20; f++) BX(1, f) = 0;
  BX(1, 2) = 1; BX(1, 3) = 1; BX(1, 4) = 1;
  BX(1, 14) = 1; BX(1, 15) = n; BX(1, 16) = 1; BX(1, 17) = nt;
  BX(1, 18) = n > 0 ? 1 : 0;
  BX(1, 19) = nt > 0 ? 1 : 0;
  laddr[0] = 1; laddr[1] = 1;
  for (int i = 0; i < n; i++) iz[i] = i + 1;
  for (int i = 0; i < nt; i++) izt[i] = i + 1;
  int iis[8] = {1, 2, 1, 2, 1, 2, 1, 2}, jjs[8] = {1, 1, 2, 2, 1, 1, 2, 2},
      kks[8] = {1, 1, 1, 1, 2, 2, 2, 2};
  int ison = 1, nlev = 0;
  int nw = (n > nt ? n : nt) + 4;
  int *iwork = (int *)malloc(sizeof(int) * nw);
  for (int level = 0; level < 198; level++) {
    laddr[2 * (level + 1)] = laddr[2 * level] + laddr[2 * level + 1];
    int nlevson = 0;
    int idad0 = laddr[2 * level], idad1 = idad0 + laddr[2 * level + 1] - 1;
    for (int idad = idad0; idad <= idad1; idad++) {
      int np = BX(idad, 15), ntd = BX(idad, 17);
      if (np <= nbox && ntd <= nbox) continue;
      if (BX(idad, 18) == 1) BX(idad, 18) = 2;
      if (BX(idad, 19) == 1) BX(idad, 19) = 2;
      int ii = BX(idad, 2), jj = BX(idad, 3), kk = BX(idad, 4);
      double cen[3];
      d3t_centf(c0, size, level, ii, jj, kk, cen);
      int iiz = BX(idad, 14), nz = BX(idad, 15), iit = BX(idad, 16), nzt = BX(idad, 17);
      int is[8], ns[8], ist[8], nst[8];
      d3t_sepa1(cen, z, iz + iiz - 1, nz, iwork, is, ns);
      d3t_sepa1(cen, zt, izt + iit - 1, nzt, iwork, ist, nst);
      int idadson = 6;
      for (int i = 0; i < 8; i++) {
        if (ns[i] == 0 && nst[i] == 0) continue;
        nlevson++;
        ison++;
        nlev = level + 1;
        if (ison > maxboxes) { free(iwork); return 4; }
        for (int f = 1; f <= 20; f++) BX(ison, f) = 0;
        BX(ison, 1) = level + 1;
        BX(ison, 2) = (ii - 1) * 2 + iis[i];
        BX(ison, 3) = (jj - 1) * 2 + jjs[i];
        BX(ison, 4) = (kk - 1) * 2 + kks[i];
        BX(ison, 5) = idad;
        BX(ison, 14) = is[i] + iiz - 1;
        BX(ison, 15) = ns[i];
        BX(ison, 16) = ist[i] + iit - 1;
        BX(ison, 17) = nst[i];
        BX(ison, 18) = ns[i] > 0 ? 1 : 0;
        BX(ison, 19) = nst[i] > 0 ? 1 : 0;
        BX(idad, idadson) = ison;
        idadson++;
      }
    }
    laddr[2 * (level + 1) + 1] = nlevson;
    if (nlevson == 0) break;
  }
  free(iwork);
  *nboxes_out = ison;
  *nlev_out = nlev;
  return 0;
}

/* simple growable per-box lists that keep insertion order */
typedef struct { int *a; int n, cap; } ivec_t;
static void iv_push(ivec_t *v, int x) {
  if (v->n == v->cap) {
    v->cap = v->cap ? 2 * v->cap : 8;
    v->a = (int *)realloc(v->a, sizeof(int) * v->cap);
  }
  v->a[v->n++] = x;
}

/* d3tifint (d3tstrcr.f:1082) on the box corners */
static void box_corner_min(const double *c0, double size, const int *boxes, int ib,
                           double *mn, double *side) {
  int level = BX(ib, 1);
  double s = size / (double)(1 << level);
  double x00 = c0[0] - size / 2, y00 = c0[1] - size / 2, z00 = c0[2] - size / 2;
  double cx = x00 + (BX(ib, 2) - 1) * s + s / 2;
  double cy = y00 + (BX(ib, 3) - 1) * s + s / 2;
  double cz = z00 + (BX(ib, 4) - 1) * s + s / 2;
  mn[0] = cx - s / 2;
  mn[1] = cy - s / 2;
  mn[2] = cz - s / 2;
  side[0] = mn[0] + s; side[1] = mn[1] + s; side[2] = mn[2] + s; /* maxima */
}

static int d3t_ifint(const double *c0, double size, const int *boxes, int b1, int b2) {
  double mn1[3], mx1[3], mn2[3], mx2[3];
  box_corner_min(c0, size, boxes, b1, mn1, mx1);
  box_corner_min(c0, size, boxes, b2, mn2, mx2);
  double eps = mx1[0] - mn1[0];
  if (eps > mx2[0] - mn2[0]) eps = mx2[0] - mn2[0];
  if (eps > mx2[1] - mn2[1]) eps = mx2[1] - mn2[1];
  if (eps > mx2[2] - mn2[2]) eps = mx2[2] - mn2[2];
  if (eps > mx1[1] - mn1[1]) eps = mx1[1] - mn1[1];
  if (eps > mx1[2] - mn1[2]) eps = mx1[2] - mn1[2];
  eps = eps / 10000;
  for (int d = 0; d < 3; d++) {
    if (mn1[d] > mx2[d] + eps) return 0;
    if (mn2[d] > mx1[d] + eps) return 0;
  }
  return 1;
}

static int nkids(const int *boxes, int ib) {
  int k = 0;
  for (int f = 6; f <= 13; f++)
    if (BX(ib, f) > 0) k++;
  return k;
}

/* d3tlst31 (d3tstrcr.f:919): DFS below colleague jbox0 of childless ibox */
static void d3t_lst31(const double *c0, double size, const int *boxes, int ibox,
                      int jbox0, ivec_t *L1, ivec_t *L3) {
  int stk_box[256], stk_n[256];
  int istack = 0;
  int jbox = jbox0;
  stk_box[0] = jbox;
  stk_n[0] = nkids(boxes, jbox);
  for (;;) {
    int ifint = d3t_ifint(c0, size, boxes, ibox, jbox);
    if (!ifint) {
      iv_push(&L3[ibox], jbox);
      istack--;
      stk_n[istack]--;
      jbox = stk_box[istack];
      continue;
    }
    if (BX(jbox, 6) == 0) {
      iv_push(&L1[ibox], jbox);
      if (BX(jbox, 1) != BX(ibox, 1)) iv_push(&L1[jbox], ibox);
      if (jbox == jbox0) return;
      istack--;
      stk_n[istack]--;
      jbox = stk_box[istack];
      continue;
    }
    int ns = stk_n[istack];
    if (ns == 0) {
      if (jbox == jbox0) return;
      istack--;
      stk_n[istack]--;
      jbox = stk_box[istack];
      continue;
    }
    jbox = BX(jbox, 5 + ns);
    istack++;
    stk_box[istack] = jbox;
    stk_n[istack] = nkids(boxes, jbox);
  }
}

/* The link store of d3tstrcr.f:1903-2350 hands lists back in insertion order
 * reversed twice (stored as a stack, flipped on retrieval) -- i.e. insertion
 * order.  We keep insertion order directly. */
static void d3t_lsts(const double *c0, double size, const int *boxes, int nboxes,
                     ivec_t *L[6]) {
  for (int ibox = 2; ibox <= nboxes; ibox++) {
    int idad = BX(ibox, 5);
    int ncoll = L[5][idad].n + 1;
    for (int i = 0; i < ncoll; i++) {
      int icoll = i == 0 ? idad : L[5][idad].a[i - 1];
      for (int j = 1; j <= 8; j++) {
        int kid = BX(icoll, 5 + j);
        if (kid <= 0) break;
        if (kid == ibox) continue;
        if (d3t_ifint(c0, size, boxes, kid, ibox)) iv_push(&L[5][ibox], kid);
        else iv_push(&L[2][ibox], kid);
      }
    }
  }
  for (int i = 1; i <= nboxes; i++) {
    if (BX(i, 6) > 0) continue;
    if (BX(i, 1) == 0) continue;
    int nl = L[5][i].n;
    for (int j = 0; j < nl; j++) d3t_lst31(c0, size, boxes, i, L[5][i].a[j], L[1], L[3]);
  }
  for (int ibox = 1; ibox <= nboxes; ibox++)
    for (int j = 0; j < L[3][ibox].n; j++) iv_push(&L[4][L[3][ibox].a[j]], ibox);
}

static otree_t *g_tree = 0;

/* build the tree and keep it; returns ier.  mindlin selects the half-space root. */
int oracle_tree_build(int n, const double *src, int nt, const double *targ, int nbox,
                      int mindlin) {
  if (g_tree) {
    free(g_tree->boxes); free(g_tree->iz); free(g_tree->iztarg);
    for (int t = 1; t <= 5; t++) { free(g_tree->lstart[t]); free(g_tree->litems[t]); }
    free(g_tree);
  }
  g_tree = (otree_t *)calloc(1, sizeof(otree_t));
  otree_t *T = g_tree;
  int maxboxes = 2 * (n + nt) + 64;
  T->boxes = (int *)calloc((size_t)20 * (maxboxes + 1), sizeof(int));
  T->iz = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  T->iztarg = (int *)malloc(sizeof(int) * (nt > 0 ? nt : 1));
  int ier = d3t_allbem(src, n, nbox, targ, nt, mindlin, T->boxes, maxboxes, &T->nboxes,
                       T->iz, T->iztarg, T->laddr, &T->nlev, T->center, &T->size);
  if (ier) return ier;
  ivec_t *L[6];
  for (int t = 1; t <= 5; t++) L[t] = (ivec_t *)calloc(T->nboxes + 1, sizeof(ivec_t));
  d3t_lsts(T->center, T->size, T->boxes, T->nboxes, L);
  for (int t = 1; t <= 5; t++) {
    int tot = 0;
    for (int b = 1; b <= T->nboxes; b++) tot += L[t][b].n;
    T->lstart[t] = (int *)malloc(sizeof(int) * (T->nboxes + 2));
    T->litems[t] = (int *)malloc(sizeof(int) * (tot > 0 ? tot : 1));
    T->lcount[t] = tot;
    int p = 0;
    for (int b = 1; b <= T->nboxes; b++) {
      T->lstart[t][b - 1] = p;
      for (int q = 0; q < L[t][b].n; q++) T->litems[t][p++] = L[t][b].a[q];
      free(L[t][b].a);
    }
    T->lstart[t][T->nboxes] = p;
    free(L[t]);
  }
  return 0;
}

void oracle_tree_info(int *nboxes, int *nlev, double *center, double *size,
                      int *lcounts) {
  *nboxes = g_tree->nboxes;
  *nlev = g_tree->nlev;
  for (int i = 0; i < 3; i++) center[i] = g_tree->center[i];
  *size = g_tree->size;
  for (int t = 1; t <= 5; t++) lcounts[t - 1] = g_tree->lcount[t];
}

void oracle_tree_get(int *boxes, int *iz, int *iztarg, int *laddr, int n, int nt,
                     int *lstart /* 5*(nboxes+1) */, int *litems /* sum lcounts */) {
  otree_t *T = g_tree;
  memcpy(boxes, T->boxes, sizeof(int) * 20 * T->nboxes);
  memcpy(iz, T->iz, sizeof(int) * n);
  memcpy(iztarg, T->iztarg, sizeof(int) * nt);
  memcpy(laddr, T->laddr, sizeof(int) * 2 * (T->nlev + 1));
  int off = 0;
  for (int t = 1; t <= 5; t++) {
    memcpy(lstart + (t - 1) * (T->nboxes + 1), T->lstart[t], sizeof(int) * (T->nboxes + 1));
    memcpy(litems + off, T->litems[t], sizeof(int) * T->lcount[t]);
    off += T->lcount[t];
  }
}
