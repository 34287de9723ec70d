/*
 * image.c -- CPU FP64 oracle: image part of the Mindlin half-space layer
 * potentials, summed directly over every (target, triangle) pair.
 *
 * TEST INFRASTRUCTURE ONLY (the same rules as oracle.c: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU legs use it, as the checker or
 * as the timed CPU stand-in for the reference).
 *
 * The reference evaluates the image part of its half-space potentials
 * (src/elhfmm3dtria_iter.f:46, the Mindlin image src/el3greenh.f:643-787)
 * by quadrature of the image kernels on each triangle, refined adaptively
 * (src/tria3adamar.f:16-548).  Here the kernels are image_gen.h, printed by
 * gen_image_c.py from oracle/mindlin.py's symbolic expressions, and each
 * pair is integrated with the 12-node degree-6 symmetric rule on
 * sub-triangles:
 *   level >= 0  every triangle split into 4**level congruent sub-triangles
 *               (the numpy oracle mindlin.image_direct: the same sums, in
 *               another rounding order);
 *   level <  0  adaptive: a sub-triangle is split in four until the reflected
 *               target lies farther than 8 diameters from its centroid, at
 *               most 8 times.
 */
#include <math.h>
#include <string.h>

#include "image_gen.h"

/* 12-node degree-6 symmetric rule, barycentric nodes, weights summing to 1 */
static void quad12(double B[12][3], double W[12]) {
  const double a1 = 0.2492867451709104212916386, w1 = 0.1167862757263793660252896;
  const double a2 = 0.0630890144915022283403316, w2 = 0.05084490637020681692093681;
  const double b3 = 0.05314504984481694735324967, c3 = 0.3103524510337844054166077;
  const double w3 = 0.08285107561837357519355346;
  int q = 0;
  const double as[2] = {a1, a2}, ws[2] = {w1, w2};
  for (int r = 0; r < 2; r++) {
    const double a = as[r], o = 1 - 2 * a;
    const double p[3][3] = {{o, a, a}, {a, o, a}, {a, a, o}};
    for (int k = 0; k < 3; k++, q++) {
      for (int v = 0; v < 3; v++) B[q][v] = p[k][v];
      W[q] = ws[r];
    }
  }
  const double o = 1 - b3 - c3;
  const double p[6][3] = {{o, b3, c3}, {o, c3, b3}, {b3, o, c3}, {c3, o, b3}, {b3, c3, o}, {c3, b3, o}};
  for (int k = 0; k < 6; k++, q++) {
    for (int v = 0; v < 3; v++) B[q][v] = p[k][v];
    W[q] = w3;
  }
}

enum { IMG_MAXDEPTH = 8, IMG_MAXLEVEL = 12, IMG_STACK = 3 * IMG_MAXLEVEL + 1 };
static const double IMG_RATIO = 8.0;

typedef struct {
  double v[9];
  int depth;
} ImgSub;

/* one (target, triangle) pair: acc[9] += displacement (3) and strain
 * (xx yy zz xy xz yz) of the densities sl (force) and dl (jump) */
static void image_pair(double lam, double mu, const double* T, const double* nrm, const double* sl,
                       const double* dl, const double X[3], int level, double B[12][3], const double W[12],
                       double acc[9]) {
  const double Xr[3] = {X[0], X[1], -X[2]};
  const int maxdepth = level >= 0 ? level : IMG_MAXDEPTH;
  /* depth-first: at most 3 pending siblings per level plus the current one */
  ImgSub stk[IMG_STACK];
  int top = 1;
  memcpy(stk[0].v, T, sizeof(double) * 9);
  stk[0].depth = 0;
  while (top > 0) {
    const ImgSub s = stk[--top];
    const double *a = s.v, *b = s.v + 3, *c = s.v + 6;
    int leaf = s.depth >= maxdepth;
    if (!leaf && level < 0) {
      double cen[3], e0 = 0, e1 = 0, e2 = 0, d2 = 0;
      for (int d = 0; d < 3; d++) {
        cen[d] = (a[d] + b[d] + c[d]) / 3.0;
        e0 += (b[d] - a[d]) * (b[d] - a[d]);
        e1 += (c[d] - b[d]) * (c[d] - b[d]);
        e2 += (a[d] - c[d]) * (a[d] - c[d]);
        d2 += (Xr[d] - cen[d]) * (Xr[d] - cen[d]);
      }
      const double diam2 = fmax(e0, fmax(e1, e2));
      leaf = d2 > IMG_RATIO * IMG_RATIO * diam2;
    }
    if (leaf) {
      const double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
      const double v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
      const double cr[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
      const double area = 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
      for (int q = 0; q < 12; q++) {
        double y[3], o[27];
        for (int d = 0; d < 3; d++) y[d] = B[q][0] * a[d] + B[q][1] * b[d] + B[q][2] * c[d];
        const double w = W[q] * area;
        if (sl) {
          oracle_image_sl(lam, mu, X[0], X[1], X[2], y[0], y[1], y[2], o);
          for (int k = 0; k < 3; k++)
            for (int r = 0; r < 9; r++) acc[r] += w * sl[k] * o[9 * k + r];
        }
        if (dl) {
          oracle_image_dl(lam, mu, X[0], X[1], X[2], y[0], y[1], y[2], nrm[0], nrm[1], nrm[2], o);
          for (int k = 0; k < 3; k++)
            for (int r = 0; r < 9; r++) acc[r] += w * dl[k] * o[9 * k + r];
        }
      }
    } else {
      double ab[3], bc[3], ca[3];
      for (int d = 0; d < 3; d++) {
        ab[d] = 0.5 * (a[d] + b[d]);
        bc[d] = 0.5 * (b[d] + c[d]);
        ca[d] = 0.5 * (c[d] + a[d]);
      }
      const double* kids[4][3] = {{a, ab, ca}, {ab, b, bc}, {ca, bc, c}, {ab, bc, ca}};
      /* pushed in reverse: summed a-corner, b-corner, c-corner, middle */
      for (int k = 3; k >= 0; k--) {
        ImgSub t;
        for (int vtx = 0; vtx < 3; vtx++) memcpy(t.v + 3 * vtx, kids[k][vtx], sizeof(double) * 3);
        t.depth = s.depth + 1;
        stk[top++] = t;
      }
    }
  }
}

/* Image displacement u (m, 3) and strain e (m, 3, 3) at targets tgt (m, 3),
 * all in z < 0, of densities on triangles tri (n, 3, 3) with normals nrm
 * (n, 3): single layer ssl (n, 3), double layer sdl (n, 3); a NULL density
 * disables its layer.  level as in the file header (0..12 or < 0).  Targets
 * are shared among the host's threads.  Returns 0, or 4 for a bad level. */
int oracle_image_direct(double lam, double mu, int n, const double* tri, const double* nrm, const double* ssl,
                        const double* sdl, int m, const double* tgt, int level, double* u, double* e) {
  if (level > IMG_MAXLEVEL) return 4;
  double B[12][3], W[12];
  quad12(B, W);
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < m; i++) {
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int t = 0; t < n; t++)
      image_pair(lam, mu, tri + 9 * (size_t)t, nrm + 3 * (size_t)t, ssl ? ssl + 3 * (size_t)t : NULL,
                 sdl ? sdl + 3 * (size_t)t : NULL, tgt + 3 * (size_t)i, level, B, W, acc);
    for (int d = 0; d < 3; d++) u[3 * (size_t)i + d] = acc[d];
    double* E = e + 9 * (size_t)i;
    E[0] = acc[3];
    E[4] = acc[4];
    E[8] = acc[5];
    E[1] = E[3] = acc[6];
    E[2] = E[6] = acc[7];
    E[5] = E[7] = acc[8];
  }
  return 0;
}

/* One kernel evaluation (layer 0: the three unit point forces, 1: the three
 * unit jumps with normal nrm) at target x from source s: out[27] as in
 * image_gen.h.  Returns 0, or 4 for a bad layer. */
int oracle_image_kernel(int layer, double lam, double mu, const double* x, const double* s, const double* nrm,
                        double* out) {
  if (layer == 0)
    oracle_image_sl(lam, mu, x[0], x[1], x[2], s[0], s[1], s[2], out);
  else if (layer == 1)
    oracle_image_dl(lam, mu, x[0], x[1], x[2], s[0], s[1], s[2], nrm[0], nrm[1], nrm[2], out);
  else
    return 4;
  return 0;
}
