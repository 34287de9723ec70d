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
 *   level <  0  refined by distance: a sub-triangle is split in four until
 *               the reflected target lies farther than 8 diameters from its
 *               centroid, at most 8 times.
 * and oracle_image_direct_adaptive integrates each pair and layer by the
 * adaptive scheme of the reference's tria3adam (src/tria3adamar.f:33-395):
 * the rule on a sub-triangle against the sum of the rule on its four
 * children, a sub-triangle accepted when every output agrees to eps times
 * the largest output of the parent estimate, depth-first with a depth cap.
 */
#include <math.h>
#include <stdlib.h>
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

/* the 12-node rule on sub-triangle (a, b, c) of one layer (0 force sl, 1
 * jump dl with normal nrm): out[9] = displacement (3), strain (6) */
static void image_rule(double lam, double mu, int layer, const double* nrm, const double* den, const double X[3],
                       const double* a, const double* b, const double* c, double B[12][3], const double W[12],
                       double out[9]) {
  const double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  const double v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  const double cr[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
  const double area = 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
  for (int r = 0; r < 9; r++) out[r] = 0.0;
  for (int q = 0; q < 12; q++) {
    double y[3], o[27];
    for (int d = 0; d < 3; d++) y[d] = B[q][0] * a[d] + B[q][1] * b[d] + B[q][2] * c[d];
    const double w = W[q] * area;
    if (layer == 0)
      oracle_image_sl(lam, mu, X[0], X[1], X[2], y[0], y[1], y[2], o);
    else
      oracle_image_dl(lam, mu, X[0], X[1], X[2], y[0], y[1], y[2], nrm[0], nrm[1], nrm[2], o);
    for (int k = 0; k < 3; k++)
      for (int r = 0; r < 9; r++) out[r] += w * den[k] * o[9 * k + r];
  }
}

enum { ADA_MAXDEPTH = 60, ADA_STACK = 3 * ADA_MAXDEPTH + 4 };

typedef struct {
  double v[9];
  double val[9];
  int depth;
} AdaSub;

/* one pair and layer, tria3adam's recursion; returns 1 if the depth cap
 * was reached somewhere (that sub-triangle's estimate is kept) */
static int image_pair_adaptive(double lam, double mu, int layer, const double* T, const double* nrm,
                               const double* den, const double X[3], double eps, int maxdepth, double B[12][3],
                               const double W[12], double acc[9]) {
  AdaSub* stk = (AdaSub*)malloc(sizeof(AdaSub) * ADA_STACK);
  int top = 1, capped = 0;
  memcpy(stk[0].v, T, sizeof(double) * 9);
  image_rule(lam, mu, layer, nrm, den, X, T, T + 3, T + 6, B, W, stk[0].val);
  stk[0].depth = 0;
  while (top > 0) {
    AdaSub s = stk[--top];
    if (s.depth >= maxdepth) {
      for (int r = 0; r < 9; r++) acc[r] += s.val[r];
      capped = 1;
      continue;
    }
    const double *a = s.v, *b = s.v + 3, *c = s.v + 6;
    double ab[3], bc[3], ca[3];
    for (int d = 0; d < 3; d++) {
      ab[d] = 0.5 * (a[d] + b[d]);
      bc[d] = 0.5 * (b[d] + c[d]);
      ca[d] = 0.5 * (c[d] + a[d]);
    }
    const double* kids[4][3] = {{a, ab, ca}, {ab, b, bc}, {ca, bc, c}, {ab, bc, ca}};
    double kv[4][9], sum[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < 4; k++) {
      image_rule(lam, mu, layer, nrm, den, X, kids[k][0], kids[k][1], kids[k][2], B, W, kv[k]);
      for (int r = 0; r < 9; r++) sum[r] += kv[k][r];
    }
    double dmax = 0.0;
    for (int r = 0; r < 9; r++) dmax = fmax(dmax, fabs(s.val[r]));
    int done = 1;
    for (int r = 0; r < 9; r++)
      if (fabs(sum[r] - s.val[r]) > eps * dmax) done = 0;
    if (done || top + 4 > ADA_STACK) {
      for (int r = 0; r < 9; r++) acc[r] += sum[r];
      if (!done) capped = 1;
      continue;
    }
    for (int k = 3; k >= 0; k--) {
      AdaSub t;
      for (int vtx = 0; vtx < 3; vtx++) memcpy(t.v + 3 * vtx, kids[k][vtx], sizeof(double) * 3);
      memcpy(t.val, kv[k], sizeof(double) * 9);
      t.depth = s.depth + 1;
      stk[top++] = t;
    }
  }
  free(stk);
  return capped;
}

/* Image displacement u (m, 3) and strain e (m, 3, 3) as oracle_image_direct,
 * every (target, triangle) pair and layer integrated adaptively to relative
 * tolerance eps with at most maxdepth (<= 60) halvings.  *ncapped = pairs
 * whose recursion reached the cap.  Returns 0, or 4 for bad arguments. */
int oracle_image_direct_adaptive(double lam, double mu, int n, const double* tri, const double* nrm,
                                 const double* ssl, const double* sdl, int m, const double* tgt, double eps,
                                 int maxdepth, double* u, double* e, int* ncapped) {
  if (maxdepth < 0 || maxdepth > ADA_MAXDEPTH || !(eps > 0)) return 4;
  double B[12][3], W[12];
  quad12(B, W);
  int capped = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : capped)
  for (int i = 0; i < m; i++) {
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const double* X = tgt + 3 * (size_t)i;
    for (int t = 0; t < n; t++) {
      const double* T = tri + 9 * (size_t)t;
      const double* nt = nrm + 3 * (size_t)t;
      if (ssl) capped += image_pair_adaptive(lam, mu, 0, T, nt, ssl + 3 * (size_t)t, X, eps, maxdepth, B, W, acc);
      if (sdl) capped += image_pair_adaptive(lam, mu, 1, T, nt, sdl + 3 * (size_t)t, X, eps, maxdepth, B, W, acc);
    }
    for (int d = 0; d < 3; d++) u[3 * (size_t)i + d] = acc[d];
    double* E = e + 9 * (size_t)i;
    E[0] = acc[3];
    E[4] = acc[4];
    E[8] = acc[5];
    E[1] = E[3] = acc[6];
    E[2] = E[6] = acc[7];
    E[5] = E[7] = acc[8];
  }
  if (ncapped) *ncapped = capped;
  return 0;
}
