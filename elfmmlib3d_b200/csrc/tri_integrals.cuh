// tri_integrals.cuh -- analytic near-field integrals over flat triangles.
//
// For a flat triangle T (in its own frame: plane z = 0, counter-clockwise
// vertices, normal +z) and a target X = (x, y, h), the elastostatic layer
// potentials need the source-derivative tables
//
//     R(a) = int_T d^a_src (1/r) dS   (|a| <= 2)
//     B(a) = int_T d^a_src (r)   dS   (|a| <= 4)
//
// (the reference's triartable/triabtable, src/triahquad.f:680 and :797).  The
// reference evaluates 51 separate integral types with per-type closed forms.
// This file uses a different, compact route:
//
//   * every derivative with an in-plane component a in {x, y} is moved onto
//     the boundary by the divergence theorem,
//         int_T d_a g dS = sum_edges m_a int_edge g dl   (m = outward normal),
//     leaving line integrals L1_e = int_e 1/r dl and Lr_e = int_e r dl whose
//     remaining target derivatives (up to third order) come from evaluating
//     their closed forms on Taylor jets (jets.cuh);
//   * pure normal derivatives follow from harmonicity of 1/r and from
//     d_h int r = h int 1/r, which needs only the triangle potential
//     Phi = int_T 1/r and the signed solid angle Omega = int_T h/r^3.
//
// On-surface evaluation (target on its own triangle) uses h = 0, Omega = 0: the
// principal value / Hadamard finite part, the reference's iquad = 0 convention
// (src/triahquad.f:4037-4055).  The line integrals use cancellation-free
// forms when both edge endpoints lie on the same side of the target's foot, so
// targets collinear with an edge (every centroid of a structured planar mesh)
// are exact.
#pragma once
#include "jets.cuh"

namespace efmm {

// Per-triangle geometry in the triangle's own frame (trilib.f:535 tri_ini):
// vertex 1 at the origin, edge 1->2 along +x, normal = (v2-v1)x(v3-v1)/|.|.
struct TriFrame {
  double e1[3], e2[3], e3[3];  // local axes in global coordinates
  double org[3];               // vertex 1
  double l1;                   // vertex 2 = (l1, 0)
  double v2x, v2y;             // vertex 3 = (v2x, v2y), v2y > 0
  double diam;                 // longest edge
};

EFMM_HD void tri_frame(const double* t, TriFrame& f) {
  double a[3] = {t[0], t[1], t[2]}, b[3] = {t[3], t[4], t[5]}, c[3] = {t[6], t[7], t[8]};
  double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  double l1 = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
  for (int i = 0; i < 3; i++) e1[i] /= l1;
  double w[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  double e3[3] = {e1[1] * w[2] - e1[2] * w[1], e1[2] * w[0] - e1[0] * w[2],
                  e1[0] * w[1] - e1[1] * w[0]};
  double l3 = sqrt(e3[0] * e3[0] + e3[1] * e3[1] + e3[2] * e3[2]);
  for (int i = 0; i < 3; i++) e3[i] /= l3;
  double e2[3] = {e3[1] * e1[2] - e3[2] * e1[1], e3[2] * e1[0] - e3[0] * e1[2],
                  e3[0] * e1[1] - e3[1] * e1[0]};
  for (int i = 0; i < 3; i++) {
    f.e1[i] = e1[i];
    f.e2[i] = e2[i];
    f.e3[i] = e3[i];
    f.org[i] = a[i];
  }
  f.l1 = l1;
  f.v2x = e1[0] * w[0] + e1[1] * w[1] + e1[2] * w[2];
  f.v2y = e2[0] * w[0] + e2[1] * w[1] + e2[2] * w[2];
  double l2 = sqrt((f.v2x - l1) * (f.v2x - l1) + f.v2y * f.v2y);
  double l3b = sqrt(f.v2x * f.v2x + f.v2y * f.v2y);
  f.diam = fmax(l1, fmax(l2, l3b));
}

// Derivative tables indexed by jidx: R up to order 2 (10), B up to order 4 (35)
struct TriTables {
  double R[10];
  double B[35];
};

// Line integrals over one edge A->B of int 1/r dl and int r dl as order-3 jets
// in the target coordinates (x, y, h).  Returns false if the target lies on
// the edge itself (singular; the reference returns 0 there, triahquad.f:1509).
EFMM_HD bool edge_jets(double ax, double ay, double bx, double by, double x0, double y0,
                       double h, Jet<3>& L1, Jet<3>& Lr, double& dsigned,
                       double& omega_part) {
  double ex = bx - ax, ey = by - ay;
  double len = sqrt(ex * ex + ey * ey);
  double tx = ex / len, ty = ey / len;
  double mx = ty, my = -tx;  // outward normal of a CCW polygon
  double u0 = (x0 - ax) * tx + (y0 - ay) * ty;
  double v0 = (x0 - ax) * mx + (y0 - ay) * my;
  dsigned = -v0;
  Jet<3> u = Jet<3>::affine(u0, tx, ty, 0.0);
  Jet<3> v = Jet<3>::affine(v0, mx, my, 0.0);
  Jet<3> H = Jet<3>::affine(h, 0.0, 0.0, 1.0);
  Jet<3> c2 = v * v + H * H;
  double sm = -u0, sp = len - u0;  // endpoint coordinates relative to the foot
  double c20 = v0 * v0 + h * h;

  // signed solid-angle contribution of this edge (h != 0 only)
  omega_part = 0.0;
  if (h != 0.0) {
    double d = dsigned, ah = fabs(h);
    double th[2];
    double ss[2] = {sm, sp};
    for (int q = 0; q < 2; q++) {
      double s = ss[q];
      double R = sqrt(s * s + d * d + h * h);
      double num = s * d * (s * s + d * d);
      double den = (R + ah) * (d * d * R + ah * s * s);
      th[q] = (den > 0.0) ? atan(num / den) : 0.0;
    }
    omega_part = th[1] - th[0];
  }

  bool same = (sm >= 0.0 && sp >= 0.0) || (sm <= 0.0 && sp <= 0.0);
  if (same) {
    double sg = (sm + sp >= 0.0) ? 1.0 : -1.0;
    if ((sg > 0 ? sm : -sp) == 0.0 && c20 == 0.0) return false;  // at a vertex
    // a = |s_-|, b = |s_+| as jets; b - a = sg*len exactly
    Jet<3> a = sg * (Jet<3>::constant(0.0) - u);
    Jet<3> b = a + sg * len;
    Jet<3> a2 = a * a, b2 = b * b;
    Jet<3> Ra = jsqrt(a2 + c2), Rb = jsqrt(b2 + c2);
    Jet<3> sab = a + b;
    // ln((b+Rb)/(a+Ra)) = log1p( sg*len*(1 + (a+b)/(Ra+Rb)) / (a+Ra) )
    Jet<3> q = (sg * len) * ((sab * jinv(Ra + Rb) + 1.0) * jinv(a + Ra));
    Jet<3> lr = jlog1p(q);
    L1 = sg * lr;
    // b Rb - a Ra = sg*len*(a+b)*(a^2+b^2+c^2)/(b Rb + a Ra)
    Jet<3> diff = (sg * len) * (sab * (a2 + b2 + c2) * jinv(b * Rb + a * Ra));
    Lr = 0.5 * (sg * diff + c2 * L1);
  } else {
    if (c20 == 0.0) return false;  // on the edge
    Jet<3> a = u;                                                   // a = -s_- = u
    Jet<3> b = Jet<3>::constant(len) - u;                          // b = s_+
    Jet<3> Ra = jsqrt(a * a + c2), Rb = jsqrt(b * b + c2);
    L1 = jlog(b + Rb) + jlog(a + Ra) - jlog(c2);
    Lr = 0.5 * (b * Rb + a * Ra + c2 * L1);
  }
  return true;
}

// Fill R (|a|<=2) and B (|a|<=4) for target (x0, y0, h) in the triangle frame.
// self: target is the triangle's own centroid (forces h = 0, Omega = 0).
EFMM_HD void tri_tables(const TriFrame& f, double x0, double y0, double h, bool self,
                        TriTables& T) {
  if (self) h = 0.0;
  for (int i = 0; i < 10; i++) T.R[i] = 0.0;
  for (int i = 0; i < 35; i++) T.B[i] = 0.0;
  double vx[3] = {0.0, f.l1, f.v2x}, vy[3] = {0.0, 0.0, f.v2y};
  double phi = 0.0, omega = 0.0, sh = 0.0;
#pragma unroll 1
  for (int e = 0; e < 3; e++) {
    int e2 = (e == 2) ? 0 : e + 1;
    double ax = vx[e], ay = vy[e], bx = vx[e2], by = vy[e2];
    Jet<3> L1, Lr;
    double ds, om;
    if (!edge_jets(ax, ay, bx, by, x0, y0, h, L1, Lr, ds, om)) continue;
    double ex = bx - ax, ey = by - ay;
    double len = sqrt(ex * ex + ey * ey);
    double m[2] = {ey / len, -ex / len};
    phi += ds * L1.c[0];
    omega += om;
    sh += m[0] * L1.deriv(1, 0, 1) + m[1] * L1.deriv(0, 1, 1);
    // in-plane entries: X(a) = sum_e m_d (-1)^(|a|-1) D^(a - e_d) L_e
    tables_edge(L1.c, Lr.c, m[0], m[1], T.R, T.B);
  }
  if (h == 0.0) omega = 0.0;
  else omega = (h > 0.0) ? omega : -omega;
  phi -= h * omega;
  double r002 = -(T.R[jidx(2, 0, 0)] + T.R[jidx(0, 2, 0)]);
  T.R[jidx(0, 0, 0)] = phi;
  T.R[jidx(0, 0, 1)] = omega;
  T.R[jidx(0, 0, 2)] = r002;
  T.B[jidx(0, 0, 1)] = -h * phi;
  T.B[jidx(0, 0, 2)] = phi - h * omega;
  T.B[jidx(0, 0, 3)] = 2.0 * omega - h * r002;
  T.B[jidx(0, 0, 4)] = 3.0 * r002 + h * sh;
}

// One (triangle, target) interaction in global coordinates.  ssl/sdl are the
// single/double layer densities already rotated into the triangle frame.
// The local-frame assembly (assemble_gen, generated) follows the single layer
// 2mu*u_i = sum_k s_k (2 d_ik R - c1 B_ik) (elfmm3dtria.f:1762-1987) and the
// traction-kernel contraction with the frame normal for the double layer
// (elfmm3dtria.f:2465-2911).  Outputs are ADDED to u[3] and e[6]
// (xx, yy, zz, xy, xz, yz); strain = -(rotated local gradient)/(2 mu).
EFMM_HD void pair_eval(const TriFrame& f, const double* ssl, const double* sdl, bool dosl,
                       bool dodl, bool dostrain, const double* X, bool self, double rlam,
                       double rmu, double* u, double* e) {
  double d[3] = {X[0] - f.org[0], X[1] - f.org[1], X[2] - f.org[2]};
  double x0 = f.e1[0] * d[0] + f.e1[1] * d[1] + f.e1[2] * d[2];
  double y0 = f.e2[0] * d[0] + f.e2[1] * d[1] + f.e2[2] * d[2];
  double h = f.e3[0] * d[0] + f.e3[1] * d[1] + f.e3[2] * d[2];
  TriTables T;
  tri_tables(f, x0, y0, h, self, T);
  double c1 = (rlam + rmu) / (rlam + 2.0 * rmu);
  double ul[3], el[6];
  assemble_gen(T.R, T.B, rlam, rmu, c1, ssl, sdl, dosl, dodl, dostrain, ul, el);
  double inv2mu = 0.5 / rmu;
#pragma unroll
  for (int i = 0; i < 3; i++)
    u[i] += inv2mu * (f.e1[i] * ul[0] + f.e2[i] * ul[1] + f.e3[i] * ul[2]);
  if (dostrain) {
    // G = Q el Q^T with Q = [e1 e2 e3]
    double E[3][3] = {{el[0], el[3], el[4]}, {el[3], el[1], el[5]}, {el[4], el[5], el[2]}};
    double t[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int k = 0; k < 3; k++)
        t[i][k] = f.e1[i] * E[0][k] + f.e2[i] * E[1][k] + f.e3[i] * E[2][k];
    const int ii[6] = {0, 1, 2, 0, 0, 1}, jj[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int q = 0; q < 6; q++) {
      int i = ii[q], j = jj[q];
      double g = t[i][0] * f.e1[j] + t[i][1] * f.e2[j] + t[i][2] * f.e3[j];
      e[q] -= inv2mu * g;
    }
  }
}

}  // namespace efmm
