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
//     leaving line integrals L1_e = int_e 1/r dl and Lr_e = int_e r dl;
//   * a line integral depends on the target only through the endpoint
//     distances and c^2 = v^2 + h^2 (v, h: in-plane normal and normal offsets
//     from the edge line), so its derivatives are endpoint terms (derivatives
//     along the edge) and derivatives of F(c^2), which need only the three
//     integrals K_n = int (s^2 + c^2)^(-n/2) ds, n = 1, 3, 5, in closed form;
//     the rotation from the edge frame to the triangle frame is generated
//     (gen_edge.py -> edge_gen.cuh);
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
#include <math.h>
#include "tri_index.cuh"
#include "assemble_gen.cuh"
#include "edge_gen.cuh"

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

// Edge-frame derivatives of the line integrals over one edge of length len
// lying on the u axis from u = 0 (vertex A) to u = len (vertex B), for a target
// at (u0, v0, h): L1[jidx(i,j,k)] = d_u^i d_v^j d_h^k int 1/r dl (|b| <= 2) and
// Lr[...] = the same of int r dl (1 <= |b| <= 3).  Returns false when the
// target lies on the closed edge (singular; the reference returns 0 there,
// src/triahquad.f:1509).
EFMM_HD bool edge_derivs(double len, double u0, double v0, double h, double* L1, double* Lr) {
  const double sm = -u0, sp = len - u0;  // endpoint coordinates relative to the foot
  const double c2 = v0 * v0 + h * h;
  const double RA = sqrt(u0 * u0 + c2), RB = sqrt(sp * sp + c2);
  // antiderivatives on [0, inf) shifted to vanish at infinity:
  //   int (w^2+c^2)^-3/2 = -1/(R (w+R)),
  //   int (w^2+c^2)^-5/2 = -(3w^2+4c^2) / (3 R^3 (w (2w^2+3c^2) + 2 R^3))
  auto A3 = [c2](double w, double R) { return -1.0 / (R * (w + R)); };
  auto A5 = [c2](double w, double R) {
    return -(3.0 * w * w + 4.0 * c2) / (3.0 * R * R * R * (w * (2.0 * w * w + 3.0 * c2) + 2.0 * R * R * R));
  };
  double K1, K3, K5;
  if ((sm >= 0.0 && sp >= 0.0) || (sm <= 0.0 && sp <= 0.0)) {
    // both endpoints on one side of the foot: cancellation-free forms
    const double sg = (sm + sp >= 0.0) ? 1.0 : -1.0;
    const double a = sg * sm, b = sg * sp;  // |s_-|, |s_+|; b - a = sg*len
    if (fmin(a, b) == 0.0 && c2 == 0.0) return false;  // at a vertex
    // ln((b+RB)/(a+RA)) with (b+RB)-(a+RA) = sg*len*(1 + (a+b)/(RA+RB))
    K1 = sg * log1p(sg * len * (1.0 + (a + b) / (RA + RB)) / (a + RA));
    K3 = sg * (A3(b, RB) - A3(a, RA));
    K5 = sg * (A5(b, RB) - A5(a, RA));
  } else {
    if (c2 == 0.0) return false;  // on the edge
    const double a = u0, b = sp;   // both > 0, split at the foot
    K1 = log((b + RB) * (a + RA) / c2);
    K3 = A3(b, RB) + A3(a, RA) + 2.0 / c2;
    K5 = A5(b, RB) + A5(a, RA) + 4.0 / (3.0 * c2 * c2);
  }
  const double iA = 1.0 / RA, iB = 1.0 / RB;
  const double iA3 = iA * iA * iA, iB3 = iB * iB * iB;
  const double ub = u0 - len;  // u-coordinate of the target relative to B
  // int 1/r dl: F(c^2) part (d/dc^2: -K3/2, 3 K5/4) and endpoint part 1/r
  {
    const double F1 = -0.5 * K3, F2 = 0.75 * K5;
    L1[jidx(0, 0, 0)] = K1;
    L1[jidx(0, 1, 0)] = 2.0 * v0 * F1;
    L1[jidx(0, 0, 1)] = 2.0 * h * F1;
    L1[jidx(0, 2, 0)] = 2.0 * F1 + 4.0 * v0 * v0 * F2;
    L1[jidx(0, 1, 1)] = 4.0 * v0 * h * F2;
    L1[jidx(0, 0, 2)] = 2.0 * F1 + 4.0 * h * h * F2;
    L1[jidx(1, 0, 0)] = iA - iB;
    L1[jidx(2, 0, 0)] = -u0 * iA3 + ub * iB3;
    L1[jidx(1, 1, 0)] = -v0 * (iA3 - iB3);
    L1[jidx(1, 0, 1)] = -h * (iA3 - iB3);
  }
  // int r dl: F(c^2) part (K1/2, -K3/4, 3 K5/8) and endpoint part r
  {
    const double F1 = 0.5 * K1, F2 = -0.25 * K3, F3 = 0.375 * K5;
    Lr[jidx(0, 1, 0)] = 2.0 * v0 * F1;
    Lr[jidx(0, 0, 1)] = 2.0 * h * F1;
    Lr[jidx(0, 2, 0)] = 2.0 * F1 + 4.0 * v0 * v0 * F2;
    Lr[jidx(0, 1, 1)] = 4.0 * v0 * h * F2;
    Lr[jidx(0, 0, 2)] = 2.0 * F1 + 4.0 * h * h * F2;
    Lr[jidx(0, 3, 0)] = 12.0 * v0 * F2 + 8.0 * v0 * v0 * v0 * F3;
    Lr[jidx(0, 2, 1)] = 4.0 * h * F2 + 8.0 * v0 * v0 * h * F3;
    Lr[jidx(0, 1, 2)] = 4.0 * v0 * F2 + 8.0 * v0 * h * h * F3;
    Lr[jidx(0, 0, 3)] = 12.0 * h * F2 + 8.0 * h * h * h * F3;
    // RA - RB without cancellation: (RA^2 - RB^2) / (RA + RB)
    Lr[jidx(1, 0, 0)] = len * (2.0 * u0 - len) / (RA + RB);
    Lr[jidx(2, 0, 0)] = u0 * iA - ub * iB;
    Lr[jidx(1, 1, 0)] = v0 * (iA - iB);
    Lr[jidx(1, 0, 1)] = h * (iA - iB);
    // second derivatives of r: d_ab r = delta_ab / r - P_a P_b / r^3
    Lr[jidx(3, 0, 0)] = (iA - u0 * u0 * iA3) - (iB - ub * ub * iB3);
    Lr[jidx(2, 1, 0)] = -v0 * (u0 * iA3 - ub * iB3);
    Lr[jidx(2, 0, 1)] = -h * (u0 * iA3 - ub * iB3);
    Lr[jidx(1, 2, 0)] = (iA - v0 * v0 * iA3) - (iB - v0 * v0 * iB3);
    Lr[jidx(1, 1, 1)] = -v0 * h * (iA3 - iB3);
    Lr[jidx(1, 0, 2)] = (iA - h * h * iA3) - (iB - h * h * iB3);
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
    const double ax = vx[e], ay = vy[e];
    const double ex = vx[e2] - ax, ey = vy[e2] - ay;
    const double len = sqrt(ex * ex + ey * ey);
    const double tx = ex / len, ty = ey / len;  // unit tangent; outward normal (ty, -tx)
    const double u0 = (x0 - ax) * tx + (y0 - ay) * ty;
    const double v0 = (x0 - ax) * ty - (y0 - ay) * tx;
    double L1[10], Lr[20];
    if (!edge_derivs(len, u0, v0, h, L1, Lr)) continue;
    // signed solid-angle contribution of this edge (h != 0 only)
    if (h != 0.0) {
      const double d = -v0, ah = fabs(h);
      const double ss[2] = {-u0, len - u0};
      double th[2];
      for (int q = 0; q < 2; q++) {
        const double s = ss[q];
        const double R = sqrt(s * s + d * d + h * h);
        const double num = s * d * (s * s + d * d);
        const double den = (R + ah) * (d * d * R + ah * s * s);
        th[q] = (den > 0.0) ? atan(num / den) : 0.0;
      }
      omega += th[1] - th[0];
    }
    phi += -v0 * L1[0];
    edge_tables_gen(tx, ty, L1, Lr, T.R, T.B, sh);
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

// Rotate local-frame outputs (ul: displacement, el: symmetric strain xx yy zz
// xy xz yz, both before the 1/(2 mu) and strain-sign factors) to the global
// frame and ADD them to u[3], e[6].
EFMM_HD void rotate_add(const TriFrame& f, const double* ul, const double* el, bool dostrain,
                        double inv2mu, double* u, double* e) {
#pragma unroll
  for (int i = 0; i < 3; i++)
    u[i] += inv2mu * (f.e1[i] * ul[0] + f.e2[i] * ul[1] + f.e3[i] * ul[2]);
  if (dostrain) {
    // G = Q el Q^T with Q = [e1 e2 e3]; strain = -G / (2 mu)
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

EFMM_HD void pair_local(const TriFrame& f, const double* X, bool self, TriTables& T) {
  double d[3] = {X[0] - f.org[0], X[1] - f.org[1], X[2] - f.org[2]};
  double x0 = f.e1[0] * d[0] + f.e1[1] * d[1] + f.e1[2] * d[2];
  double y0 = f.e2[0] * d[0] + f.e2[1] * d[1] + f.e2[2] * d[2];
  double h = f.e3[0] * d[0] + f.e3[1] * d[1] + f.e3[2] * d[2];
  tri_tables(f, x0, y0, h, self, T);
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
  TriTables T;
  pair_local(f, X, self, T);
  double c1 = (rlam + rmu) / (rlam + 2.0 * rmu);
  double ul[3], el[6];
  assemble_gen(T.R, T.B, rlam, rmu, c1, ssl, sdl, dosl, dodl, dostrain, ul, el);
  rotate_add(f, ul, el, dostrain, 0.5 / rmu, u, e);
}

// Response of one (triangle, target) pair to unit densities along the global
// axes, the stored near-field operator of the ITER mode
// (src/elfmm3dtria_iter_1.f:1559-1760 stores the same three unit responses):
// for each enabled layer (single, then double) and direction k = x, y, z the
// displacement (3 doubles, if dodisp) and strain (6, if dostrain) in global
// coordinates.  Returns the number of doubles written to out.
EFMM_HD int pair_blocks(const TriFrame& f, bool dosl, bool dodl, bool dodisp, bool dostrain,
                        const double* X, bool self, double rlam, double rmu, double* out) {
  TriTables T;
  pair_local(f, X, self, T);
  double c1 = (rlam + rmu) / (rlam + 2.0 * rmu);
  double inv2mu = 0.5 / rmu;
  const double zero[3] = {0.0, 0.0, 0.0};
  int w = 0;
  for (int layer = 0; layer < 2; layer++) {
    if ((layer == 0 && !dosl) || (layer == 1 && !dodl)) continue;
    for (int k = 0; k < 3; k++) {
      const double s[3] = {f.e1[k], f.e2[k], f.e3[k]};  // global e_k in the triangle frame
      double ul[3], el[6];
      assemble_gen(T.R, T.B, rlam, rmu, c1, layer == 0 ? s : zero, layer == 1 ? s : zero,
                   layer == 0, layer == 1, dostrain, ul, el);
      double u[3] = {0, 0, 0}, e[6] = {0, 0, 0, 0, 0, 0};
      rotate_add(f, ul, el, dostrain, inv2mu, u, e);
      if (dodisp) {
        out[w] = u[0]; out[w + 1] = u[1]; out[w + 2] = u[2];
        w += 3;
      }
      if (dostrain) {
        for (int q = 0; q < 6; q++) out[w + q] = e[q];
        w += 6;
      }
    }
  }
  return w;
}

}  // namespace efmm
