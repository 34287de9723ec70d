// particles.cu -- the near field and the direct sum of the elastostatic
// particle FMM (src/elfmm3dpart.f: elfmm3dpart / elfmm3dparttarg /
// el3dpartdirecttarg): point forces sigma_sl and point displacement
// discontinuities sigma_dl with orientations sigma_dv at the sources,
// displacement and strain at the sources (self-interaction excluded) and at
// targets.
//
// The particle FMM shares the tree, translations and L2T of the triangle
// FMM; its P2M is k_p2m with one node per source (fmm.cu).  The near field
// uses the same canonical decomposition as the far field, applied pair by
// pair: each source carries, per pass q (three Cartesian passes and the
// linear one), a charge and a dipole (src/elfmm3dpart.f:319-420, the
// formulas of k_p2m); the near sources' Laplace potential, gradient and
// Hessian are summed per pass at the evaluation point, and the Lame
// recombination of the L2T (u_a = (2 - c1) phi_a - c1 x_j d_a phi_j +
// d_a Phi_4, strain the symmetric part of its gradient) turns them into
// displacement and strain.  Laplace kernels: phi = q / r + d . rho / r^3,
// rho = x - y (the dipole convention of the multipole expansions).
#include "common.cuh"
#include "kernels.h"
#include "particles.h"

namespace efmm {

// charges q[4] and dipoles d[4][3] of one source (passes 0..2: the force
// and jump components, 3: the linear pass), as k_p2m forms them
EFMM_HD void part_terms(const double y[3], const double sl[3], const double dl[3], const double nu[3],
                               double c1, double c2, double inv2mu, double q[4], double d[4][3]) {
  for (int j = 0; j < 3; j++) {
    q[j] = sl[j] * inv2mu;
    for (int c = 0; c < 3; c++) d[j][c] = 0.5 * (nu[c] * dl[j] + dl[c] * nu[j]);
  }
  const double sly = sl[0] * y[0] + sl[1] * y[1] + sl[2] * y[2];
  const double dly = dl[0] * y[0] + dl[1] * y[1] + dl[2] * y[2];
  const double dln = dl[0] * nu[0] + dl[1] * nu[1] + dl[2] * nu[2];
  const double ny = nu[0] * y[0] + nu[1] * y[1] + nu[2] * y[2];
  q[3] = sly * c1 * inv2mu + dln * c2;
  for (int c = 0; c < 3; c++) d[3][c] = 0.5 * c1 * (nu[c] * dly + dl[c] * ny);
}

// acc[10 q + (0: phi, 1..3: gradient, 4..9: Hessian xx yy zz xy xz yz)] +=
// the Laplace fields at x of the source at y; nothing for coincident points
EFMM_HD void part_pair(const double x[3], const double y[3], const double q[4], const double d[4][3],
                              double* acc) {
  const double r0 = x[0] - y[0], r1 = x[1] - y[1], r2 = x[2] - y[2];
  const double rr = r0 * r0 + r1 * r1 + r2 * r2;
  if (rr == 0.0) return;
  const double ir = 1.0 / sqrt(rr), ir2 = ir * ir, ir3 = ir * ir2, ir5 = ir3 * ir2, ir7 = ir5 * ir2;
  const double rho[3] = {r0, r1, r2};
  for (int k = 0; k < 4; k++) {
    const double qq = q[k];
    const double dr = d[k][0] * r0 + d[k][1] * r1 + d[k][2] * r2;
    double* o = acc + 10 * k;
    o[0] += qq * ir + dr * ir3;
    for (int a = 0; a < 3; a++) o[1 + a] += -qq * rho[a] * ir3 + d[k][a] * ir3 - 3.0 * dr * rho[a] * ir5;
    const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
    for (int h = 0; h < 6; h++) {
      const int a = ia[h], b = ib[h];
      const double dab = a == b ? 1.0 : 0.0;
      o[4 + h] += qq * (3.0 * rho[a] * rho[b] * ir5 - dab * ir3) - 3.0 * (d[k][a] * rho[b] + d[k][b] * rho[a]) * ir5 -
                  3.0 * dr * dab * ir5 + 15.0 * dr * rho[a] * rho[b] * ir7;
    }
  }
}

// the Lame recombination of the four passes' fields at x (as k_l2t): u[3],
// strain e6 (xx yy zz xy xz yz)
EFMM_HD void part_recombine(const double x[3], const double* acc, double c1, double u[3], double e6[6]) {
  double g[4][3], H[4][3][3];
  for (int k = 0; k < 4; k++) {
    const double* o = acc + 10 * k;
    for (int a = 0; a < 3; a++) g[k][a] = o[1 + a];
    H[k][0][0] = o[4]; H[k][1][1] = o[5]; H[k][2][2] = o[6];
    H[k][0][1] = H[k][1][0] = o[7];
    H[k][0][2] = H[k][2][0] = o[8];
    H[k][1][2] = H[k][2][1] = o[9];
  }
  for (int i = 0; i < 3; i++) {
    u[i] = (2.0 - c1) * acc[10 * i] + g[3][i];
    for (int j = 0; j < 3; j++) u[i] -= c1 * x[j] * g[j][i];
  }
  double G[3][3];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) {
      double v = (2.0 - c1) * g[a][b] - c1 * g[b][a] + H[3][a][b];
      for (int j = 0; j < 3; j++) v -= c1 * x[j] * H[j][a][b];
      G[a][b] = v;
    }
  e6[0] = G[0][0];
  e6[1] = G[1][1];
  e6[2] = G[2][2];
  e6[3] = 0.5 * (G[0][1] + G[1][0]);
  e6[4] = 0.5 * (G[0][2] + G[2][0]);
  e6[5] = 0.5 * (G[1][2] + G[2][1]);
}

constexpr int NP_THREADS = 256, NP_TILE = 128;

struct PartRec {  // a source's position, charges and dipoles
  double y[3], q[4], d[4][3];
};

// One CTA per near leaf: the evaluation points of the leaf (its sources,
// then its targets) one warp each, the near sources streamed through shared
// memory in tiles (lanes over the tile), per-lane sums of the 40 Laplace
// fields reduced over the warp, then the recombination ADDED to the outputs
// (tree order; strain as 6 symmetric entries).  A source does not act on
// itself.
__global__ void __launch_bounds__(NP_THREADS)
k_near_points(const NearArgs a, const double* __restrict__ nu, double c1, double c2, double inv2mu) {
  __shared__ PartRec tile[NP_TILE];
  const int leaf = a.leaves[blockIdx.x];
  const int sn = a.do_src ? a.box_src_count[leaf] : 0, tn = a.do_tgt ? a.box_tgt_count[leaf] : 0;
  const int s0 = a.box_src_start[leaf], tt0 = a.box_tgt_start[leaf];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = NP_THREADS / 32;
  for (int e0 = 0; e0 < sn + tn; e0 += nw) {
    const int e = e0 + warp;
    const bool act = e < sn + tn;
    const bool is_src = e < sn;
    const int pidx = is_src ? s0 + e : tt0 + (e - sn);
    double x[3] = {0, 0, 0};
    if (act) {
      const double* X = is_src ? a.src_pts + 3 * (size_t)pidx : a.tgt_pts + 3 * (size_t)pidx;
      x[0] = X[0]; x[1] = X[1]; x[2] = X[2];
    }
    double acc[40];
#pragma unroll
    for (int k = 0; k < 40; k++) acc[k] = 0.0;
    for (int b = a.nb_start[blockIdx.x]; b < a.nb_start[blockIdx.x + 1]; b++) {
      const int sb = a.nb_items[b], cnt = a.box_src_count[sb], base = a.box_src_start[sb];
      for (int c0 = 0; c0 < cnt; c0 += NP_TILE) {
        const int m = min(NP_TILE, cnt - c0);
        __syncthreads();
        for (int k = threadIdx.x; k < m; k += NP_THREADS) {
          const int j = base + c0 + k;
          PartRec r;
          double slv[3] = {0, 0, 0}, dlv[3] = {0, 0, 0}, nv[3];
          for (int c = 0; c < 3; c++) {
            r.y[c] = a.src_pts[3 * (size_t)j + c];
            if (a.dosl) slv[c] = a.part_sl[3 * (size_t)j + c];
            if (a.dodl) dlv[c] = a.part_dl[3 * (size_t)j + c];
            nv[c] = nu[3 * (size_t)j + c];
          }
          part_terms(r.y, slv, dlv, nv, c1, c2, inv2mu, r.q, r.d);
          tile[k] = r;
        }
        __syncthreads();
        if (act)
          for (int k = lane; k < m; k += 32) {
            if (is_src && base + c0 + k == pidx) continue;  // self-interaction excluded
            part_pair(x, tile[k].y, tile[k].q, tile[k].d, acc);
          }
      }
    }
#pragma unroll
    for (int k = 0; k < 40; k++) acc[k] = warp_sum(acc[k]);
    if (act && lane == 0) {
      double u[3], e6[6];
      part_recombine(x, acc, c1, u, e6);
      double* U = (is_src ? a.u_src : a.u_tgt) + 3 * (size_t)pidx;
      double* E = (is_src ? a.e_src : a.e_tgt) + 6 * (size_t)pidx;
      for (int c = 0; c < 3; c++) U[c] += u[c];
      if (is_src ? a.dostrain_src : a.dostrain_tgt)
        for (int c = 0; c < 6; c++) E[c] += e6[c];
    }
  }
}

void launch_near_points(cudaStream_t st, const NearArgs& a, const double* nu, double rlam, double rmu) {
  if (a.nleaf <= 0) return;
  const double c1 = (rlam + rmu) / (rlam + 2 * rmu), c2 = rmu / (rlam + 2 * rmu);
  k_near_points<<<a.nleaf, NP_THREADS, 0, st>>>(a, nu, c1, c2, 0.5 / rmu);
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}

// Direct O(N^2) sum (el3dpartdirecttarg, src/elfmm3dpart.f:506): one warp per
// evaluation point (the first ne sources, then the m targets), lanes over
// all n sources; user order; outputs overwritten (strain as 6 entries).
__global__ void __launch_bounds__(256)
k_part_direct(int n, int ne, const double* __restrict__ src, const double* __restrict__ sl,
              const double* __restrict__ dl, const double* __restrict__ nu, int m, const double* __restrict__ tgt,
              double c1, double c2, double inv2mu, double* __restrict__ u_src, double* __restrict__ e_src,
              double* __restrict__ u_tgt, double* __restrict__ e_tgt) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= ne + m) return;
  const bool is_src = warp < ne;
  const int idx = is_src ? warp : warp - ne;
  const double* X = is_src ? src + 3 * (size_t)idx : tgt + 3 * (size_t)idx;
  const double x[3] = {X[0], X[1], X[2]};
  double acc[40];
  for (int k = 0; k < 40; k++) acc[k] = 0.0;
  for (int j = lane; j < n; j += 32) {
    if (is_src && j == idx) continue;
    double y[3], slv[3] = {0, 0, 0}, dlv[3] = {0, 0, 0}, nv[3], q[4], d[4][3];
    for (int c = 0; c < 3; c++) {
      y[c] = src[3 * (size_t)j + c];
      if (sl) slv[c] = sl[3 * (size_t)j + c];
      if (dl) dlv[c] = dl[3 * (size_t)j + c];
      nv[c] = nu ? nu[3 * (size_t)j + c] : 0.0;
    }
    part_terms(y, slv, dlv, nv, c1, c2, inv2mu, q, d);
    part_pair(x, y, q, d, acc);
  }
  for (int k = 0; k < 40; k++) acc[k] = warp_sum(acc[k]);
  if (lane) return;
  double u[3], e6[6];
  part_recombine(x, acc, c1, u, e6);
  double* U = is_src ? u_src : u_tgt;
  double* E = is_src ? e_src : e_tgt;
  if (U)
    for (int c = 0; c < 3; c++) U[3 * (size_t)idx + c] = u[c];
  if (E)
    for (int c = 0; c < 6; c++) E[6 * (size_t)idx + c] = e6[c];
}

void launch_part_direct(cudaStream_t st, int n, int ne, const double* src, const double* sl, const double* dl,
                        const double* nu, int m, const double* tgt, double rlam, double rmu, double* u_src,
                        double* e_src, double* u_tgt, double* e_tgt) {
  if (ne + m <= 0) return;
  const double c1 = (rlam + rmu) / (rlam + 2 * rmu), c2 = rmu / (rlam + 2 * rmu);
  const int blocks = (int)(((long long)(ne + m) * 32 + 255) / 256);
  k_part_direct<<<blocks, 256, 0, st>>>(n, ne, src, sl, dl, nu, m, tgt, c1, c2, 0.5 / rmu, u_src, e_src, u_tgt,
                                        e_tgt);
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}

}  // namespace efmm

// Host evaluation of one (point, particle) pair of the particle near field:
// displacement u[3] and strain e6[6] (xx yy zz xy xz yz) at x of a point
// force sl and a point displacement discontinuity dl with orientation nu at
// y (either may be NULL), through the decomposition the device uses.
extern "C" int efmm_part_pair_host(double rlam, double rmu, const double* x, const double* y, const double* sl,
                                   const double* dl, const double* nu, double* u, double* e6) {
  using namespace efmm;
  if (!x || !y || !u || !e6 || (!sl && !dl) || (dl && !nu) || rmu <= 0) return 16;
  const double c1 = (rlam + rmu) / (rlam + 2 * rmu), c2 = rmu / (rlam + 2 * rmu);
  const double z[3] = {0, 0, 0};
  double q[4], d[4][3], acc[40] = {0};
  part_terms(y, sl ? sl : z, dl ? dl : z, nu ? nu : z, c1, c2, 0.5 / rmu, q, d);
  part_pair(x, y, q, d, acc);
  part_recombine(x, acc, c1, u, e6);
  return 0;
}
