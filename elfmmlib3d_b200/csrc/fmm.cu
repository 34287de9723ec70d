// fmm.cu -- Laplace far field for the four canonical-decomposition passes.
//
// The elastostatic far field is the reference's canonical decomposition
// (src/elfmm3dtria.f:437-615, recombination src/el3routs.f:1392/:1452): three
// Laplace passes with constant densities per Cartesian component j plus one
// with linear densities.  All four passes share one tree and are carried as
// four columns of every expansion, so each translation operator is applied to
// a [D x 4*pairs] panel at once.
//
//   P2M  leaf boxes: 12-node degree-6 quadrature of the (linear) charge and
//        dipole densities on every triangle (src/lfmm3dtrilhess.f:671-748).
//   M2M / M2L / L2L: dense real operator per relative offset (level
//        independent in box units), applied by one grouped gather-GEMM-scatter
//        kernel; M2L order truncated per offset (src/l3dterms.f:144).
//   L2T  leaf boxes: potential, gradient and Hessian of the local expansion
//        with the Lame recombination fused in, writing displacement and strain.
#include "common.cuh"
#include "fmm.h"
#include "kernels.h"
#include "tc_common.cuh"

namespace efmm {

// Origin o of the Lame decomposition for the points of box: the linear
// pass carries the charge (y - o).sigma and the recombination reads
// u_a = (2 - c1) phi_a - c1 (x - o)_j d_a phi_j + d_a Phi_4, which gives the
// same field for every o shared by a source and a target.  In a forest of
// problems (flev >= 0) o is the centre (x, y) of the box's column of level
// flev, so that the FP32 forms see coordinates of the problem's own size
// rather than of its offset in the forest; else o = 0.  o_z is always 0
// (the half-space image formulas read the absolute depth).
__device__ __forceinline__ void lame_origin(const int* ijk, const int* level, int box, const double* c0, double size,
                                            int flev, double o[3]) {
  o[0] = o[1] = o[2] = 0.0;
  const int sh = level[box] - flev;
  if (flev < 0 || sh < 0) return;
  const double w = size / (double)(1 << flev);
  for (int d = 0; d < 2; d++) o[d] = c0[d] - 0.5 * size + (((ijk[3 * box + d] - 1) >> sh) + 0.5) * w;
}

// -------------------------------------------------------------- operators
// Build one real operator matrix per CTA.  kind 0: M2L (offset vector in box
// units), kind 1: M2M (child centre - parent centre, parent units), kind 2:
// L2L (child centre - parent centre, parent units).
__global__ void k_build_ops(int nop, const OpDesc* __restrict__ ops, double* __restrict__ mats) {
  extern __shared__ cplx tab[];
  const OpDesc o = ops[blockIdx.x];
  int p = o.p;
  if (o.kind == 0) {
    if (threadIdx.x == 0) irregular_harmonics(2 * p, o.d[0], o.d[1], o.d[2], tab);
  } else if (o.kind == 3) {  // M2L of the half-space kernel U: T replaced by J
    if (threadIdx.x == 0) u_harmonics(2 * p, o.d[0], o.d[1], o.d[2], tab);
  } else {
    if (threadIdx.x == 0) regular_harmonics(p, o.d[0], o.d[1], o.d[2], tab);
  }
  __syncthreads();
  int nc = ncoef(p), dim = 2 * nc;
  double* M = mats + o.off;
  long long tot = (long long)nc * nc;
  for (long long q = threadIdx.x; q < tot; q += blockDim.x) {
    int r = (int)(q / nc), c = (int)(q % nc);
    double rr, ri, ir, ii;
    op_entry(o.kind == 3 ? 0 : o.kind, tab, r, c, &rr, &ri, &ir, &ii);
    size_t r2 = 2 * (size_t)r, c2 = 2 * (size_t)c;
    M[r2 * dim + c2] = rr;
    M[r2 * dim + c2 + 1] = ri;
    M[(r2 + 1) * dim + c2] = ir;
    M[(r2 + 1) * dim + c2 + 1] = ii;
  }
}

// -------------------------------------------------------------------- P2M
constexpr int P2M_THREADS = 256;
constexpr int P2M_NODES = 8;  // quadrature nodes per batch (one per warp)

__global__ void __launch_bounds__(P2M_THREADS)
k_p2m(const P2MArgs a) {
  extern __shared__ double sm[];
  int box = a.leaves[blockIdx.x];
  int p = a.p, nc = ncoef(p), D = 2 * nc;
  cplx* Ys = reinterpret_cast<cplx*>(sm);                       // [P2M_NODES][nc]
  double* qd = sm + 2 * (size_t)P2M_NODES * nc;                 // [P2M_NODES][16]
  int lev = a.level[box];
  double s = a.size / (double)(1ull << lev);
  double c[3];
  for (int d = 0; d < 3; d++) c[d] = a.c0[d] - a.size / 2 + (a.ijk[3 * box + d] - 1) * s + s / 2;
  int t0 = a.sstart[box], tn = a.scount[box];
  int nnode = a.points ? tn : 12 * tn;
  double org[3];
  lame_origin(a.ijk, a.level, box, a.c0, a.size, a.flev, org);
  const int CMAX = 6;  // coefficients per thread (ncoef(p) <= 1536)
  double acc[CMAX][4][2];
#pragma unroll
  for (int i = 0; i < CMAX; i++)
#pragma unroll
    for (int q = 0; q < 4; q++) acc[i][q][0] = acc[i][q][1] = 0.0;
  Quad12 Q;
  quad12(Q);
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double c1 = a.c1, inv2mu = a.inv2mu, c2 = a.c2;
  for (int b0 = 0; b0 < nnode; b0 += P2M_NODES) {
    __syncthreads();
    int node = b0 + warp;
    if (node < nnode) {
      int it, iq = 0;
      double y[3], w;
      if (a.points) {  // a particle: one node of weight 1
        it = t0 + node;
        for (int d = 0; d < 3; d++) y[d] = a.pts[3 * (size_t)it + d];
        w = 1.0;
      } else {
        it = t0 + node / 12;
        iq = node % 12;
        const double* T = a.tri + 9 * (size_t)it;
        for (int d = 0; d < 3; d++)
          y[d] = Q.b[iq][0] * T[d] + Q.b[iq][1] * T[3 + d] + Q.b[iq][2] * T[6 + d];
        double e1[3] = {T[3] - T[0], T[4] - T[1], T[5] - T[2]};
        double e2[3] = {T[6] - T[0], T[7] - T[1], T[8] - T[2]};
        double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                        e1[0] * e2[1] - e1[1] * e2[0]};
        double area = 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        w = Q.w[iq] * area;
      }
      double z[3] = {(y[0] - c[0]) / s, (y[1] - c[1]) / s, (y[2] - c[2]) / s};
      // column chains of the regular harmonics, one order m per lane
      cplx* Y = Ys + (size_t)warp * nc;
      for (int m = lane; m <= p; m += 32) {
        cplx dm = {1.0, 0.0}, wv = {-0.5 * z[0], -0.5 * z[1]};
        for (int k = 1; k <= m; k++) dm = cscale(1.0 / k, cmul(dm, wv));
        double r2 = z[0] * z[0] + z[1] * z[1] + z[2] * z[2];
        Y[cidx(m, m)] = dm;
        cplx ym2 = {0, 0}, ym1 = dm;
        for (int n = m + 1; n <= p; n++) {
          double aa = (2.0 * n - 1.0) * z[2];
          double inv = 1.0 / ((double)(n - m) * (double)(n + m));
          cplx yn = {(aa * ym1.re - r2 * ym2.re) * inv, (aa * ym1.im - r2 * ym2.im) * inv};
          Y[cidx(n, m)] = yn;
          ym2 = ym1;
          ym1 = yn;
        }
      }
      if (lane == 0) {
        const long long off = blockIdx.y * a.rstride + it * a.tstride, ds = a.dstride;
        const double* nn = a.nrm + 3 * (size_t)it;
        double* o = qd + 16 * warp;
        double sl[3] = {0, 0, 0}, dl[3] = {0, 0, 0};
        if (a.dosl) { sl[0] = a.ssl[off]; sl[1] = a.ssl[off + ds]; sl[2] = a.ssl[off + 2 * ds]; }
        if (a.dodl) { dl[0] = a.sdl[off]; dl[1] = a.sdl[off + ds]; dl[2] = a.sdl[off + 2 * ds]; }
        // passes 0..2: charge s_j/(2mu), dipole (n s_j + s n_j)/2
        for (int j = 0; j < 3; j++) {
          o[j] = w * sl[j] * inv2mu;
          for (int d = 0; d < 3; d++) o[4 + 3 * j + d] = w * 0.5 * (nn[d] * dl[j] + dl[d] * nn[j]);
        }
        // pass 3: charge (s_sl.y) c1/(2mu) + (s_dl.n) c2, dipole c1 [n (s_dl.y) + s_dl (n.y)]/2
        // (y relative to the origin of lame_origin)
        const double yo[3] = {y[0] - org[0], y[1] - org[1], y[2] - org[2]};
        double sly = sl[0] * yo[0] + sl[1] * yo[1] + sl[2] * yo[2];
        double dly = dl[0] * yo[0] + dl[1] * yo[1] + dl[2] * yo[2];
        double dln = dl[0] * nn[0] + dl[1] * nn[1] + dl[2] * nn[2];
        double ny = nn[0] * yo[0] + nn[1] * yo[1] + nn[2] * yo[2];
        o[3] = w * (sly * c1 * inv2mu + dln * c2);
        for (int d = 0; d < 3; d++) o[13 + d] = w * 0.5 * c1 * (nn[d] * dly + dl[d] * ny);
      }
    }
    __syncthreads();
    int nb = min(P2M_NODES, nnode - b0);
    double is = 1.0 / s;
#pragma unroll
    for (int i = 0; i < CMAX; i++) {
      int cc = threadIdx.x + i * P2M_THREADS;
      if (cc >= nc) break;
      int n = 0;
      while ((n + 1) * (n + 2) / 2 <= cc) n++;
      int m = cc - n * (n + 1) / 2;
      for (int k = 0; k < nb; k++) {
        const cplx* Y = Ys + (size_t)k * nc;
        const double* o = qd + 16 * k;
        cplx y = Y[cc];
        cplx ya = {0, 0}, yb = {0, 0}, yc = {0, 0};
        if (n > 0) {
          ya = hget(Y, n - 1, m);
          yb = hget(Y, n - 1, m + 1);
          yc = hget(Y, n - 1, m - 1);
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const double* dv = (q < 3) ? o + 4 + 3 * q : o + 13;
          // conj(d.grad Y) = conj(dz ya + (dx - i dy)/2 yb - (dx + i dy)/2 yc)
          double gre = dv[2] * ya.re + 0.5 * (dv[0] * yb.re + dv[1] * yb.im) -
                       0.5 * (dv[0] * yc.re - dv[1] * yc.im);
          double gim = dv[2] * ya.im + 0.5 * (dv[0] * yb.im - dv[1] * yb.re) -
                       0.5 * (dv[0] * yc.im + dv[1] * yc.re);
          double qq = o[q];
          acc[i][q][0] += qq * y.re + is * gre;
          acc[i][q][1] -= qq * y.im + is * gim;
        }
      }
    }
  }
  double* M = a.mpole + ((size_t)box * a.C + 4 * blockIdx.y) * D;
#pragma unroll
  for (int i = 0; i < CMAX; i++) {
    int cc = threadIdx.x + i * P2M_THREADS;
    if (cc >= nc) break;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      M[(size_t)q * D + 2 * cc] = acc[i][q][0];
      M[(size_t)q * D + 2 * cc + 1] = acc[i][q][1];
    }
  }
}

// ---------------------------------------------- P2M, many right-hand sides
// For C = 4R columns the multipole of a leaf is a product
//   M[row][col] = sum over (node, k) F[row][node, k] * W[node, k][col]
// with F the conjugated regular harmonics and their gradients at the 12 P2M
// nodes of each triangle (k = 0 charge, 1..3 dipole x, y, z) and W the per
// node charge and dipole strengths of column col = (rhs r, pass q).  One CTA
// per (leaf, 128-row tile, 128-column tile); node chunks of PG_NODES nodes
// build Y in shared memory, then the F and W tiles, then an 8 x 8-per-thread
// register-blocked product.  Rows are the interleaved (re, im) coefficients.
constexpr int PG_NODES = 8, PG_K = 4 * PG_NODES, PG_R = 128, PG_C = 128;

template <class T>
__global__ void __launch_bounds__(256, 1)
k_p2m_gemm(const P2MArgs a, int R, T* __restrict__ mpole) {
  using V2 = typename Vec2<T>::type;
  extern __shared__ __align__(16) unsigned char pg_smem[];
  const int p = a.p, nc = ncoef(p), D = 2 * nc, C = 4 * R;
  cplx* Ys = reinterpret_cast<cplx*>(pg_smem);                  // [PG_NODES][nc]
  double* nd = reinterpret_cast<double*>(Ys + PG_NODES * nc);   // [PG_NODES][8]: y, n, w
  int* nt = reinterpret_cast<int*>(nd + PG_NODES * 8);          // [PG_NODES] triangle
  T* Fs = reinterpret_cast<T*>(nt + PG_NODES + (PG_NODES & 1)); // [PG_K][PG_R]
  T* Ws = Fs + PG_K * PG_R;                                      // [PG_K][PG_C]
  const int box = a.leaves[blockIdx.x];
  const int row0 = blockIdx.y * PG_R, col0 = blockIdx.z * PG_C;
  const int lev = a.level[box];
  const double s = a.size / (double)(1ull << lev), is = 1.0 / s;
  double c[3];
  for (int d = 0; d < 3; d++) c[d] = a.c0[d] - a.size / 2 + (a.ijk[3 * box + d] - 1) * s + s / 2;
  const int t0 = a.sstart[box], tn = a.scount[box];
  const int nnode = 12 * tn;
  double org[3];
  lame_origin(a.ijk, a.level, box, a.c0, a.size, a.flev, org);
  Quad12 Q;
  quad12(Q);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // F-tile role: one row, nodes j = (tid >> 7) + 2 i
  const int frow = tid & 127, fj0 = tid >> 7;
  const int grow = row0 + frow;
  const bool frow_ok = grow < D;
  const int cc = frow_ok ? grow >> 1 : 0, part = grow & 1;
  int fn = 0;
  while ((fn + 1) * (fn + 2) / 2 <= cc) fn++;
  const int fm = cc - fn * (fn + 1) / 2;
  const double c1 = a.c1, c2 = a.c2, inv2mu = a.inv2mu;
  const int tx = tid & 15, ty = tid >> 4;
  T acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) acc[i][j] = T(0);
  for (int b0 = 0; b0 < nnode; b0 += PG_NODES) {
    __syncthreads();
    // Y of node b0 + warp (regular harmonics, one order m per lane)
    if (warp < PG_NODES) {
      const int node = b0 + warp;
      cplx* Y = Ys + (size_t)warp * nc;
      if (node < nnode) {
        const int it = t0 + node / 12, iq = node % 12;
        const double* Tr = a.tri + 9 * (size_t)it;
        double y[3];
        for (int d = 0; d < 3; d++)
          y[d] = Q.b[iq][0] * Tr[d] + Q.b[iq][1] * Tr[3 + d] + Q.b[iq][2] * Tr[6 + d];
        const double z[3] = {(y[0] - c[0]) * is, (y[1] - c[1]) * is, (y[2] - c[2]) * is};
        const double r2 = z[0] * z[0] + z[1] * z[1] + z[2] * z[2];
        for (int m = lane; m <= p; m += 32) {
          cplx dm = {1.0, 0.0}, wv = {-0.5 * z[0], -0.5 * z[1]};
          for (int k = 1; k <= m; k++) dm = cscale(1.0 / k, cmul(dm, wv));
          Y[cidx(m, m)] = dm;
          cplx ym2 = {0, 0}, ym1 = dm;
          for (int n = m + 1; n <= p; n++) {
            const double aa = (2.0 * n - 1.0) * z[2];
            const double inv = 1.0 / ((double)(n - m) * (double)(n + m));
            cplx yn = {(aa * ym1.re - r2 * ym2.re) * inv, (aa * ym1.im - r2 * ym2.im) * inv};
            Y[cidx(n, m)] = yn;
            ym2 = ym1;
            ym1 = yn;
          }
        }
        if (lane == 0) {
          const double e1[3] = {Tr[3] - Tr[0], Tr[4] - Tr[1], Tr[5] - Tr[2]};
          const double e2[3] = {Tr[6] - Tr[0], Tr[7] - Tr[1], Tr[8] - Tr[2]};
          const double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                                e1[0] * e2[1] - e1[1] * e2[0]};
          const double area = 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
          double* o = nd + 8 * warp;  // position relative to the origin of lame_origin
          o[0] = y[0] - org[0]; o[1] = y[1] - org[1]; o[2] = y[2] - org[2];
          const double* nn = a.nrm + 3 * (size_t)it;
          o[3] = nn[0]; o[4] = nn[1]; o[5] = nn[2];
          o[6] = Q.w[iq] * area;
          nt[warp] = it;
        }
      } else if (lane == 0) {
        nd[8 * warp + 6] = 0.0;
        nt[warp] = -1;
      }
    }
    __syncthreads();
    // F tile: rows x (node, k)
    for (int j = fj0; j < PG_NODES; j += 2) {
      T f[4] = {T(0), T(0), T(0), T(0)};
      if (frow_ok && nt[j] >= 0) {
        const double sc = a.wnorm ? a.wnorm[grow] : 1.0;
        const cplx* Y = Ys + (size_t)j * nc;
        const cplx y = Y[cc];
        cplx ya = {0, 0}, yb = {0, 0}, yc = {0, 0};
        if (fn > 0) {
          ya = hget(Y, fn - 1, fm);
          yb = hget(Y, fn - 1, fm + 1);
          yc = hget(Y, fn - 1, fm - 1);
        }
        if (part == 0) {
          f[0] = (T)(sc * y.re);
          f[1] = (T)(sc * 0.5 * is * (yb.re - yc.re));
          f[2] = (T)(sc * 0.5 * is * (yb.im + yc.im));
          f[3] = (T)(sc * is * ya.re);
        } else {
          f[0] = (T)(-sc * y.im);
          f[1] = (T)(-sc * 0.5 * is * (yb.im - yc.im));
          f[2] = (T)(sc * 0.5 * is * (yb.re + yc.re));
          f[3] = (T)(-sc * is * ya.im);
        }
      }
#pragma unroll
      for (int k = 0; k < 4; k++) Fs[(4 * j + k) * PG_R + frow] = f[k];
    }
    // W tile: (node, k) x columns; column = (rhs r, pass q)
    for (int q2 = tid; q2 < PG_NODES * PG_C; q2 += 256) {
      const int j = q2 / PG_C, col = q2 % PG_C, gcol = col0 + col;
      T wv[4] = {T(0), T(0), T(0), T(0)};
      const int it = nt[j];
      if (it >= 0 && gcol < C) {
        const int r = gcol >> 2, q = gcol & 3;
        const double* o = nd + 8 * j;
        const double y[3] = {o[0], o[1], o[2]}, nn[3] = {o[3], o[4], o[5]}, w = o[6];
        const long long off = r * a.rstride + it * a.tstride, ds = a.dstride;
        double sl[3] = {0, 0, 0}, dl[3] = {0, 0, 0};
        if (a.dosl) { sl[0] = a.ssl[off]; sl[1] = a.ssl[off + ds]; sl[2] = a.ssl[off + 2 * ds]; }
        if (a.dodl) { dl[0] = a.sdl[off]; dl[1] = a.sdl[off + ds]; dl[2] = a.sdl[off + 2 * ds]; }
        if (q < 3) {
          // pass q: charge s_q/(2mu), dipole (n s_q + s n_q)/2
          wv[0] = (T)(w * sl[q] * inv2mu);
          for (int d = 0; d < 3; d++) wv[1 + d] = (T)(w * 0.5 * (nn[d] * dl[q] + dl[d] * nn[q]));
        } else {
          // pass 3: charge (s_sl.y) c1/(2mu) + (s_dl.n) c2, dipole c1 [n (s_dl.y) + s_dl (n.y)]/2
          const double sly = sl[0] * y[0] + sl[1] * y[1] + sl[2] * y[2];
          const double dly = dl[0] * y[0] + dl[1] * y[1] + dl[2] * y[2];
          const double dln = dl[0] * nn[0] + dl[1] * nn[1] + dl[2] * nn[2];
          const double ny = nn[0] * y[0] + nn[1] * y[1] + nn[2] * y[2];
          wv[0] = (T)(w * (sly * c1 * inv2mu + dln * c2));
          for (int d = 0; d < 3; d++) wv[1 + d] = (T)(w * 0.5 * c1 * (nn[d] * dly + dl[d] * ny));
        }
      }
#pragma unroll
      for (int k = 0; k < 4; k++) Ws[(4 * j + k) * PG_C + col] = wv[k];
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < PG_K; kk++) {
      T av[8], bv[8];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        V2 v = *reinterpret_cast<const V2*>(Fs + kk * PG_R + ty * 8 + 2 * i);
        av[2 * i] = v.x;
        av[2 * i + 1] = v.y;
      }
#pragma unroll
      for (int j = 0; j < 4; j++) {
        V2 v = *reinterpret_cast<const V2*>(Ws + kk * PG_C + 32 * j + 2 * tx);
        bv[2 * j] = v.x;
        bv[2 * j + 1] = v.y;
      }
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] += av[i] * bv[j];
    }
  }
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const int gcol = col0 + 32 * (j >> 1) + 2 * tx + (j & 1);
    if (gcol >= C) continue;
    T* M = mpole + ((size_t)box * C + gcol) * D;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int r = row0 + ty * 8 + i;
      if (r < D) M[r] = acc[i][j];
    }
  }
}

// ------------------------------------------- P2M in two stages (product form)
// Stage 1 writes, per leaf, the node features A[k][row] (k = 4 node + comp,
// comp 0 charge, 1..3 dipole x, y, z; rows the interleaved coefficients) and
// the node weights B[col][k] of every column; stage 2 is the plain batched
// product  mpole[box][col][row] = sum_k A[k][row] B[col][k]  (k_gemm_tn).
// The features depend on the geometry only; each is computed once per node
// instead of once per output tile.
// NF = 4: charge and dipole rows per node; NF = 9 adds the five second
// derivatives (xx, yy, xy, xz, yz; zz = -xx - yy) that carry quadrupole
// sources (the half-space image columns).
template <class T, int NF>
__global__ void __launch_bounds__(256)
k_p2m_features(const P2MArgs a, const int* __restrict__ wleaves, const long long* __restrict__ foff,
               const long long* __restrict__ noff, double* __restrict__ nrec, T* __restrict__ F) {
  extern __shared__ __align__(16) unsigned char pf_smem[];
  const int p = a.p, nc = ncoef(p), D = 2 * nc;
  const int box = a.leaves[wleaves[blockIdx.x]];
  const int t0 = a.sstart[box], tn = a.scount[box];
  const int nnode = 12 * tn;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int node = blockIdx.y * 8 + warp;
  if (node >= nnode) return;
  cplx* Y = reinterpret_cast<cplx*>(pf_smem) + (size_t)warp * nc;
  const int lev = a.level[box];
  const double s = a.size / (double)(1ull << lev), is = 1.0 / s;
  double c[3];
  for (int d = 0; d < 3; d++) c[d] = a.c0[d] - a.size / 2 + (a.ijk[3 * box + d] - 1) * s + s / 2;
  Quad12 Q;
  quad12(Q);
  const int it = t0 + node / 12, iq = node % 12;
  const double* Tr = a.tri + 9 * (size_t)it;
  double y[3];
  for (int d = 0; d < 3; d++) y[d] = Q.b[iq][0] * Tr[d] + Q.b[iq][1] * Tr[3 + d] + Q.b[iq][2] * Tr[6 + d];
  const double z[3] = {(y[0] - c[0]) * is, (y[1] - c[1]) * is, (y[2] - c[2]) * is};
  const double r2 = z[0] * z[0] + z[1] * z[1] + z[2] * z[2];
  if (lane == 0) {
    // node record for the weights: position (relative to the origin of
    // lame_origin), normal, weight x area, triangle
    const double e1[3] = {Tr[3] - Tr[0], Tr[4] - Tr[1], Tr[5] - Tr[2]};
    const double e2[3] = {Tr[6] - Tr[0], Tr[7] - Tr[1], Tr[8] - Tr[2]};
    const double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                          e1[0] * e2[1] - e1[1] * e2[0]};
    double* o = nrec + 8 * (noff[blockIdx.x] + node);
    const double* nn = a.nrm + 3 * (size_t)it;
    double org[3];
    lame_origin(a.ijk, a.level, box, a.c0, a.size, a.flev, org);
    o[0] = y[0] - org[0]; o[1] = y[1] - org[1]; o[2] = y[2] - org[2];
    o[3] = nn[0]; o[4] = nn[1]; o[5] = nn[2];
    o[6] = Q.w[iq] * 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    o[7] = (double)it;
  }
  for (int m = lane; m <= p; m += 32) {
    cplx dm = {1.0, 0.0}, wv = {-0.5 * z[0], -0.5 * z[1]};
    for (int k = 1; k <= m; k++) dm = cscale(1.0 / k, cmul(dm, wv));
    Y[cidx(m, m)] = dm;
    cplx ym2 = {0, 0}, ym1 = dm;
    for (int n = m + 1; n <= p; n++) {
      const double aa = (2.0 * n - 1.0) * z[2];
      const double inv = 1.0 / ((double)(n - m) * (double)(n + m));
      cplx yn = {(aa * ym1.re - r2 * ym2.re) * inv, (aa * ym1.im - r2 * ym2.im) * inv};
      Y[cidx(n, m)] = yn;
      ym2 = ym1;
      ym1 = yn;
    }
  }
  __syncwarp();
  // rows: charge/dipole rows of every node first (4 node + f), then (NF = 9)
  // the five second-derivative rows (4 nnode + 5 node + f - 4), so that
  // columns without quadrupole sources multiply the first block only
  T* out = F + foff[blockIdx.x] + (size_t)(4 * node) * D;
  T* outq = F + foff[blockIdx.x] + (size_t)(4 * nnode + 5 * node) * D;
  for (int cc = lane; cc < nc; cc += 32) {
    int fn = 0;
    while ((fn + 1) * (fn + 2) / 2 <= cc) fn++;
    const int fm = cc - fn * (fn + 1) / 2;
    const cplx yv = Y[cc];
    cplx ya = {0, 0}, yb = {0, 0}, yc = {0, 0};
    if (fn > 0) {
      ya = hget(Y, fn - 1, fm);
      yb = hget(Y, fn - 1, fm + 1);
      yc = hget(Y, fn - 1, fm - 1);
    }
    const double sr = a.wnorm ? a.wnorm[2 * cc] : 1.0;
    // real row 2cc, imaginary row 2cc + 1 (as in k_p2m_gemm)
    out[2 * cc] = (T)(sr * yv.re);
    out[2 * cc + 1] = (T)(-sr * yv.im);
    out[D + 2 * cc] = (T)(sr * 0.5 * is * (yb.re - yc.re));
    out[D + 2 * cc + 1] = (T)(-sr * 0.5 * is * (yb.im - yc.im));
    out[2 * D + 2 * cc] = (T)(sr * 0.5 * is * (yb.im + yc.im));
    out[2 * D + 2 * cc + 1] = (T)(sr * 0.5 * is * (yb.re + yc.re));
    out[3 * D + 2 * cc] = (T)(sr * is * ya.re);
    out[3 * D + 2 * cc + 1] = (T)(-sr * is * ya.im);
    if (NF == 9) {
      // second derivatives from the ladder relations (conjugated rows):
      //   xx = (Y^{m+2} - 2 Y^m + Y^{m-2}) / 4,  yy = -(Y^{m+2} + 2 Y^m + Y^{m-2}) / 4,
      //   xy = (Y^{m+2} - Y^{m-2}) / 4i,  xz = (Y^{m+1} - Y^{m-1}) / 2,  yz = (Y^{m+1} + Y^{m-1}) / 2i
      // (all of degree n - 2)
      cplx y0 = {0, 0}, yp1 = {0, 0}, ym1 = {0, 0}, yp2 = {0, 0}, ym2 = {0, 0};
      if (fn > 1) {
        y0 = hget(Y, fn - 2, fm);
        yp1 = hget(Y, fn - 2, fm + 1);
        ym1 = hget(Y, fn - 2, fm - 1);
        yp2 = hget(Y, fn - 2, fm + 2);
        ym2 = hget(Y, fn - 2, fm - 2);
      }
      const double q = sr * is * is;
      outq[2 * cc] = (T)(q * 0.25 * (yp2.re - 2.0 * y0.re + ym2.re));
      outq[2 * cc + 1] = (T)(-q * 0.25 * (yp2.im - 2.0 * y0.im + ym2.im));
      outq[D + 2 * cc] = (T)(-q * 0.25 * (yp2.re + 2.0 * y0.re + ym2.re));
      outq[D + 2 * cc + 1] = (T)(q * 0.25 * (yp2.im + 2.0 * y0.im + ym2.im));
      outq[2 * D + 2 * cc] = (T)(q * 0.25 * (yp2.im - ym2.im));
      outq[2 * D + 2 * cc + 1] = (T)(q * 0.25 * (yp2.re - ym2.re));
      outq[3 * D + 2 * cc] = (T)(q * 0.5 * (yp1.re - ym1.re));
      outq[3 * D + 2 * cc + 1] = (T)(-q * 0.5 * (yp1.im - ym1.im));
      outq[4 * D + 2 * cc] = (T)(q * 0.5 * (yp1.im + ym1.im));
      outq[4 * D + 2 * cc + 1] = (T)(q * 0.5 * (yp1.re + ym1.re));
    }
  }
}

// Node weights of the half-space image columns, 7R per box, column
// kind * R + r for right-hand side r: kinds 0..3 the anti-image passes (the
// free-space passes with the anti-image constants c1, c2 of P2MArgs), 4 and 5
// the two 1/r potentials Phi_a, Phi_c of the C piece, 6 the U potential W of
// the B piece.  Per node 9 weights: charge, dipole (3) and the five
// second-derivative weights (xx - zz, yy - zz, 2xy, 2xz, 2yz of the
// quadrupole tensor).  With f the single-layer density, T the double-layer
// tensor lam (b.n) I + mu (b n^T + n b^T), h = -y_3 the source depth and
// alpha = (lam + mu)/(lam + 2 mu) (sources in the gradient-of-source
// convention of the features):
//   Phi_a: q = -(2 - alpha) f_3, D = -h alpha f - (2 - 2 alpha) T e_3, Q = -h alpha T
//   Phi_c: D = -f, Q = -T
//   W:     D = (f_1, f_2, -f_3), Q = -(S T + T S)/2, S = diag(-1, -1, 1)
// (the B and C pieces of src/mindlinpieces.f:29-520 written as Laplace-type
// potentials; their double layers by differentiation at the source).
__device__ void img_node_weights(int kind, const double sl[3], const double dl[3], const double nn[3],
                                 const double y[3], const P2MArgs& a, double wv[9]) {
  const double c1 = a.c1, c2 = a.c2, inv2mu = a.inv2mu, al = a.alpha, lam = a.lam, mu = a.mu;
  for (int k = 0; k < 9; k++) wv[k] = 0.0;
  double Qm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  const double dln = dl[0] * nn[0] + dl[1] * nn[1] + dl[2] * nn[2];
  double Tm[3][3];
  for (int k = 0; k < 3; k++)
    for (int l = 0; l < 3; l++) Tm[k][l] = (k == l ? lam * dln : 0.0) + mu * (dl[k] * nn[l] + dl[l] * nn[k]);
  const double h = -y[2];
  if (kind < 3) {
    wv[0] = sl[kind] * inv2mu;
    for (int d = 0; d < 3; d++) wv[1 + d] = 0.5 * (nn[d] * dl[kind] + dl[d] * nn[kind]);
  } else if (kind == 3) {
    const double sly = sl[0] * y[0] + sl[1] * y[1] + sl[2] * y[2];
    const double dly = dl[0] * y[0] + dl[1] * y[1] + dl[2] * y[2];
    const double ny = nn[0] * y[0] + nn[1] * y[1] + nn[2] * y[2];
    wv[0] = sly * c1 * inv2mu + dln * c2;
    for (int d = 0; d < 3; d++) wv[1 + d] = 0.5 * c1 * (nn[d] * dly + dl[d] * ny);
  } else if (kind == 4) {
    wv[0] = -(2.0 - al) * sl[2];
    for (int d = 0; d < 3; d++) wv[1 + d] = -h * al * sl[d] - (2.0 - 2.0 * al) * Tm[2][d];
    for (int k = 0; k < 3; k++)
      for (int l = 0; l < 3; l++) Qm[k][l] = -h * al * Tm[k][l];
  } else if (kind == 5) {
    for (int d = 0; d < 3; d++) wv[1 + d] = -sl[d];
    for (int k = 0; k < 3; k++)
      for (int l = 0; l < 3; l++) Qm[k][l] = -Tm[k][l];
  } else {
    wv[1] = sl[0];
    wv[2] = sl[1];
    wv[3] = -sl[2];
    Qm[0][0] = Tm[0][0]; Qm[1][1] = Tm[1][1]; Qm[2][2] = -Tm[2][2];
    Qm[0][1] = Qm[1][0] = Tm[0][1];
  }
  wv[4] = Qm[0][0] - Qm[2][2];
  wv[5] = Qm[1][1] - Qm[2][2];
  wv[6] = 2.0 * Qm[0][1];
  wv[7] = 2.0 * Qm[0][2];
  wv[8] = 2.0 * Qm[1][2];
}

// Weights matrix per leaf: column col of ldb K = 9 nnode, rows in the
// feature order (4 node + f, then 4 nnode + 5 node + f - 4).
template <class T>
__global__ void __launch_bounds__(256)
k_p2m_weights_img(const P2MArgs a, int R, const int* __restrict__ wleaves, const long long* __restrict__ woff,
                  const long long* __restrict__ noff, const double* __restrict__ nrec, T* __restrict__ W) {
  const int box = a.leaves[wleaves[blockIdx.x]];
  const int tn = a.scount[box];
  const int nnode = 12 * tn, K = 9 * nnode, C = 7 * R;
  const double* nd = nrec + 8 * noff[blockIdx.x];
  T* out = W + woff[blockIdx.x];
  for (long long q = blockIdx.y * (long long)blockDim.x + threadIdx.x; q < (long long)nnode * C;
       q += (long long)gridDim.y * blockDim.x) {
    const int col = (int)(q / nnode), node = (int)(q % nnode);
    const int kind = col / R, r = col % R;
    const double* o = nd + 8 * node;
    const double y[3] = {o[0], o[1], o[2]}, nn[3] = {o[3], o[4], o[5]}, w = o[6];
    const long long it = (long long)o[7];
    const long long off = r * a.rstride + it * a.tstride, ds = a.dstride;
    double sl[3] = {0, 0, 0}, dl[3] = {0, 0, 0};
    if (a.dosl) { sl[0] = a.ssl[off]; sl[1] = a.ssl[off + ds]; sl[2] = a.ssl[off + 2 * ds]; }
    if (a.dodl) { dl[0] = a.sdl[off]; dl[1] = a.sdl[off + ds]; dl[2] = a.sdl[off + 2 * ds]; }
    double wv[9];
    img_node_weights(kind, sl, dl, nn, y, a, wv);
    T* ow = out + (size_t)col * K;
#pragma unroll
    for (int k = 0; k < 4; k++) ow[4 * node + k] = (T)(w * wv[k]);
    if (kind >= 4) {
#pragma unroll
      for (int k = 0; k < 5; k++) ow[4 * nnode + 5 * node + k] = (T)(w * wv[4 + k]);
    }
  }
}

// ------------------------------- P2M factored through unit-density multipoles
// The node weights of every column are linear in the six density components
// of the node's triangle (sl_0..2, dl_0..2), with coefficients that depend on
// the geometry only.  The P2M of a leaf therefore factors as
//   mpole[box][kind, r] = sum_{t in box} sum_s H[kind][t][s] sigma_s(t, r),
// where H[kind][t][s] (D coefficients) is the multipole of triangle t with
// unit density component s in column kind.  Stage 1 (k_p2m_unit) builds H
// once per triangle, independent of the right-hand sides; stage 2 is the
// batched product of H (K = 6 x triangles per leaf) with the densities
// (k_p2m_sigma gathers them, N = R).  Per triangle, H follows from 26 node
// moments of the features F (rows as in k_p2m_features):
//   M0[row] = sum_nodes w F[row],  M1_e[row] = sum_nodes w y_e F[row]
// (w: quadrature weight x area, y: node position), by the combinations of
// the weights in k_p2m_weights / img_node_weights:
//   kinds p = 0..2: H[sl_p] = inv2mu M0[0],
//                   H[dl_e] = (delta_ep n.M0[1..3] + n_p M0[1 + e]) / 2
//   kind 3:         H[sl_e] = c1 inv2mu M1_e[0],
//                   H[dl_e] = c2 n_e M0[0] + c1 (sum_d n_d M1_e[1 + d] + sum_j n_j M1_j[1 + e]) / 2
//   kind 4:         H[sl_e] = alpha M1_3[1 + e] - delta_e3 (2 - alpha) M0[0],
//                   H[dl_e] = -(2 - 2 alpha) Te_3.M0[1..3] + alpha qv(Te).M1_3[4..8]
//   kind 5:         H[sl_e] = -M0[1 + e],  H[dl_e] = -qv(Te).M0[4..8]
//   kind 6:         H[sl] = (M0[1], M0[2], -M0[3]),  H[dl_e] = qvU(Te).M0[4..8]
// with Te[k][l] = lam delta_kl n_e + mu (delta_ke n_l + delta_le n_k) the
// double-layer tensor of a unit jump e, qv(T) = (T00 - T22, T11 - T22, 2 T01,
// 2 T02, 2 T12) and qvU(T) = (T00 + T22, T11 + T22, 2 T01, 0, 0).  NK = 4:
// the four free-space (or anti-image) columns; NK = 7 adds the image columns.
constexpr int UNIT_TB = 16;  // triangles per CTA

// Largest CTA of k_p2m_unit (the FP64 form; register budget of the moments
// about 240 per thread; CTAs of whole warp quadruples, so that every
// sub-partition's register file holds its share); the launch uses the fewest
// such threads that cover the coefficients in the same number of rounds.
// The FP32 form runs k_p2m_unit_f.
template <class T>
__host__ __device__ constexpr int unit_threads() { return sizeof(T) == 4 ? 512 : 256; }

// Shared-memory layout of the node harmonics in k_p2m_unit: row n = -2..p
// holds m = -2..n+4 (zero outside 0 <= |m| <= n; Y_n^{-m} = (-1)^m conj Y_n^m
// for m = 1, 2), so every ladder neighbour of (n, m) is a plain load.
__host__ __device__ constexpr int unit_yoff(int n, int m) { return (n + 6) * (n + 7) / 2 + m - 8; }
__host__ __device__ constexpr int unit_ylen(int p) { return unit_yoff(p + 1, -2); }

// Unit-density columns H[kind][s] of one coefficient from its (scaled)
// moments: put(kind, s, re, im) for s = 0..2 (single layer), 3..5 (double
// layer); nv the triangle normal.  Kinds reading the first moments come
// first so that their registers free up early.
template <class T, int NK, class Put>
__device__ __forceinline__ void unit_combine(Put& put, const T* m0r, const T* m0i, const T (*m1r)[4],
                                             const T (*m1i)[4], const T* mqr, const T* mqi, const T* nv3, T tc1,
                                             T tc2, T ti2, T tal, T tlam, T tmu) {
  for (int e = 0; e < 3; e++) put(3, e, tc1 * ti2 * m1r[e][0], tc1 * ti2 * m1i[e][0]);
  for (int e = 0; e < 3; e++) {
    T vr = tc2 * nv3[e] * m0r[0], vi = tc2 * nv3[e] * m0i[0];
    for (int d = 0; d < 3; d++) {
      vr += (T)0.5 * tc1 * (nv3[d] * m1r[e][1 + d] + nv3[d] * m1r[d][1 + e]);
      vi += (T)0.5 * tc1 * (nv3[d] * m1i[e][1 + d] + nv3[d] * m1i[d][1 + e]);
    }
    put(3, 3 + e, vr, vi);
  }
  // Te: the double-layer tensor of a unit jump in direction e,
  // qv(Te) = (T00 - T22, T11 - T22, 2 T01, 2 T02, 2 T12), qvU(Te) = (T00 + T22, T11 + T22, 2 T01)
  auto tens = [&](int e, int k, int l) {
    return (k == l ? tlam * nv3[e] : (T)0) + tmu * ((k == e ? nv3[l] : (T)0) + (l == e ? nv3[k] : (T)0));
  };
  if constexpr (NK == 7) {
    for (int e = 0; e < 3; e++) {
      put(4, e, tal * m1r[2][1 + e] - (e == 2 ? ((T)2 - tal) * m0r[0] : (T)0),
          tal * m1i[2][1 + e] - (e == 2 ? ((T)2 - tal) * m0i[0] : (T)0));
      const T qv[5] = {tens(e, 0, 0) - tens(e, 2, 2), tens(e, 1, 1) - tens(e, 2, 2), 2 * tens(e, 0, 1),
                       2 * tens(e, 0, 2), 2 * tens(e, 1, 2)};
      T r4 = 0, i4 = 0;
      for (int d = 0; d < 3; d++) {
        r4 -= ((T)2 - 2 * tal) * tens(e, 2, d) * m0r[1 + d];
        i4 -= ((T)2 - 2 * tal) * tens(e, 2, d) * m0i[1 + d];
      }
      for (int f = 0; f < 5; f++) {
        r4 += tal * qv[f] * mqr[f];
        i4 += tal * qv[f] * mqi[f];
      }
      put(4, 3 + e, r4, i4);
    }
  }
  const T ndr = nv3[0] * m0r[1] + nv3[1] * m0r[2] + nv3[2] * m0r[3];
  const T ndi = nv3[0] * m0i[1] + nv3[1] * m0i[2] + nv3[2] * m0i[3];
#pragma unroll
  for (int pk = 0; pk < 3; pk++) {
    for (int e = 0; e < 3; e++) put(pk, e, e == pk ? ti2 * m0r[0] : (T)0, e == pk ? ti2 * m0i[0] : (T)0);
    for (int e = 0; e < 3; e++)
      put(pk, 3 + e, (T)0.5 * ((e == pk ? ndr : (T)0) + nv3[pk] * m0r[1 + e]),
          (T)0.5 * ((e == pk ? ndi : (T)0) + nv3[pk] * m0i[1 + e]));
  }
  if constexpr (NK == 7) {
    for (int e = 0; e < 3; e++) {
      const T qv[5] = {tens(e, 0, 0) - tens(e, 2, 2), tens(e, 1, 1) - tens(e, 2, 2), 2 * tens(e, 0, 1),
                       2 * tens(e, 0, 2), 2 * tens(e, 1, 2)};
      const T qu[3] = {tens(e, 0, 0) + tens(e, 2, 2), tens(e, 1, 1) + tens(e, 2, 2), 2 * tens(e, 0, 1)};
      T r5 = 0, i5 = 0, r6 = 0, i6 = 0;
      for (int f = 0; f < 5; f++) {
        r5 -= qv[f] * m0r[4 + f];
        i5 -= qv[f] * m0i[4 + f];
      }
      for (int f = 0; f < 3; f++) {
        r6 += qu[f] * m0r[4 + f];
        i6 += qu[f] * m0i[4 + f];
      }
      put(5, 3 + e, r5, i5);
      put(6, 3 + e, r6, i6);
      put(5, e, -m0r[1 + e], -m0i[1 + e]);
    }
    put(6, 0, m0r[1], m0i[1]);
    put(6, 1, m0r[2], m0i[2]);
    put(6, 2, -m0r[3], -m0i[3]);
  }
}

template <class T, int NK, int NT>
__global__ void __launch_bounds__(NT, 1)
k_p2m_unit(const P2MArgs a, const int* __restrict__ wleaves, const long long* __restrict__ hoff, int sbase,
           int ns, T* __restrict__ H) {
  constexpr int NF = NK == 7 ? 9 : 4;
  extern __shared__ __align__(16) unsigned char pu_smem[];
  const int p = a.p, nc = ncoef(p), D = 2 * nc, NY = unit_ylen(p);
  cplx* Ys = reinterpret_cast<cplx*>(pu_smem);    // [12][NY] node harmonics (extended rows)
  double* rtab = reinterpret_cast<double*>(Ys + 12 * NY);  // [nc]: 1/m! at (m, m), 1/((n-m)(n+m)) at n > m
  int* nmtab = reinterpret_cast<int*>(rtab + nc);          // [nc]: n | m << 16
  double* sct = reinterpret_cast<double*>(nmtab + nc + (nc & 1));  // [18]: row scales (re, im)
  T* geo = reinterpret_cast<T*>(sct + 18);                          // [12][4]: w, w y
  const int box = a.leaves[wleaves[blockIdx.x]];
  const int t0 = a.sstart[box], tn = a.scount[box];
  const int tl0 = blockIdx.y * UNIT_TB, tl1 = min(tn, tl0 + UNIT_TB);
  if (tl0 >= tn) return;
  const int tid = threadIdx.x, NTr = blockDim.x;
  const int lev = a.level[box];
  const double s = a.size / (double)(1ull << lev), is = 1.0 / s, q2 = is * is;
  double c[3];
  for (int d = 0; d < 3; d++) c[d] = a.c0[d] - a.size / 2 + (a.ijk[3 * box + d] - 1) * s + s / 2;
  double org[3];
  lame_origin(a.ijk, a.level, box, a.c0, a.size, a.flev, org);
  for (int i = tid; i < 12 * NY; i += NTr) Ys[i] = {0.0, 0.0};
  for (int i = tid; i < nc; i += NTr) {
    int n = 0;
    while ((n + 1) * (n + 2) / 2 <= i) n++;
    const int m = i - n * (n + 1) / 2;
    double f = 1.0;
    for (int k = 2; k <= m; k++) f /= k;
    rtab[i] = n > m ? 1.0 / ((double)(n - m) * (double)(n + m)) : f;
    nmtab[i] = n | (m << 16);
  }
  Quad12 Q;
  quad12(Q);
  const double lam = a.lam, mu = a.mu, al = a.alpha, c1 = a.c1, c2 = a.c2, inv2mu = a.inv2mu;
  const long long kstride = (long long)ns * tn * D;  // one kind of the leaf
  T* Hb = H + hoff[blockIdx.x];
  // scales of the feature rows (re, im) applied to the moments: the node
  // loop accumulates the unscaled ladder combinations below
  if (tid == 0) {
    const double sr9[9] = {1.0, 0.5 * is, 0.5 * is, is, 0.25 * q2, -0.25 * q2, 0.25 * q2, 0.5 * q2, 0.5 * q2};
    const double si9[9] = {-1.0, -0.5 * is, 0.5 * is, -is, -0.25 * q2, 0.25 * q2, 0.25 * q2, -0.5 * q2, 0.5 * q2};
    for (int f = 0; f < 9; f++) {
      sct[f] = sr9[f];
      sct[9 + f] = si9[f];
    }
  }
  const double* scr = sct;
  const double* sci = sct + 9;
  for (int tl = tl0; tl < tl1; tl++) {
    const int it = t0 + tl;
    const double* Tr = a.tri + 9 * (size_t)it;
    __syncthreads();  // the previous triangle's harmonics have been read (and the tables written)
    // column m of node j: Y_m^m = (-(z_x + i z_y)/2)^m / m!, then
    // Y_n^m = ((2n - 1) z_3 Y_{n-1}^m - |z|^2 Y_{n-2}^m) / ((n - m)(n + m))
    for (int task = tid; task < 12 * (p + 1); task += NTr) {
      const int m = task / 12, j = task % 12;
      double y[3];
      for (int d = 0; d < 3; d++) y[d] = Q.b[j][0] * Tr[d] + Q.b[j][1] * Tr[3 + d] + Q.b[j][2] * Tr[6 + d];
      const double z[3] = {(y[0] - c[0]) * is, (y[1] - c[1]) * is, (y[2] - c[2]) * is};
      const double r2 = z[0] * z[0] + z[1] * z[1] + z[2] * z[2];
      if (m == 0) {
        const double e1[3] = {Tr[3] - Tr[0], Tr[4] - Tr[1], Tr[5] - Tr[2]};
        const double e2[3] = {Tr[6] - Tr[0], Tr[7] - Tr[1], Tr[8] - Tr[2]};
        const double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                              e1[0] * e2[1] - e1[1] * e2[0]};
        const double w = Q.w[j] * 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        T* gq = geo + 4 * j;
        gq[0] = (T)w; gq[1] = (T)(w * (y[0] - org[0])); gq[2] = (T)(w * (y[1] - org[1]));
        gq[3] = (T)(w * (y[2] - org[2]));
      }
      cplx pw = {1.0, 0.0}, b = {-0.5 * z[0], -0.5 * z[1]};
      for (int e = m; e; e >>= 1) {
        if (e & 1) pw = cmul(pw, b);
        if (e > 1) b = cmul(b, b);
      }
      cplx* Y = Ys + (size_t)j * NY;
      cplx ym2 = {0, 0}, ym1 = cscale(rtab[cidx(m, m)], pw);
      for (int n = m;;) {
        Y[unit_yoff(n, m)] = ym1;
        if (m == 1) Y[unit_yoff(n, -1)] = {-ym1.re, ym1.im};
        if (m == 2) Y[unit_yoff(n, -2)] = {ym1.re, -ym1.im};
        if (++n > p) break;
        const double aa = (2.0 * n - 1.0) * z[2], inv = rtab[cidx(n, m)];
        const cplx yn = {(aa * ym1.re - r2 * ym2.re) * inv, (aa * ym1.im - r2 * ym2.im) * inv};
        ym2 = ym1;
        ym1 = yn;
      }
    }
    __syncthreads();
    const double* nv = a.nrm + 3 * (size_t)it;
    const double nn[3] = {nv[0], nv[1], nv[2]};
    for (int cc = tid; cc < nc; cc += NTr) {
      const int nm = nmtab[cc], fn = nm & 0xFFFF, fm = nm >> 16;
      const int o0 = unit_yoff(fn, fm), o1 = unit_yoff(fn - 1, fm), o2 = unit_yoff(fn - 2, fm);
      const double srd = a.wnorm ? a.wnorm[2 * cc] : 1.0;
      // moments (re, im) of the unscaled rows: M0 rows 0..NF-1, M1_e rows 0..3, M1_3 rows 4..8
      T m0r[NF], m0i[NF], m1r[3][4], m1i[3][4], mqr[5], mqi[5];
#pragma unroll
      for (int f = 0; f < NF; f++) m0r[f] = m0i[f] = (T)0;
#pragma unroll
      for (int e = 0; e < 3; e++)
#pragma unroll
        for (int f = 0; f < 4; f++) m1r[e][f] = m1i[e][f] = (T)0;
#pragma unroll
      for (int f = 0; f < 5; f++) mqr[f] = mqi[f] = (T)0;
#pragma unroll 1
      for (int j = 0; j < 12; j++) {
        const cplx* Y = Ys + (size_t)j * NY;
        const T* gq = geo + 4 * j;
        const T w = gq[0], wy[3] = {gq[1], gq[2], gq[3]};
        // Y, d_x, d_y, d_z (and xx, yy, xy, xz, yz) by the ladder relations, unscaled
        T fr[NF], fi[NF];
        // (the ladder sums in T, the harmonics scaled by the coefficient's
        // basis normalisation when one is given)
        auto ld = [&](int o, T& re, T& im) {
          const cplx v = Y[o];
          re = (T)(srd * v.re);
          im = (T)(srd * v.im);
        };
        T ar, ai, br, bi, cr, ci;
        ld(o0, fr[0], fi[0]);
        ld(o1, ar, ai);
        ld(o1 + 1, br, bi);
        ld(o1 - 1, cr, ci);
        fr[1] = br - cr; fi[1] = bi - ci;
        fr[2] = bi + ci; fi[2] = br + cr;
        fr[3] = ar; fi[3] = ai;
        if constexpr (NF == 9) {
          T zr, zi, p1r, p1i, m1r_, m1i_, p2r, p2i, m2r, m2i;
          ld(o2, zr, zi);
          ld(o2 + 1, p1r, p1i);
          ld(o2 - 1, m1r_, m1i_);
          ld(o2 + 2, p2r, p2i);
          ld(o2 - 2, m2r, m2i);
          fr[4] = p2r - 2 * zr + m2r; fi[4] = p2i - 2 * zi + m2i;
          fr[5] = p2r + 2 * zr + m2r; fi[5] = p2i + 2 * zi + m2i;
          fr[6] = p2i - m2i; fi[6] = p2r - m2r;
          fr[7] = p1r - m1r_; fi[7] = p1i - m1i_;
          fr[8] = p1i + m1i_; fi[8] = p1r + m1r_;
        }
#pragma unroll
        for (int f = 0; f < NF; f++) {
          m0r[f] += w * fr[f];
          m0i[f] += w * fi[f];
        }
#pragma unroll
        for (int e = 0; e < 3; e++)
#pragma unroll
          for (int f = 0; f < 4; f++) {
            m1r[e][f] += wy[e] * fr[f];
            m1i[e][f] += wy[e] * fi[f];
          }
        if constexpr (NF == 9) {
#pragma unroll
          for (int f = 0; f < 5; f++) {
            mqr[f] += wy[2] * fr[4 + f];
            mqi[f] += wy[2] * fi[4 + f];
          }
        }
      }
      // the row scales (conjugation signs, 1/s per derivative, ladder factors)
#pragma unroll
      for (int f = 0; f < NF; f++) {
        m0r[f] = (T)(scr[f] * m0r[f]);
        m0i[f] = (T)(sci[f] * m0i[f]);
      }
#pragma unroll
      for (int e = 0; e < 3; e++)
#pragma unroll
        for (int f = 0; f < 4; f++) {
          m1r[e][f] = (T)(scr[f] * m1r[e][f]);
          m1i[e][f] = (T)(sci[f] * m1i[e][f]);
        }
#pragma unroll
      for (int f = 0; f < 5; f++) {
        mqr[f] = (T)(scr[4 + f] * mqr[f]);
        mqi[f] = (T)(sci[4 + f] * mqi[f]);
      }
      // the combinations in T
      T* o = Hb + (size_t)(ns * tl) * D + 2 * cc;
      // column s (0..2 single layer, 3..5 double layer) of kind q, if carried
      auto put = [&](int q, int sidx, T vr, T vi) {
        const int sl = sidx - sbase;
        if (sl < 0 || sl >= ns) return;
        T* oo = o + q * kstride + (size_t)sl * D;
        oo[0] = vr;
        oo[1] = vi;
      };
      const T nv3[3] = {(T)nn[0], (T)nn[1], (T)nn[2]};
      unit_combine<T, NK>(put, m0r, m0i, m1r, m1i, mqr, mqi, nv3, (T)c1, (T)c2, (T)inv2mu, (T)al, (T)lam, (T)mu);
    }
  }
}

// FP32 form of k_p2m_unit (the mixed-precision P2M).  The node harmonics
// are computed in FP64 and stored in FP32 in the normalised basis
// Yh_n^m = Y_n^m sqrt((n + m)! (n - m)!) (bounded by |z|^n, no underflow);
// a coefficient (n, m) reads its ladder neighbours (n', m') times
// sqrt((n + m)! (n - m)! / ((n' + m')! (n' - m')!)), which yields the
// features of the normalised basis directly.  Two harmonic buffers: the
// recurrences of triangle t + 1 run while the moments of triangle t
// accumulate (one barrier per triangle).
constexpr int UNITF_THREADS = 512;

__host__ __device__ inline size_t unitf_smem(int p) {
  const size_t nc = (size_t)(p + 1) * (p + 2) / 2;
  return 2 * 12 * (size_t)unit_ylen(p) * sizeof(float2) + 2 * nc * sizeof(double) + 2 * 12 * 4 * sizeof(float) +
         18 * sizeof(float);
}

template <int NK>
__global__ void __launch_bounds__(UNITF_THREADS, 1)
k_p2m_unit_f(const P2MArgs a, const int* __restrict__ wleaves, const long long* __restrict__ hoff, int sbase,
             int ns, float* __restrict__ H, int split) {
  constexpr int NF = NK == 7 ? 9 : 4;
  extern __shared__ __align__(16) unsigned char pf_smem2[];
  const int p = a.p, nc = ncoef(p), D = 2 * nc, NY = unit_ylen(p);
  float2* Yb = reinterpret_cast<float2*>(pf_smem2);                  // [2][12][NY]
  double* rtab = reinterpret_cast<double*>(Yb + 2 * 12 * NY);        // [nc]: 1/m!, 1/((n-m)(n+m))
  double* wtab = rtab + nc;                                          // [nc]: sqrt((n+m)!(n-m)!)
  float* geo = reinterpret_cast<float*>(wtab + nc);                  // [2][12][4]: w, w y
  float* sct = geo + 2 * 12 * 4;                                     // [18]: row scales (re, im)
  const int box = a.leaves[wleaves[blockIdx.x]];
  const int t0 = a.sstart[box], tn = a.scount[box];
  const int tl0 = blockIdx.y * UNIT_TB, tl1 = min(tn, tl0 + UNIT_TB);
  if (tl0 >= tn) return;
  const int tid = threadIdx.x, NTr = blockDim.x;
  const int lev = a.level[box];
  const double s = a.size / (double)(1ull << lev), is = 1.0 / s, q2 = is * is;
  double c[3];
  for (int d = 0; d < 3; d++) c[d] = a.c0[d] - a.size / 2 + (a.ijk[3 * box + d] - 1) * s + s / 2;
  double org[3];
  lame_origin(a.ijk, a.level, box, a.c0, a.size, a.flev, org);
  for (int i = tid; i < 2 * 12 * NY; i += NTr) Yb[i] = make_float2(0.f, 0.f);
  for (int i = tid; i < nc; i += NTr) {
    int n = 0;
    while ((n + 1) * (n + 2) / 2 <= i) n++;
    const int m = i - n * (n + 1) / 2;
    double f = 1.0;
    for (int k = 2; k <= m; k++) f /= k;
    rtab[i] = n > m ? 1.0 / ((double)(n - m) * (double)(n + m)) : f;
    wtab[i] = a.wnorm[2 * i];
  }
  if (tid == 0) {
    const double sr9[9] = {1.0, 0.5 * is, 0.5 * is, is, 0.25 * q2, -0.25 * q2, 0.25 * q2, 0.5 * q2, 0.5 * q2};
    const double si9[9] = {-1.0, -0.5 * is, 0.5 * is, -is, -0.25 * q2, 0.25 * q2, 0.25 * q2, -0.5 * q2, 0.5 * q2};
    for (int f = 0; f < 9; f++) {
      sct[f] = (float)sr9[f];
      sct[9 + f] = (float)si9[f];
    }
  }
  Quad12 Q;
  quad12(Q);
  const float lam = (float)a.lam, mu = (float)a.mu, al = (float)a.alpha, c1 = (float)a.c1, c2 = (float)a.c2,
              inv2mu = (float)a.inv2mu;
  const long long kstride = (long long)ns * tn * D;  // one kind of the leaf
  float* Hb = H + hoff[blockIdx.x];
  // harmonics of the 12 nodes of triangle tl into buffer b: task (m, j) =
  // column m of node j, Y_m^m = (-(z_x + i z_y)/2)^m / m! then the recurrence
  // Y_n^m = ((2n - 1) z_3 Y_{n-1}^m - |z|^2 Y_{n-2}^m) / ((n - m)(n + m))
  // (tasks from the last thread down: the threads with one coefficient round
  // less take the longest columns)
  auto harmonics = [&](int tl, int b) {
    const double* Tr = a.tri + 9 * (size_t)(t0 + tl);
    for (int task = NTr - 1 - tid; task < 12 * (p + 1); task += NTr) {
      const int m = task / 12, j = task % 12;
      double y[3];
      for (int d = 0; d < 3; d++) y[d] = Q.b[j][0] * Tr[d] + Q.b[j][1] * Tr[3 + d] + Q.b[j][2] * Tr[6 + d];
      const double z[3] = {(y[0] - c[0]) * is, (y[1] - c[1]) * is, (y[2] - c[2]) * is};
      const double r2 = z[0] * z[0] + z[1] * z[1] + z[2] * z[2];
      if (m == 0) {
        const double e1[3] = {Tr[3] - Tr[0], Tr[4] - Tr[1], Tr[5] - Tr[2]};
        const double e2[3] = {Tr[6] - Tr[0], Tr[7] - Tr[1], Tr[8] - Tr[2]};
        const double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                              e1[0] * e2[1] - e1[1] * e2[0]};
        const double w = Q.w[j] * 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        float* gq = geo + (b * 12 + j) * 4;
        gq[0] = (float)w; gq[1] = (float)(w * (y[0] - org[0])); gq[2] = (float)(w * (y[1] - org[1]));
        gq[3] = (float)(w * (y[2] - org[2]));
      }
      cplx pw = {1.0, 0.0}, bb = {-0.5 * z[0], -0.5 * z[1]};
      for (int e = m; e; e >>= 1) {
        if (e & 1) pw = cmul(pw, bb);
        if (e > 1) bb = cmul(bb, bb);
      }
      float2* Y = Yb + (size_t)(b * 12 + j) * NY;
      cplx ym2 = {0, 0}, ym1 = cscale(rtab[cidx(m, m)], pw);
      for (int n = m;;) {
        const double wn = wtab[cidx(n, m)];
        const float2 v = make_float2((float)(wn * ym1.re), (float)(wn * ym1.im));
        Y[unit_yoff(n, m)] = v;
        if (m == 1) Y[unit_yoff(n, -1)] = make_float2(-v.x, v.y);
        if (m == 2) Y[unit_yoff(n, -2)] = make_float2(v.x, -v.y);
        if (++n > p) break;
        const double aa = (2.0 * n - 1.0) * z[2], inv = rtab[cidx(n, m)];
        const cplx yn = {(aa * ym1.re - r2 * ym2.re) * inv, (aa * ym1.im - r2 * ym2.im) * inv};
        ym2 = ym1;
        ym1 = yn;
      }
    }
  };
  __syncthreads();  // zeroed buffers and tables
  harmonics(tl0, 0);
  __syncthreads();
  for (int tl = tl0; tl < tl1; tl++) {
    const int b = (tl - tl0) & 1;
    if (tl + 1 < tl1) harmonics(tl + 1, b ^ 1);
    const double* nvp = a.nrm + 3 * (size_t)(t0 + tl);
    const float nv3[3] = {(float)nvp[0], (float)nvp[1], (float)nvp[2]};
    for (int cc = tid; cc < nc; cc += NTr) {
      int fn = (int)((sqrtf(8.0f * cc + 1.0f) - 1.0f) * 0.5f);
      while ((fn + 1) * (fn + 2) / 2 <= cc) fn++;
      while (fn * (fn + 1) / 2 > cc) fn--;
      const int fm = cc - fn * (fn + 1) / 2;
      const float np_ = (float)(fn + fm), nm_ = (float)(fn - fm);
      // normalisation ratios of the ladder neighbours (0 where the neighbour is outside the table)
      auto rt = [](float x) { return sqrtf(fmaxf(x, 0.0f)); };
      const float rA = rt(np_ * nm_), rB = rt(nm_ * (nm_ - 1)), rC = rt(np_ * (np_ - 1));
      const float rZ = rt(np_ * (np_ - 1) * nm_ * (nm_ - 1)), rP1 = rt(np_ * nm_ * (nm_ - 1) * (nm_ - 2));
      const float rM1 = rt(np_ * (np_ - 1) * (np_ - 2) * nm_), rP2 = rt(nm_ * (nm_ - 1) * (nm_ - 2) * (nm_ - 3));
      const float rM2 = rt(np_ * (np_ - 1) * (np_ - 2) * (np_ - 3));
      const int o0 = unit_yoff(fn, fm), o1 = unit_yoff(fn - 1, fm), o2 = unit_yoff(fn - 2, fm);
      float m0r[NF], m0i[NF], m1r[3][4], m1i[3][4], mqr[5], mqi[5];
#pragma unroll
      for (int f = 0; f < NF; f++) m0r[f] = m0i[f] = 0.f;
#pragma unroll
      for (int e = 0; e < 3; e++)
#pragma unroll
        for (int f = 0; f < 4; f++) m1r[e][f] = m1i[e][f] = 0.f;
#pragma unroll
      for (int f = 0; f < 5; f++) mqr[f] = mqi[f] = 0.f;
#pragma unroll 1
      for (int j = 0; j < 12; j++) {
        const float2* Y = Yb + (size_t)(b * 12 + j) * NY;
        const float* gq = geo + (b * 12 + j) * 4;
        const float w = gq[0], wy[3] = {gq[1], gq[2], gq[3]};
        float fr[NF], fi[NF];
        const float2 v0 = Y[o0], A = Y[o1], B = Y[o1 + 1], C = Y[o1 - 1];
        fr[0] = v0.x; fi[0] = v0.y;
        fr[1] = rB * B.x - rC * C.x; fi[1] = rB * B.y - rC * C.y;
        fr[2] = rB * B.y + rC * C.y; fi[2] = rB * B.x + rC * C.x;
        fr[3] = rA * A.x; fi[3] = rA * A.y;
        if constexpr (NF == 9) {
          const float2 Z = Y[o2], P1 = Y[o2 + 1], M1 = Y[o2 - 1], P2 = Y[o2 + 2], M2 = Y[o2 - 2];
          const float zr = 2 * rZ * Z.x, zi = 2 * rZ * Z.y;
          fr[4] = rP2 * P2.x - zr + rM2 * M2.x; fi[4] = rP2 * P2.y - zi + rM2 * M2.y;
          fr[5] = rP2 * P2.x + zr + rM2 * M2.x; fi[5] = rP2 * P2.y + zi + rM2 * M2.y;
          fr[6] = rP2 * P2.y - rM2 * M2.y; fi[6] = rP2 * P2.x - rM2 * M2.x;
          fr[7] = rP1 * P1.x - rM1 * M1.x; fi[7] = rP1 * P1.y - rM1 * M1.y;
          fr[8] = rP1 * P1.y + rM1 * M1.y; fi[8] = rP1 * P1.x + rM1 * M1.x;
        }
#pragma unroll
        for (int f = 0; f < NF; f++) {
          m0r[f] += w * fr[f];
          m0i[f] += w * fi[f];
        }
#pragma unroll
        for (int e = 0; e < 3; e++)
#pragma unroll
          for (int f = 0; f < 4; f++) {
            m1r[e][f] += wy[e] * fr[f];
            m1i[e][f] += wy[e] * fi[f];
          }
        if constexpr (NF == 9) {
#pragma unroll
          for (int f = 0; f < 5; f++) {
            mqr[f] += wy[2] * fr[4 + f];
            mqi[f] += wy[2] * fi[4 + f];
          }
        }
      }
      const float* scr = sct;
      const float* sci = sct + 9;
#pragma unroll
      for (int f = 0; f < NF; f++) {
        m0r[f] *= scr[f];
        m0i[f] *= sci[f];
      }
#pragma unroll
      for (int e = 0; e < 3; e++)
#pragma unroll
        for (int f = 0; f < 4; f++) {
          m1r[e][f] *= scr[f];
          m1i[e][f] *= sci[f];
        }
#pragma unroll
      for (int f = 0; f < 5; f++) {
        mqr[f] *= scr[4 + f];
        mqi[f] *= sci[4 + f];
      }
      float* o = Hb + (size_t)(ns * tl) * D + 2 * cc;
      auto put = [&](int q, int sidx, float vr, float vi) {
        const int sl = sidx - sbase;
        if (sl < 0 || sl >= ns) return;
        if (split) {
          // split tiles: kind q's (row, k = ns tl + sl) in tile (row / 128, k / 32)
          const int k = ns * tl + sl, kl = k & 31, nmt = (D + 127) / 128, snkt = (ns * tn + 31) / 32;
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const int row = 2 * cc + h;
            float* tile = Hb + ((long long)(q * nmt + (row >> 7)) * snkt + (k >> 5)) * 8192;
            const int idx = (kl & 3) + 4 * (row & 7) + 32 * (kl >> 2) + 256 * ((row & 127) >> 3);
            const float v = h ? vi : vr, hd = tf32_head(v);
            tile[idx] = hd;
            tile[4096 + idx] = v - hd;
          }
          return;
        }
        float* oo = o + q * kstride + (size_t)sl * D;
        oo[0] = vr;
        oo[1] = vi;
      };
      unit_combine<float, NK>(put, m0r, m0i, m1r, m1i, mqr, mqi, nv3, c1, c2, inv2mu, al, lam, mu);
    }
    __syncthreads();  // buffer b is free, buffer b ^ 1 complete
  }
}

// Densities of the leaves as the B operand of the factored P2M product:
// per leaf at soff, R rows of Kp = ns tn rounded up to 4, entry ns t + j =
// density component sbase + j of triangle t (components 0..2 single layer,
// 3..5 double layer).
template <class T>
__global__ void __launch_bounds__(256)
k_p2m_sigma(const P2MArgs a, int R, const int* __restrict__ wleaves, const long long* __restrict__ soff,
            int sbase, int ns, T* __restrict__ S) {
  const int box = a.leaves[wleaves[blockIdx.x]];
  const int t0 = a.sstart[box], tn = a.scount[box];
  const int K = ns * tn, Kp = (K + 3) & ~3;
  T* out = S + soff[blockIdx.x];
  for (long long q = blockIdx.y * (long long)blockDim.x + threadIdx.x; q < (long long)R * Kp;
       q += (long long)gridDim.y * blockDim.x) {
    const int r = (int)(q / Kp), k = (int)(q % Kp);
    double v = 0.0;
    if (k < K) {
      const int tl = k / ns, sc = sbase + k % ns;
      const long long off = r * a.rstride + (long long)(t0 + tl) * a.tstride + (sc % 3) * a.dstride;
      if (sc < 3) {
        if (a.dosl) v = a.ssl[off];
      } else if (a.dodl) {
        v = a.sdl[off];
      }
    }
    out[q] = (T)v;
  }
}

// The densities of each leaf of the wave as split B tiles of 64 columns
// (right-hand sides) x 32 k (k = ns t + j: density component sbase + j of the
// leaf's triangle t), 4096 floats a tile (TF32 head then tail, canonical
// layout; column tile ct, K tile kt at soff[i] + (ct nkt + kt) 4096);
// positions past R or K written as zeros.  A tile is read k-fastest into
// shared memory (rows of 36 floats) and written in tile order.
__global__ void __launch_bounds__(256)
k_p2m_sigma_split(const P2MArgs a, int R, const int* __restrict__ wleaves, const long long* __restrict__ soff,
                  int sbase, int ns, float* __restrict__ S) {
  __shared__ float sv[64][36];
  const int box = a.leaves[wleaves[blockIdx.x]];
  const int t0 = a.sstart[box], tn = a.scount[box];
  const int K = ns * tn, nkt = (K + 31) / 32, nct = (R + 63) / 64;
  float* o = S + soff[blockIdx.x];
  for (int tile = blockIdx.y; tile < nct * nkt; tile += gridDim.y) {
    const int ct = tile / nkt, kt = tile % nkt;
    __syncthreads();  // the previous tile's reads of sv are done
    for (int q = threadIdx.x; q < 2048; q += blockDim.x) {
      const int k = q & 31, n = q >> 5, r = 64 * ct + n, kk = 32 * kt + k;
      float v = 0.0f;
      if (r < R && kk < K) {
        const int tl = kk / ns, sc = sbase + kk % ns;
        const long long off = r * a.rstride + (long long)(t0 + tl) * a.tstride + (sc % 3) * a.dstride;
        if (sc < 3) {
          if (a.dosl) v = (float)a.ssl[off];
        } else if (a.dodl) {
          v = (float)a.sdl[off];
        }
      }
      sv[n][k] = v;
    }
    __syncthreads();
    float* t = o + (long long)tile * 4096;
    for (int q = threadIdx.x; q < 2048; q += blockDim.x) {
      const int k = (q & 3) | (((q >> 5) & 7) << 2), n = ((q >> 2) & 7) | ((q >> 8) << 3);
      const float v = sv[n][k], h = tf32_head(v);
      t[q] = h;
      t[2048 + q] = v - h;
    }
  }
}

// Direct image P2M (few right-hand sides): one CTA per (leaf, right-hand
// side r = blockIdx.y), nodes in batches of P2M_NODES (one warp each builds
// the regular harmonics), every thread accumulating 7 columns of its
// coefficients from the charge, dipole and second-derivative terms.  T =
// float writes the normalised basis (x wnorm).
template <class T>
__global__ void __launch_bounds__(P2M_THREADS)
k_p2m_img(const P2MArgs a, int R, long long ubase, T* __restrict__ mpole) {
  extern __shared__ double sm[];
  const int box = a.leaves[blockIdx.x];
  const int p = a.p, nc = ncoef(p), D = 2 * nc;
  cplx* Ys = reinterpret_cast<cplx*>(sm);             // [P2M_NODES][nc]
  double* qd = sm + 2 * (size_t)P2M_NODES * nc;       // [P2M_NODES][7][9]
  const int lev = a.level[box];
  const double s = a.size / (double)(1ull << lev), is = 1.0 / s;
  double c[3];
  for (int d = 0; d < 3; d++) c[d] = a.c0[d] - a.size / 2 + (a.ijk[3 * box + d] - 1) * s + s / 2;
  double org[3];
  lame_origin(a.ijk, a.level, box, a.c0, a.size, a.flev, org);
  const int t0 = a.sstart[box], tn = a.scount[box];
  const int nnode = a.points ? tn : 12 * tn;
  constexpr int CMAX = 6;  // coefficients per thread (ncoef(p) <= 1536)
  double acc[CMAX][7][2];
#pragma unroll
  for (int i = 0; i < CMAX; i++)
#pragma unroll
    for (int q = 0; q < 7; q++) acc[i][q][0] = acc[i][q][1] = 0.0;
  Quad12 Q;
  quad12(Q);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = blockIdx.y;
  for (int b0 = 0; b0 < nnode; b0 += P2M_NODES) {
    __syncthreads();
    const int node = b0 + warp;
    if (node < nnode) {
      int it;
      double y[3], w;
      if (a.points) {  // a particle: one node of weight 1
        it = t0 + node;
        for (int d = 0; d < 3; d++) y[d] = a.pts[3 * (size_t)it + d];
        w = 1.0;
      } else {
        it = t0 + node / 12;
        const int iq = node % 12;
        const double* Tr = a.tri + 9 * (size_t)it;
        for (int d = 0; d < 3; d++) y[d] = Q.b[iq][0] * Tr[d] + Q.b[iq][1] * Tr[3 + d] + Q.b[iq][2] * Tr[6 + d];
        const double e1[3] = {Tr[3] - Tr[0], Tr[4] - Tr[1], Tr[5] - Tr[2]};
        const double e2[3] = {Tr[6] - Tr[0], Tr[7] - Tr[1], Tr[8] - Tr[2]};
        const double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                              e1[0] * e2[1] - e1[1] * e2[0]};
        w = Q.w[iq] * 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
      }
      const double z[3] = {(y[0] - c[0]) * is, (y[1] - c[1]) * is, (y[2] - c[2]) * is};
      cplx* Y = Ys + (size_t)warp * nc;
      const double r2 = z[0] * z[0] + z[1] * z[1] + z[2] * z[2];
      for (int m = lane; m <= p; m += 32) {
        cplx dm = {1.0, 0.0}, wv = {-0.5 * z[0], -0.5 * z[1]};
        for (int k = 1; k <= m; k++) dm = cscale(1.0 / k, cmul(dm, wv));
        Y[cidx(m, m)] = dm;
        cplx ym2 = {0, 0}, ym1 = dm;
        for (int n = m + 1; n <= p; n++) {
          const double aa = (2.0 * n - 1.0) * z[2];
          const double inv = 1.0 / ((double)(n - m) * (double)(n + m));
          cplx yn = {(aa * ym1.re - r2 * ym2.re) * inv, (aa * ym1.im - r2 * ym2.im) * inv};
          Y[cidx(n, m)] = yn;
          ym2 = ym1;
          ym1 = yn;
        }
      }
      if (lane < 7) {
        const long long off = r * a.rstride + it * a.tstride, ds = a.dstride;
        const double* nn = a.nrm + 3 * (size_t)it;
        double sl[3] = {0, 0, 0}, dl[3] = {0, 0, 0};
        if (a.dosl) { sl[0] = a.ssl[off]; sl[1] = a.ssl[off + ds]; sl[2] = a.ssl[off + 2 * ds]; }
        if (a.dodl) { dl[0] = a.sdl[off]; dl[1] = a.sdl[off + ds]; dl[2] = a.sdl[off + 2 * ds]; }
        const double nv[3] = {nn[0], nn[1], nn[2]};
        double wv[9];
        const double yo[3] = {y[0] - org[0], y[1] - org[1], y[2] - org[2]};
        img_node_weights(lane, sl, dl, nv, yo, a, wv);
        for (int k = 0; k < 9; k++) qd[(warp * 7 + lane) * 9 + k] = w * wv[k];
      }
    }
    __syncthreads();
    const int nb = min(P2M_NODES, nnode - b0);
#pragma unroll
    for (int i = 0; i < CMAX; i++) {
      const int cc = threadIdx.x + i * P2M_THREADS;
      if (cc >= nc) break;
      int n = 0;
      while ((n + 1) * (n + 2) / 2 <= cc) n++;
      const int m = cc - n * (n + 1) / 2;
      for (int k = 0; k < nb; k++) {
        const cplx* Y = Ys + (size_t)k * nc;
        // conjugated feature values (re, im) of rows: Y, d_x, d_y, d_z, xx, yy, xy, xz, yz
        double fr[9], fi[9];
        const cplx y = Y[cc];
        fr[0] = y.re; fi[0] = -y.im;
        cplx ya = {0, 0}, yb = {0, 0}, yc = {0, 0};
        if (n > 0) {
          ya = hget(Y, n - 1, m);
          yb = hget(Y, n - 1, m + 1);
          yc = hget(Y, n - 1, m - 1);
        }
        fr[1] = 0.5 * is * (yb.re - yc.re); fi[1] = -0.5 * is * (yb.im - yc.im);
        fr[2] = 0.5 * is * (yb.im + yc.im); fi[2] = 0.5 * is * (yb.re + yc.re);
        fr[3] = is * ya.re; fi[3] = -is * ya.im;
        cplx y0 = {0, 0}, yp1 = {0, 0}, ym1 = {0, 0}, yp2 = {0, 0}, ym2 = {0, 0};
        if (n > 1) {
          y0 = hget(Y, n - 2, m);
          yp1 = hget(Y, n - 2, m + 1);
          ym1 = hget(Y, n - 2, m - 1);
          yp2 = hget(Y, n - 2, m + 2);
          ym2 = hget(Y, n - 2, m - 2);
        }
        const double q2 = is * is;
        fr[4] = q2 * 0.25 * (yp2.re - 2.0 * y0.re + ym2.re); fi[4] = -q2 * 0.25 * (yp2.im - 2.0 * y0.im + ym2.im);
        fr[5] = -q2 * 0.25 * (yp2.re + 2.0 * y0.re + ym2.re); fi[5] = q2 * 0.25 * (yp2.im + 2.0 * y0.im + ym2.im);
        fr[6] = q2 * 0.25 * (yp2.im - ym2.im); fi[6] = q2 * 0.25 * (yp2.re - ym2.re);
        fr[7] = q2 * 0.5 * (yp1.re - ym1.re); fi[7] = -q2 * 0.5 * (yp1.im - ym1.im);
        fr[8] = q2 * 0.5 * (yp1.im + ym1.im); fi[8] = q2 * 0.5 * (yp1.re + ym1.re);
        const double* o = qd + (size_t)k * 63;
#pragma unroll
        for (int q = 0; q < 7; q++) {
          double ar = 0.0, ai = 0.0;
#pragma unroll
          for (int f = 0; f < 9; f++) {
            ar += o[9 * q + f] * fr[f];
            ai += o[9 * q + f] * fi[f];
          }
          acc[i][q][0] += ar;
          acc[i][q][1] += ai;
        }
      }
    }
  }
#pragma unroll
  for (int i = 0; i < CMAX; i++) {
    const int cc = threadIdx.x + i * P2M_THREADS;
    if (cc >= nc) break;
    const double sr = a.wnorm ? a.wnorm[2 * cc] : 1.0;
#pragma unroll
    for (int q = 0; q < 7; q++) {
      T* M = q < 6 ? mpole + ((size_t)box * 6 * R + (size_t)q * R + r) * D
                   : mpole + ubase + ((size_t)box * R + r) * D;
      M[2 * cc] = (T)(sr * acc[i][q][0]);
      M[2 * cc + 1] = (T)(sr * acc[i][q][1]);
    }
  }
}

template <class T>
__global__ void __launch_bounds__(256)
k_p2m_weights(const P2MArgs a, int R, const int* __restrict__ wleaves, const long long* __restrict__ woff,
              const long long* __restrict__ noff, const double* __restrict__ nrec, T* __restrict__ W) {
  const int box = a.leaves[wleaves[blockIdx.x]];
  const int tn = a.scount[box];
  const int nnode = 12 * tn, K = 4 * nnode, C = 4 * R;
  const double c1 = a.c1, c2 = a.c2, inv2mu = a.inv2mu;
  const double* nd = nrec + 8 * noff[blockIdx.x];
  T* out = W + woff[blockIdx.x];
  for (long long q = blockIdx.y * (long long)blockDim.x + threadIdx.x; q < (long long)nnode * C;
       q += (long long)gridDim.y * blockDim.x) {
    const int col = (int)(q / nnode), node = (int)(q % nnode);
    const int r = col >> 2, pass = col & 3;
    const double* o = nd + 8 * node;
    const double y[3] = {o[0], o[1], o[2]}, nn[3] = {o[3], o[4], o[5]}, w = o[6];
    const long long it = (long long)o[7];
    const long long off = r * a.rstride + it * a.tstride, ds = a.dstride;
    double sl[3] = {0, 0, 0}, dl[3] = {0, 0, 0};
    if (a.dosl) { sl[0] = a.ssl[off]; sl[1] = a.ssl[off + ds]; sl[2] = a.ssl[off + 2 * ds]; }
    if (a.dodl) { dl[0] = a.sdl[off]; dl[1] = a.sdl[off + ds]; dl[2] = a.sdl[off + 2 * ds]; }
    double wv[4];
    if (pass < 3) {
      wv[0] = w * sl[pass] * inv2mu;
      for (int d = 0; d < 3; d++) wv[1 + d] = w * 0.5 * (nn[d] * dl[pass] + dl[d] * nn[pass]);
    } else {
      const double sly = sl[0] * y[0] + sl[1] * y[1] + sl[2] * y[2];
      const double dly = dl[0] * y[0] + dl[1] * y[1] + dl[2] * y[2];
      const double dln = dl[0] * nn[0] + dl[1] * nn[1] + dl[2] * nn[2];
      const double ny = nn[0] * y[0] + nn[1] * y[1] + nn[2] * y[2];
      wv[0] = w * (sly * c1 * inv2mu + dln * c2);
      for (int d = 0; d < 3; d++) wv[1 + d] = w * 0.5 * c1 * (nn[d] * dly + dl[d] * ny);
    }
    T* ow = out + (size_t)col * K + 4 * node;
#pragma unroll
    for (int k = 0; k < 4; k++) ow[k] = (T)wv[k];
  }
}

// Batched product  C[col][row] = sum_k A[k][row] * B[col][k]  over 128 x 128
// output tiles (GemmTask), 8 x 8 outputs per thread, K tiles of 16
// double-buffered in shared memory; C is stored (each task owns its tile).
template <class T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1)
k_gemm_tn(const GemmTask* __restrict__ tasks, const T* __restrict__ A, const T* __restrict__ B,
          T* __restrict__ Cm) {
  using V2 = typename Vec2<T>::type;
  extern __shared__ __align__(16) unsigned char gt_smem[];
  T* As = reinterpret_cast<T*>(gt_smem);  // [2][16][128]
  T* Bs = As + 2 * 16 * 128;              // [2][16][128]
  const GemmTask t = tasks[blockIdx.x];
  const int tid = threadIdx.x;
  // A loader: k row (tid >> 4), 8 consecutive output rows from (tid & 15) * 8
  const int ak = tid >> 4, ar = (tid & 15) * 8;
  const T* Ap = A + t.a_off + t.row0 + ar;
  const bool arow_all = t.row0 + ar + 8 <= t.M;
  // B loader: column (tid & 127), k half (tid >> 7)
  const int bcol = tid & 127, bkh = (tid >> 7) * 8;
  const bool bcol_ok = t.col0 + bcol < t.N;
  const T* Bp = B + t.b_off + (size_t)(bcol_ok ? t.col0 + bcol : 0) * t.ldb;
  T ra[8], rb[8];
  auto load = [&](int k0) {
    const int k = k0 + ak;
    if (k < t.K && arow_all) {
#pragma unroll
      for (int i = 0; i < 4; i++) {
        V2 v = *reinterpret_cast<const V2*>(Ap + (size_t)k * t.lda + 2 * i);
        ra[2 * i] = v.x;
        ra[2 * i + 1] = v.y;
      }
    } else {
#pragma unroll
      for (int i = 0; i < 8; i++)
        ra[i] = (k < t.K && t.row0 + ar + i < t.M) ? Ap[(size_t)k * t.lda + i] : T(0);
    }
    const int kb = k0 + bkh;
    if (bcol_ok && kb + 8 <= t.K) {
#pragma unroll
      for (int i = 0; i < 4; i++) {
        V2 v = *reinterpret_cast<const V2*>(Bp + kb + 2 * i);
        rb[2 * i] = v.x;
        rb[2 * i + 1] = v.y;
      }
    } else {
#pragma unroll
      for (int i = 0; i < 8; i++) rb[i] = (bcol_ok && kb + i < t.K) ? Bp[kb + i] : T(0);
    }
  };
  auto store = [&](int buf) {
    T* as = As + buf * 16 * 128;
    T* bs = Bs + buf * 16 * 128;
#pragma unroll
    for (int i = 0; i < 8; i++) as[ak * 128 + ar + i] = ra[i];
#pragma unroll
    for (int i = 0; i < 8; i++) bs[(bkh + i) * 128 + bcol] = rb[i];
  };
  const int tx = tid & 15, ty = tid >> 4;
  T acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) acc[i][j] = T(0);
  const int nk = (t.K + 15) / 16;
  load(0);
  store(0);
  __syncthreads();
  for (int kt = 0; kt < nk; kt++) {
    const int cur = kt & 1;
    if (kt + 1 < nk) load((kt + 1) * 16);
    const T* as = As + cur * 16 * 128;
    const T* bs = Bs + cur * 16 * 128;
#pragma unroll
    for (int kk = 0; kk < 16; kk++) {
      T av[8], bv[8];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        V2 v = *reinterpret_cast<const V2*>(as + kk * 128 + ty * 8 + 2 * i);
        av[2 * i] = v.x;
        av[2 * i + 1] = v.y;
      }
#pragma unroll
      for (int j = 0; j < 4; j++) {
        V2 v = *reinterpret_cast<const V2*>(bs + kk * 128 + 32 * j + 2 * tx);
        bv[2 * j] = v.x;
        bv[2 * j + 1] = v.y;
      }
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] += av[i] * bv[j];
    }
    if (kt + 1 < nk) store(cur ^ 1);
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const int col = t.col0 + 32 * (j >> 1) + 2 * tx + (j & 1);
    if (col >= t.N) continue;
    T* cp = Cm + t.c_off + (size_t)col * t.ldc;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int r = t.row0 + ty * 8 + i;
      if (r < t.M) cp[r] = acc[i][j];
    }
  }
}

// --------------------------------------------------- grouped translations
// A task is one 128 x 128 output tile of the product Op(group) * B, where B's
// columns are the concatenated columns of the group's (src, dst) pairs: column
// j of the task is column c = (col0 + j) % C of pair pair0 + (col0 + j) / C.
// Each box carries C columns (4 Laplace passes x right-hand sides) of length D.
//   dst[pair.dst][c][rows] += alpha * Op[rows][:] * src[pair.src][c][:]
// 256 threads, 8 x 8 outputs per thread, K tiles of 16 double-buffered in
// shared memory (one barrier per tile), results scattered with atomics (the
// pairs of one group have distinct destinations, different groups overlap).
constexpr int TR_R = 128, TR_C = 128, TR_K = 16;

template <class T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1)
k_translate(const TransTask* __restrict__ tasks, const TransPair* __restrict__ pairs,
            const T* __restrict__ mats, const long long* __restrict__ mat_off,
            const int* __restrict__ mat_dim, int D, int C, const T* __restrict__ src,
            T* __restrict__ dst) {
  using V2 = typename Vec2<T>::type;
  extern __shared__ __align__(16) unsigned char tr_smem[];
  T* As = reinterpret_cast<T*>(tr_smem);          // [2][TR_K][TR_R]
  T* Bs = As + 2 * TR_K * TR_R;                    // [2][TR_K][TR_C]
  const TransTask t = tasks[blockIdx.x];
  const T* A = mats + mat_off[t.group];
  const int dim = mat_dim[t.group];
  const int r0 = t.row0;
  const int tid = threadIdx.x;
  // loader roles: A row (tid >> 1), k half (tid & 1); B column (tid & 127), k half (tid >> 7)
  const int arow = tid >> 1, akh = (tid & 1) * 8;
  const bool arow_ok = r0 + arow < dim;
  const T* Ap = A + (size_t)(arow_ok ? r0 + arow : 0) * dim;
  const int bcol = tid & 127, bkh = (tid >> 7) * 8;
  const T* Bp = nullptr;
  {
    int col = t.col0 + bcol;
    if (col < t.ncols) {
      const TransPair pr = pairs[t.pair0 + col / C];
      Bp = src + ((size_t)pr.src * C + (col % C)) * D;
    }
  }
  T ra[8], rb[8];
  auto load = [&](int k0) {
    int ka = k0 + akh, kb = k0 + bkh;
    if (arow_ok && ka + 8 <= dim) {
#pragma unroll
      for (int i = 0; i < 4; i++) {
        V2 v = *reinterpret_cast<const V2*>(Ap + ka + 2 * i);
        ra[2 * i] = v.x;
        ra[2 * i + 1] = v.y;
      }
    } else {
#pragma unroll
      for (int i = 0; i < 8; i++) ra[i] = (arow_ok && ka + i < dim) ? Ap[ka + i] : T(0);
    }
    if (Bp && kb + 8 <= dim) {
#pragma unroll
      for (int i = 0; i < 4; i++) {
        V2 v = *reinterpret_cast<const V2*>(Bp + kb + 2 * i);
        rb[2 * i] = v.x;
        rb[2 * i + 1] = v.y;
      }
    } else {
#pragma unroll
      for (int i = 0; i < 8; i++) rb[i] = (Bp && kb + i < dim) ? Bp[kb + i] : T(0);
    }
  };
  auto store = [&](int buf) {
    T* as = As + buf * TR_K * TR_R;
    T* bs = Bs + buf * TR_K * TR_C;
#pragma unroll
    for (int i = 0; i < 8; i++) as[(akh + i) * TR_R + arow] = ra[i];
#pragma unroll
    for (int i = 0; i < 8; i++) bs[(bkh + i) * TR_C + bcol] = rb[i];
  };
  const int tx = tid & 15, ty = tid >> 4;
  T acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) acc[i][j] = T(0);
  const int nk = (dim + TR_K - 1) / TR_K;
  load(0);
  store(0);
  __syncthreads();
  for (int kt = 0; kt < nk; kt++) {
    const int cur = kt & 1;
    if (kt + 1 < nk) load((kt + 1) * TR_K);
    const T* as = As + cur * TR_K * TR_R;
    const T* bs = Bs + cur * TR_K * TR_C;
#pragma unroll
    for (int kk = 0; kk < TR_K; kk++) {
      T a[8], b[8];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        V2 v = *reinterpret_cast<const V2*>(as + kk * TR_R + ty * 8 + 2 * i);
        a[2 * i] = v.x;
        a[2 * i + 1] = v.y;
      }
#pragma unroll
      for (int j = 0; j < 4; j++) {
        V2 v = *reinterpret_cast<const V2*>(bs + kk * TR_C + 32 * j + 2 * tx);
        b[2 * j] = v.x;
        b[2 * j + 1] = v.y;
      }
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] += a[i] * b[j];
    }
    if (kt + 1 < nk) store(cur ^ 1);
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 8; j++) {
    int col = t.col0 + 32 * (j >> 1) + 2 * tx + (j & 1);
    if (col >= t.ncols) continue;
    const TransPair pr = pairs[t.pair0 + col / C];
    T* dp = dst + ((size_t)pr.dst * C + (col % C)) * D;
    T al = (T)pr.alpha;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      int r = r0 + ty * 8 + i;
      if (r < dim) atomicAdd(dp + r, al * acc[i][j]);
    }
  }
}

// ------------------------------------------------- L2T + recombination
constexpr int L2T_WARPS = 8;

__global__ void __launch_bounds__(L2T_WARPS * 32)
k_l2t(const L2TArgs a) {
  // blockDim.x = 32 * (number of warps); each warp owns one Y table in smem
  extern __shared__ double sm[];
  int box = a.leaves[blockIdx.x];
  int p = a.p, nc = ncoef(p), D = 2 * nc;
  double* Ls = sm;                                              // [4][D]
  cplx* Yall = reinterpret_cast<cplx*>(sm + 4 * (size_t)D);     // [warps][nc]
  const double* L = a.local + ((size_t)box * a.C + 4 * blockIdx.y) * D;
  for (int q = threadIdx.x; q < 4 * D; q += blockDim.x) Ls[q] = L[q];
  int lev = a.level[box];
  double s = a.size / (double)(1ull << lev);
  double c[3];
  for (int d = 0; d < 3; d++) c[d] = a.c0[d] - a.size / 2 + (a.ijk[3 * box + d] - 1) * s + s / 2;
  double org[3];
  lame_origin(a.ijk, a.level, box, a.c0, a.size, a.flev, org);
  __syncthreads();
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  cplx* Y = Yall + (size_t)warp * nc;
  int sn = a.do_src ? a.scount[box] : 0, tn = a.do_tgt ? a.tcount[box] : 0;
  int s0 = a.sstart[box], t0 = a.tstart[box];
  double is = 1.0 / s, is2 = is * is;
  int nw = blockDim.x >> 5;
  for (int e = warp; e < sn + tn; e += nw) {
    bool is_src = e < sn;
    int pidx = is_src ? s0 + e : t0 + (e - sn);
    const double* X = is_src ? a.src_pts + 3 * (size_t)pidx : a.tgt_pts + 3 * (size_t)pidx;
    double x[3] = {X[0], X[1], X[2]};
    double z[3] = {(x[0] - c[0]) * is, (x[1] - c[1]) * is, (x[2] - c[2]) * is};
    __syncwarp();
    double r2 = z[0] * z[0] + z[1] * z[1] + z[2] * z[2];
    for (int m = lane; m <= p; m += 32) {
      cplx dm = {1.0, 0.0}, wv = {-0.5 * z[0], -0.5 * z[1]};
      for (int k = 1; k <= m; k++) dm = cscale(1.0 / k, cmul(dm, wv));
      Y[cidx(m, m)] = dm;
      cplx ym2 = {0, 0}, ym1 = dm;
      for (int n = m + 1; n <= p; n++) {
        double aa = (2.0 * n - 1.0) * z[2];
        double inv = 1.0 / ((double)(n - m) * (double)(n + m));
        cplx yn = {(aa * ym1.re - r2 * ym2.re) * inv, (aa * ym1.im - r2 * ym2.im) * inv};
        Y[cidx(n, m)] = yn;
        ym2 = ym1;
        ym1 = yn;
      }
    }
    __syncwarp();
    // per pass: phi, dz, dzz (real); dp, dpz, dpp (complex) -> 9 doubles x 4
    double S[4][9];
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int v = 0; v < 9; v++) S[q][v] = 0.0;
    // iterate over (n, m) with m in [-n, n]: total (p+1)^2 terms
    int tot = (p + 1) * (p + 1);
    for (int idx = lane; idx < tot; idx += 32) {
      int n = (int)sqrt((double)idx);
      while (n * n > idx) n--;
      while ((n + 1) * (n + 1) <= idx) n++;
      int m = idx - n * n - n;
      cplx yc = cconj(hget(Y, n, m));
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const double* Lq = Ls + (size_t)q * D;
        auto Lg = [&](int nn, int mm) -> cplx {
          if (nn > p || mm > nn || -mm > nn) return cplx{0.0, 0.0};
          if (mm >= 0) return cplx{Lq[2 * cidx(nn, mm)], Lq[2 * cidx(nn, mm) + 1]};
          double re = Lq[2 * cidx(nn, -mm)], im = Lq[2 * cidx(nn, -mm) + 1];
          return ((-mm) & 1) ? cplx{-re, im} : cplx{re, -im};
        };
        cplx c0 = Lg(n, m);
        S[q][0] += c0.re * yc.re - c0.im * yc.im;
        if (n + 1 <= p) {
          cplx c1 = Lg(n + 1, m);
          S[q][1] += c1.re * yc.re - c1.im * yc.im;
          cplx c2 = Lg(n + 1, m + 1);  // D+ : -L_{n+1}^{m+1}
          S[q][3] -= c2.re * yc.re - c2.im * yc.im;
          S[q][4] -= c2.re * yc.im + c2.im * yc.re;
        }
        if (n + 2 <= p) {
          cplx c3 = Lg(n + 2, m);
          S[q][2] += c3.re * yc.re - c3.im * yc.im;
          cplx c4 = Lg(n + 2, m + 1);  // D+Dz : -L_{n+2}^{m+1}
          S[q][5] -= c4.re * yc.re - c4.im * yc.im;
          S[q][6] -= c4.re * yc.im + c4.im * yc.re;
          cplx c5 = Lg(n + 2, m + 2);  // D+D+ : L_{n+2}^{m+2}
          S[q][7] += c5.re * yc.re - c5.im * yc.im;
          S[q][8] += c5.re * yc.im + c5.im * yc.re;
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int v = 0; v < 9; v++) S[q][v] = warp_sum(S[q][v]);
    if (lane == 0) {
      double pot[4], g[4][3], H[4][3][3];
      for (int q = 0; q < 4; q++) {
        pot[q] = S[q][0];
        g[q][0] = S[q][3] * is;
        g[q][1] = S[q][4] * is;
        g[q][2] = S[q][1] * is;
        double hzz = S[q][2];
        double hxx = 0.5 * (S[q][7] - hzz), hyy = 0.5 * (-S[q][7] - hzz), hxy = 0.5 * S[q][8];
        double hxz = S[q][5], hyz = S[q][6];
        H[q][0][0] = hxx * is2; H[q][1][1] = hyy * is2; H[q][2][2] = hzz * is2;
        H[q][0][1] = H[q][1][0] = hxy * is2;
        H[q][0][2] = H[q][2][0] = hxz * is2;
        H[q][1][2] = H[q][2][1] = hyz * is2;
      }
      double c1 = a.c1;
      // u_a = (2-c1) phi_a - c1 x_j d_a phi_j + d_a Phi4
      double u[3];
      for (int i = 0; i < 3; i++) {
        u[i] = (2.0 - c1) * pot[i] + g[3][i];
        for (int j = 0; j < 3; j++) u[i] -= c1 * (x[j] - org[j]) * g[j][i];
      }
      const size_t np = is_src ? a.nsrc : a.ntgt;
      double* U = (is_src ? a.u_src : a.u_tgt) + 3 * np * blockIdx.y;
      double* E = (is_src ? a.e_src : a.e_tgt) + 6 * np * blockIdx.y;
      U[3 * (size_t)pidx] += u[0];
      U[3 * (size_t)pidx + 1] += u[1];
      U[3 * (size_t)pidx + 2] += u[2];
      bool dostrain = is_src ? a.dostrain_src : a.dostrain_tgt;
      if (dostrain) {
        // G_ab = d_b u_a = (2-c1) d_b phi_a - c1 d_a phi_b - c1 x_j d_ab phi_j + d_ab Phi4
        double G[3][3];
        for (int aa = 0; aa < 3; aa++)
          for (int bb = 0; bb < 3; bb++) {
            double v = (2.0 - c1) * g[aa][bb] - c1 * g[bb][aa] + H[3][aa][bb];
            for (int j = 0; j < 3; j++) v -= c1 * (x[j] - org[j]) * H[j][aa][bb];
            G[aa][bb] = v;
          }
        double* ee = E + 6 * (size_t)pidx;
        ee[0] += G[0][0];
        ee[1] += G[1][1];
        ee[2] += G[2][2];
        ee[3] += 0.5 * (G[0][1] + G[1][0]);
        ee[4] += 0.5 * (G[0][2] + G[2][0]);
        ee[5] += 0.5 * (G[1][2] + G[2][1]);
      }
    }
  }
}

// ----------------------------------------- L2T, many right-hand sides
// For C = 4R columns the nine derivative sums of a local expansion at a point
// are linear functionals of the stored real coefficient rows:
//   S[point, v][col] = sum over rows G_v[row](point) * L_box[row][col]
// (v: pot, d_z, d_zz, the D+ pair, the D+D_z pair, the D+D+ pair; the same
// sums as k_l2t, with the m < 0 terms folded onto the stored m >= 0 rows by
// conjugate symmetry).  One CTA per (leaf, chunk of 8 points, 256 columns):
// warp w owns point w, lane l the columns of right-hand sides l and l + 32;
// FP64 throughout (the local expansions may be FP32 in the normalised
// basis, converted while staged), then the Lame recombination of k_l2t.
constexpr int LG_PTS = 8, LG_K = 16, LG_C = 256, LG_CP = LG_C + 2;  // padded row: conflict-light staging

struct LgTerm {
  int a, b, sg, im;  // shift in n, shift in m, sign, imaginary part
};
__constant__ LgTerm c_lg_terms[9] = {{0, 0, 1, 0},  {1, 0, 1, 0},  {2, 0, 1, 0},
                                     {1, 1, -1, 0}, {1, 1, -1, 1}, {2, 1, -1, 0},
                                     {2, 1, -1, 1}, {2, 2, 1, 0},  {2, 2, 1, 1}};

template <class TB>
__global__ void __launch_bounds__(256, 1)
k_l2t_gemm(const L2TArgs a, const int* __restrict__ chunk_leaf, const int* __restrict__ chunk_e0, int R,
           const TB* __restrict__ local, const double* __restrict__ wnorm) {
  extern __shared__ __align__(16) unsigned char lg_smem[];
  const int p = a.p, nc = ncoef(p), D = 2 * nc, C = 4 * R;
  cplx* Ys = reinterpret_cast<cplx*>(lg_smem);                     // [LG_PTS][nc]
  double* Gs = reinterpret_cast<double*>(Ys + LG_PTS * nc);         // [LG_K][LG_PTS][9]
  double* Bs = Gs + LG_K * LG_PTS * 9;                              // [LG_K][LG_CP]
  const int box = a.leaves[chunk_leaf[blockIdx.x]];
  const int e0 = chunk_e0[blockIdx.x];
  const int col0 = blockIdx.y * LG_C;
  const int lev = a.level[box];
  const double s = a.size / (double)(1ull << lev), is = 1.0 / s, is2 = is * is;
  double c[3];
  for (int d = 0; d < 3; d++) c[d] = a.c0[d] - a.size / 2 + (a.ijk[3 * box + d] - 1) * s + s / 2;
  double org[3];
  lame_origin(a.ijk, a.level, box, a.c0, a.size, a.flev, org);
  const int sn = a.do_src ? a.scount[box] : 0, tn = a.do_tgt ? a.tcount[box] : 0;
  const int s0 = a.sstart[box], t0 = a.tstart[box];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // this warp's point
  const int e = e0 + warp;
  const bool ok = e < sn + tn;
  const bool is_src = e < sn;
  const int pidx = ok ? (is_src ? s0 + e : t0 + (e - sn)) : 0;
  double x[3] = {0, 0, 0};
  if (ok) {
    const double* X = is_src ? a.src_pts + 3 * (size_t)pidx : a.tgt_pts + 3 * (size_t)pidx;
    x[0] = X[0]; x[1] = X[1]; x[2] = X[2];
  }
  {
    cplx* Y = Ys + (size_t)warp * nc;
    const double z[3] = {(x[0] - c[0]) * is, (x[1] - c[1]) * is, (x[2] - c[2]) * is};
    const double r2 = z[0] * z[0] + z[1] * z[1] + z[2] * z[2];
    for (int m = lane; m <= p; m += 32) {
      cplx dm = {1.0, 0.0}, wv = {-0.5 * z[0], -0.5 * z[1]};
      for (int k = 1; k <= m; k++) dm = cscale(1.0 / k, cmul(dm, wv));
      Y[cidx(m, m)] = dm;
      cplx ym2 = {0, 0}, ym1 = dm;
      for (int n = m + 1; n <= p; n++) {
        const double aa = (2.0 * n - 1.0) * z[2];
        const double inv = 1.0 / ((double)(n - m) * (double)(n + m));
        cplx yn = {(aa * ym1.re - r2 * ym2.re) * inv, (aa * ym1.im - r2 * ym2.im) * inv};
        Y[cidx(n, m)] = yn;
        ym2 = ym1;
        ym1 = yn;
      }
    }
  }
  double acc[9][8];
#pragma unroll
  for (int v = 0; v < 9; v++)
#pragma unroll
    for (int j = 0; j < 8; j++) acc[v][j] = 0.0;
  const TB* Lb = local + (size_t)box * C * D;
  for (int k0 = 0; k0 < D; k0 += LG_K) {
    __syncthreads();
    // G tile: (k, point, v)
    for (int q = tid; q < LG_K * LG_PTS * 9; q += 256) {
      const int kk = q / (LG_PTS * 9), pt = (q / 9) % LG_PTS, v = q % 9;
      const int row = k0 + kk;
      double g = 0.0;
      if (row < D) {
        const int cc = row >> 1, part = row & 1;
        int N = 0;
        while ((N + 1) * (N + 2) / 2 <= cc) N++;
        const int M = cc - N * (N + 1) / 2;
        const LgTerm t = c_lg_terms[v];
        const int n = N - t.a;
        if (n >= 0) {
          const cplx* Y = Ys + (size_t)pt * nc;
          const double sM = (M & 1) ? -1.0 : 1.0;
          double yrd = 0, yid = 0, yrm = 0, yim = 0;
          const int md = M - t.b, mm = -M - t.b;
          if (md >= -n && md <= n) {
            cplx y = hget(Y, n, md);
            yrd = y.re; yid = y.im;
          }
          if (M > 0 && mm >= -n && mm <= n) {
            cplx y = hget(Y, n, mm);
            yrm = y.re; yim = y.im;
          }
          if (!t.im)
            g = part == 0 ? yrd + sM * yrm : yid - sM * yim;
          else
            g = part == 0 ? -yid - sM * yim : yrd - sM * yrm;
          g *= t.sg;
        }
      }
      Gs[q] = g;
    }
    // B tile: rows k0.., columns col0..; FP32 normalised rows are rescaled by w
    for (int q = tid; q < LG_K * LG_C; q += 256) {
      const int kk = q % LG_K, col = q / LG_K;
      const int row = k0 + kk, gcol = col0 + col;
      double b = 0.0;
      if (row < D && gcol < C) {
        b = (double)Lb[(size_t)gcol * D + row];
        if (wnorm) b *= wnorm[row];
      }
      Bs[kk * LG_CP + col] = b;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < LG_K; kk++) {
      double gv[9], bv[8];
#pragma unroll
      for (int v = 0; v < 9; v++) gv[v] = Gs[(kk * LG_PTS + warp) * 9 + v];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const double* br = Bs + kk * LG_CP + 128 * h + 4 * lane;
        const double2 u0 = *reinterpret_cast<const double2*>(br);
        const double2 u1 = *reinterpret_cast<const double2*>(br + 2);
        bv[4 * h] = u0.x; bv[4 * h + 1] = u0.y; bv[4 * h + 2] = u1.x; bv[4 * h + 3] = u1.y;
      }
#pragma unroll
      for (int v = 0; v < 9; v++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[v][j] += gv[v] * bv[j];
    }
  }
  if (!ok) return;
  const double c1 = a.c1;
  const bool dostrain = is_src ? a.dostrain_src : a.dostrain_tgt;
  const size_t np = is_src ? a.nsrc : a.ntgt;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int r = (col0 >> 2) + 32 * h + lane;
    if (r >= R) continue;
    double pot[4], g[4][3], H[4][3][3];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int j = 4 * h + q;
      pot[q] = acc[0][j];
      g[q][0] = acc[3][j] * is;
      g[q][1] = acc[4][j] * is;
      g[q][2] = acc[1][j] * is;
      const double hzz = acc[2][j];
      const double hxx = 0.5 * (acc[7][j] - hzz), hyy = 0.5 * (-acc[7][j] - hzz), hxy = 0.5 * acc[8][j];
      const double hxz = acc[5][j], hyz = acc[6][j];
      H[q][0][0] = hxx * is2; H[q][1][1] = hyy * is2; H[q][2][2] = hzz * is2;
      H[q][0][1] = H[q][1][0] = hxy * is2;
      H[q][0][2] = H[q][2][0] = hxz * is2;
      H[q][1][2] = H[q][2][1] = hyz * is2;
    }
    double u[3];
    for (int i = 0; i < 3; i++) {
      u[i] = (2.0 - c1) * pot[i] + g[3][i];
      for (int j = 0; j < 3; j++) u[i] -= c1 * (x[j] - org[j]) * g[j][i];
    }
    double* U = (is_src ? a.u_src : a.u_tgt) + 3 * (np * r + pidx);
    U[0] += u[0];
    U[1] += u[1];
    U[2] += u[2];
    if (dostrain) {
      double G[3][3];
      for (int aa = 0; aa < 3; aa++)
        for (int bb = 0; bb < 3; bb++) {
          double v = (2.0 - c1) * g[aa][bb] - c1 * g[bb][aa] + H[3][aa][bb];
          for (int j = 0; j < 3; j++) v -= c1 * (x[j] - org[j]) * H[j][aa][bb];
          G[aa][bb] = v;
        }
      double* E = (is_src ? a.e_src : a.e_tgt) + 6 * (np * r + pidx);
      E[0] += G[0][0];
      E[1] += G[1][1];
      E[2] += G[2][2];
      E[3] += 0.5 * (G[0][1] + G[1][0]);
      E[4] += 0.5 * (G[0][2] + G[2][0]);
      E[5] += 0.5 * (G[1][2] + G[2][1]);
    }
  }
}

// ------------------------------------------- L2T in two stages (product form)
// Stage 1 writes, per leaf, the functionals G[row][9 point + v] of the nine
// derivative sums (the same coefficients as k_l2t_gemm's G tile); stage 2 is
// the FP64 product S[col][9 point + v] = sum_row G[row][.] L[col][row]
// (k_gemm_tn); stage 3 applies the Lame recombination per (point, rhs).
// T = float: the functionals of the normalised basis (x wnorm), multiplied
// with the FP32 normalised local expansions on the tensor cores.
// snkt > 0 (T = float): G written as split tiles instead (rows 9 point + v
// in tiles of 128, coefficients in K tiles of 32, snkt of them; tile
// (mt, kt) at goff + (mt snkt + kt) 8192 floats, TF32 head then tail in the
// tensor cores' canonical layout; the product is k_tc_bulk).
template <class T>
__global__ void __launch_bounds__(256)
k_l2t_features(const L2TArgs a, const int* __restrict__ wleaves, const long long* __restrict__ goff,
               T* __restrict__ G, int snkt) {
  extern __shared__ __align__(16) unsigned char lf_smem[];
  const int p = a.p, nc = ncoef(p), D = 2 * nc;
  const int box = a.leaves[wleaves[blockIdx.x]];
  const int sn = a.do_src ? a.scount[box] : 0, tn = a.do_tgt ? a.tcount[box] : 0;
  const int P = sn + tn;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int e = blockIdx.y * 8 + warp;
  if (e >= P) return;
  const bool is_src = e < sn;
  const int pidx = is_src ? a.sstart[box] + e : a.tstart[box] + (e - sn);
  const double* X = is_src ? a.src_pts + 3 * (size_t)pidx : a.tgt_pts + 3 * (size_t)pidx;
  const int lev = a.level[box];
  const double s = a.size / (double)(1ull << lev), is = 1.0 / s;
  double c[3];
  for (int d = 0; d < 3; d++) c[d] = a.c0[d] - a.size / 2 + (a.ijk[3 * box + d] - 1) * s + s / 2;
  cplx* Y = reinterpret_cast<cplx*>(lf_smem) + (size_t)warp * nc;
  {
    const double z[3] = {(X[0] - c[0]) * is, (X[1] - c[1]) * is, (X[2] - c[2]) * is};
    const double r2 = z[0] * z[0] + z[1] * z[1] + z[2] * z[2];
    for (int m = lane; m <= p; m += 32) {
      cplx dm = {1.0, 0.0}, wv = {-0.5 * z[0], -0.5 * z[1]};
      for (int k = 1; k <= m; k++) dm = cscale(1.0 / k, cmul(dm, wv));
      Y[cidx(m, m)] = dm;
      cplx ym2 = {0, 0}, ym1 = dm;
      for (int n = m + 1; n <= p; n++) {
        const double aa = (2.0 * n - 1.0) * z[2];
        const double inv = 1.0 / ((double)(n - m) * (double)(n + m));
        cplx yn = {(aa * ym1.re - r2 * ym2.re) * inv, (aa * ym1.im - r2 * ym2.im) * inv};
        Y[cidx(n, m)] = yn;
        ym2 = ym1;
        ym1 = yn;
      }
    }
  }
  __syncwarp();
  T* out = G + goff[blockIdx.x] + 9 * (size_t)e;
  const size_t lda = (size_t)l2t_ld(P);
  for (int row = lane; row < D; row += 32) {
    const int cc = row >> 1, part = row & 1;
    int N = 0;
    while ((N + 1) * (N + 2) / 2 <= cc) N++;
    const int M = cc - N * (N + 1) / 2;
    const double sM = (M & 1) ? -1.0 : 1.0;
#pragma unroll
    for (int v = 0; v < 9; v++) {
      const LgTerm t = c_lg_terms[v];
      const int n = N - t.a;
      double g = 0.0;
      if (n >= 0) {
        double yrd = 0, yid = 0, yrm = 0, yim = 0;
        const int md = M - t.b, mm = -M - t.b;
        if (md >= -n && md <= n) {
          cplx y = hget(Y, n, md);
          yrd = y.re; yid = y.im;
        }
        if (M > 0 && mm >= -n && mm <= n) {
          cplx y = hget(Y, n, mm);
          yrm = y.re; yim = y.im;
        }
        if (!t.im)
          g = part == 0 ? yrd + sM * yrm : yid - sM * yim;
        else
          g = part == 0 ? -yid - sM * yim : yrd - sM * yrm;
        g *= t.sg;
      }
      const T val = (T)(a.wnorm ? g * a.wnorm[row] : g);
      if constexpr (sizeof(T) == 4) {
        if (snkt > 0) {
          const int m = 9 * e + v, kl = row & 31;
          float* tile = G + goff[blockIdx.x] + ((long long)(m >> 7) * snkt + (row >> 5)) * 8192;
          const int idx = (kl & 3) + 4 * (m & 7) + 32 * (kl >> 2) + 256 * ((m & 127) >> 3);
          const float h = tf32_head(val);
          tile[idx] = h;
          tile[4096 + idx] = val - h;
          continue;
        }
      }
      out[(size_t)row * lda + v] = val;
    }
  }
}

// The local expansions of each leaf of the wave as split B tiles of 128
// columns x 32 coefficients (8192 floats, TF32 head then tail, canonical
// layout; column tile ct, K tile kt at boff[i] + (ct nkt + kt) 8192): the C
// columns of the box (free space, C = 4R: local[(box C + col) D + k]; image,
// C = 7R: the 6R columns at local[(box 6R + col) D + k], then the R columns
// of U after all nb boxes' 6R columns).  CTAs (leaf, blockIdx.y) over the
// leaf's tiles: a tile is read column by column (128-byte runs) into shared
// memory (rows of 36 floats: neither phase has bank conflicts) and written
// in tile order, both coalesced; positions past C or D are written as zeros.
__global__ void __launch_bounds__(256)
k_l2t_local_split(const L2TArgs a, int R, int image, long long nb, const int* __restrict__ wleaves,
                  const long long* __restrict__ boff, const float* __restrict__ local, float* __restrict__ Bs) {
  __shared__ float sv[128][36];
  const int box = a.leaves[wleaves[blockIdx.x]];
  const int D = 2 * ncoef(a.p), nkt = (D + 31) / 32, C = image ? 7 * R : 4 * R, nct = (C + 127) / 128;
  float* o = Bs + boff[blockIdx.x];
  for (int tile = blockIdx.y; tile < nct * nkt; tile += gridDim.y) {
    const int ct = tile / nkt, kt = tile % nkt;
    __syncthreads();  // the previous tile's reads of sv are done
    for (int q = threadIdx.x; q < 4096; q += blockDim.x) {
      const int n = q >> 5, k = q & 31, col = 128 * ct + n, kk = 32 * kt + k;
      float v = 0.0f;
      if (col < C && kk < D) {
        const float* src;
        if (!image)
          src = local + ((long long)box * C + col) * D;
        else if (col < 6 * R)
          src = local + ((long long)box * 6 * R + col) * D;
        else
          src = local + nb * 6 * R * D + ((long long)box * R + (col - 6 * R)) * D;
        v = src[kk];
      }
      sv[n][k] = v;
    }
    __syncthreads();
    float* t = o + (long long)tile * 8192;
    for (int q = threadIdx.x; q < 4096; q += blockDim.x) {
      const int k = (q & 3) | (((q >> 5) & 7) << 2), n = ((q >> 2) & 7) | ((q >> 8) << 3);
      const float v = sv[n][k], h = tf32_head(v);
      t[q] = h;
      t[4096 + q] = v - h;
    }
  }
}

template <class TS>
__global__ void k_l2t_finish(const L2TArgs a, int R, const int* __restrict__ wleaves,
                             const long long* __restrict__ soff, const TS* __restrict__ S) {
  const int box = a.leaves[wleaves[blockIdx.x]];
  const int sn = a.do_src ? a.scount[box] : 0, tn = a.do_tgt ? a.tcount[box] : 0;
  const int P = sn + tn;
  const size_t ldc = (size_t)l2t_ld(P);
  const int lev = a.level[box];
  const double s = a.size / (double)(1ull << lev), is = 1.0 / s, is2 = is * is;
  const double c1 = a.c1;
  double org[3];
  lame_origin(a.ijk, a.level, box, a.c0, a.size, a.flev, org);
  for (int q = threadIdx.x; q < P * R; q += blockDim.x) {
    const int e = q % P, r = q / P;
    const bool is_src = e < sn;
    const int pidx = is_src ? a.sstart[box] + e : a.tstart[box] + (e - sn);
    const double* X = is_src ? a.src_pts + 3 * (size_t)pidx : a.tgt_pts + 3 * (size_t)pidx;
    const double x[3] = {X[0], X[1], X[2]};
    double pot[4], g[4][3], H[4][3][3];
    for (int pass = 0; pass < 4; pass++) {
      const TS* sv = S + soff[blockIdx.x] + (size_t)(4 * r + pass) * ldc + 9 * (size_t)e;
      pot[pass] = sv[0];
      g[pass][0] = sv[3] * is;
      g[pass][1] = sv[4] * is;
      g[pass][2] = sv[1] * is;
      const double hzz = sv[2];
      const double hxx = 0.5 * (sv[7] - hzz), hyy = 0.5 * (-sv[7] - hzz), hxy = 0.5 * sv[8];
      const double hxz = sv[5], hyz = sv[6];
      H[pass][0][0] = hxx * is2; H[pass][1][1] = hyy * is2; H[pass][2][2] = hzz * is2;
      H[pass][0][1] = H[pass][1][0] = hxy * is2;
      H[pass][0][2] = H[pass][2][0] = hxz * is2;
      H[pass][1][2] = H[pass][2][1] = hyz * is2;
    }
    const size_t np = is_src ? a.nsrc : a.ntgt;
    double u[3];
    for (int i = 0; i < 3; i++) {
      u[i] = (2.0 - c1) * pot[i] + g[3][i];
      for (int j = 0; j < 3; j++) u[i] -= c1 * (x[j] - org[j]) * g[j][i];
    }
    double* U = (is_src ? a.u_src : a.u_tgt) + 3 * (np * r + pidx);
    U[0] += u[0];
    U[1] += u[1];
    U[2] += u[2];
    const bool dostrain = is_src ? a.dostrain_src : a.dostrain_tgt;
    if (dostrain) {
      double Gm[3][3];
      for (int aa = 0; aa < 3; aa++)
        for (int bb = 0; bb < 3; bb++) {
          double v = (2.0 - c1) * g[aa][bb] - c1 * g[bb][aa] + H[3][aa][bb];
          for (int j = 0; j < 3; j++) v -= c1 * (x[j] - org[j]) * H[j][aa][bb];
          Gm[aa][bb] = v;
        }
      double* E = (is_src ? a.e_src : a.e_tgt) + 6 * (np * r + pidx);
      E[0] += Gm[0][0];
      E[1] += Gm[1][1];
      E[2] += Gm[2][2];
      E[3] += 0.5 * (Gm[0][1] + Gm[1][0]);
      E[4] += 0.5 * (Gm[0][2] + Gm[2][0]);
      E[5] += 0.5 * (Gm[1][2] + Gm[2][1]);
    }
  }
}

// Image displacement and strain at the original target from the value,
// gradient and Hessian of the 7 columns at the reflected target x (columns:
// 0..3 anti-image passes, 4 Phi_a, 5 Phi_c, 6 W; org the origin of
// lame_origin); ADDED to U (3) and, if E is set, E (6).
__device__ __forceinline__ void img_recombine(const double x[3], const double org[3], const double pot[7],
                                              const double g[7][3], const double H[7][3][3], double c1, double al,
                                              double imu, double sc,
                                              double* U, double* E) {
  const double x3 = -x[2];
  const double Pv[3] = {g[4][0], g[4][1], -g[4][2] - (2.0 - al) * pot[5]};
  double u[3], Gm[3][3];
  for (int i = 0; i < 3; i++) {
    u[i] = (2.0 - c1) * pot[i] + g[3][i];
    for (int j = 0; j < 3; j++) u[i] -= c1 * (x[j] - org[j]) * g[j][i];
    u[i] += sc * imu * g[6][i] + x3 * imu * Pv[i];
  }
  U[0] += u[0];
  U[1] += u[1];
  U[2] += u[2];
  if (!E) return;
  for (int aa = 0; aa < 3; aa++)
    for (int bb = 0; bb < 3; bb++) {
      double v = (2.0 - c1) * g[aa][bb] - c1 * g[bb][aa] + H[3][aa][bb];
      for (int j = 0; j < 3; j++) v -= c1 * (x[j] - org[j]) * H[j][aa][bb];
      v += sc * imu * H[6][aa][bb];
      const double dP = aa < 2 ? H[4][aa][bb] : -H[4][2][bb] - (2.0 - al) * g[5][bb];
      v += imu * ((bb == 2 ? -Pv[aa] : 0.0) + x3 * dP);
      Gm[aa][bb] = v;  // d u_a / d xb_b
    }
  // d u_a / d x_b = s_b Gm[a][b], s = (1, 1, -1)
  E[0] += Gm[0][0];
  E[1] += Gm[1][1];
  E[2] -= Gm[2][2];
  E[3] += 0.5 * (Gm[0][1] + Gm[1][0]);
  E[4] += 0.5 * (-Gm[0][2] + Gm[2][0]);
  E[5] += 0.5 * (-Gm[1][2] + Gm[2][1]);
}

// Direct image L2T (few right-hand sides): one CTA per (leaf, right-hand
// side r = blockIdx.y), the leaf's 7 local expansions in shared memory, a
// warp per target point (lanes over the (n, m) terms, warp-shuffle sums),
// then img_recombine.  local: columns kind * R + r of 6R per box, the U
// column at local + ubase + (box R + r) D.
__global__ void __launch_bounds__(L2T_WARPS * 32)
k_l2t_img(const L2TArgs a, int R, long long ubase) {
  extern __shared__ double lim_sm[];
  const int box = a.leaves[blockIdx.x];
  const int p = a.p, nc = ncoef(p), D = 2 * nc;
  const int r = blockIdx.y;
  double* Ls = lim_sm;                                            // [7][D]
  cplx* Yall = reinterpret_cast<cplx*>(lim_sm + 7 * (size_t)D);  // [warps][nc]
  for (int q = threadIdx.x; q < 7 * D; q += blockDim.x) {
    const int col = q / D, row = q % D;
    const double* L = col < 6 ? a.local + ((size_t)box * 6 * R + (size_t)col * R + r) * D
                              : a.local + ubase + ((size_t)box * R + r) * D;
    Ls[q] = L[row];
  }
  const int lev = a.level[box];
  const double s = a.size / (double)(1ull << lev), is = 1.0 / s, is2 = is * is;
  double c[3];
  for (int d = 0; d < 3; d++) c[d] = a.c0[d] - a.size / 2 + (a.ijk[3 * box + d] - 1) * s + s / 2;
  double org[3];
  lame_origin(a.ijk, a.level, box, a.c0, a.size, a.flev, org);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  cplx* Y = Yall + (size_t)warp * nc;
  const int tn = a.tcount[box], t0 = a.tstart[box];
  const double al = a.alpha, imu = 1.0 / a.mu, sc = (1.0 - al) / al;
  for (int e = warp; e < tn; e += nw) {
    const int pidx = t0 + e;
    const double* X = a.tgt_pts + 3 * (size_t)pidx;
    const double x[3] = {X[0], X[1], X[2]};
    const double z[3] = {(x[0] - c[0]) * is, (x[1] - c[1]) * is, (x[2] - c[2]) * is};
    __syncwarp();
    const double r2 = z[0] * z[0] + z[1] * z[1] + z[2] * z[2];
    for (int m = lane; m <= p; m += 32) {
      cplx dm = {1.0, 0.0}, wv = {-0.5 * z[0], -0.5 * z[1]};
      for (int k = 1; k <= m; k++) dm = cscale(1.0 / k, cmul(dm, wv));
      Y[cidx(m, m)] = dm;
      cplx ym2 = {0, 0}, ym1 = dm;
      for (int n = m + 1; n <= p; n++) {
        const double aa = (2.0 * n - 1.0) * z[2];
        const double inv = 1.0 / ((double)(n - m) * (double)(n + m));
        cplx yn = {(aa * ym1.re - r2 * ym2.re) * inv, (aa * ym1.im - r2 * ym2.im) * inv};
        Y[cidx(n, m)] = yn;
        ym2 = ym1;
        ym1 = yn;
      }
    }
    __syncwarp();
    double S[7][9];
#pragma unroll
    for (int q = 0; q < 7; q++)
#pragma unroll
      for (int v = 0; v < 9; v++) S[q][v] = 0.0;
    const int tot = (p + 1) * (p + 1);
    for (int idx = lane; idx < tot; idx += 32) {
      int n = (int)sqrt((double)idx);
      while (n * n > idx) n--;
      while ((n + 1) * (n + 1) <= idx) n++;
      const int m = idx - n * n - n;
      const cplx yc = cconj(hget(Y, n, m));
#pragma unroll
      for (int q = 0; q < 7; q++) {
        const double* Lq = Ls + (size_t)q * D;
        auto Lg = [&](int nn, int mm) -> cplx {
          if (nn > p || mm > nn || -mm > nn) return cplx{0.0, 0.0};
          if (mm >= 0) return cplx{Lq[2 * cidx(nn, mm)], Lq[2 * cidx(nn, mm) + 1]};
          const double re = Lq[2 * cidx(nn, -mm)], im = Lq[2 * cidx(nn, -mm) + 1];
          return ((-mm) & 1) ? cplx{-re, im} : cplx{re, -im};
        };
        const cplx c0 = Lg(n, m);
        S[q][0] += c0.re * yc.re - c0.im * yc.im;
        if (n + 1 <= p) {
          const cplx c1 = Lg(n + 1, m);
          S[q][1] += c1.re * yc.re - c1.im * yc.im;
          const cplx c2 = Lg(n + 1, m + 1);
          S[q][3] -= c2.re * yc.re - c2.im * yc.im;
          S[q][4] -= c2.re * yc.im + c2.im * yc.re;
        }
        if (n + 2 <= p) {
          const cplx c3 = Lg(n + 2, m);
          S[q][2] += c3.re * yc.re - c3.im * yc.im;
          const cplx c4 = Lg(n + 2, m + 1);
          S[q][5] -= c4.re * yc.re - c4.im * yc.im;
          S[q][6] -= c4.re * yc.im + c4.im * yc.re;
          const cplx c5 = Lg(n + 2, m + 2);
          S[q][7] += c5.re * yc.re - c5.im * yc.im;
          S[q][8] += c5.re * yc.im + c5.im * yc.re;
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 7; q++)
#pragma unroll
      for (int v = 0; v < 9; v++) S[q][v] = warp_sum(S[q][v]);
    if (lane == 0) {
      double pot[7], g[7][3], H[7][3][3];
      for (int q = 0; q < 7; q++) {
        pot[q] = S[q][0];
        g[q][0] = S[q][3] * is;
        g[q][1] = S[q][4] * is;
        g[q][2] = S[q][1] * is;
        const double hzz = S[q][2];
        const double hxx = 0.5 * (S[q][7] - hzz), hyy = 0.5 * (-S[q][7] - hzz), hxy = 0.5 * S[q][8];
        H[q][0][0] = hxx * is2; H[q][1][1] = hyy * is2; H[q][2][2] = hzz * is2;
        H[q][0][1] = H[q][1][0] = hxy * is2;
        H[q][0][2] = H[q][2][0] = S[q][5] * is2;
        H[q][1][2] = H[q][2][1] = S[q][6] * is2;
      }
      img_recombine(x, org, pot, g, H, a.c1, al, imu, sc, a.u_tgt + 3 * (a.ntgt * r + pidx),
                    a.dostrain_tgt ? a.e_tgt + 6 * (a.ntgt * r + pidx) : nullptr);
    }
  }
}

// Half-space image recombination at the reflected targets xb = (x1, x2, -x3)
// of the plan (columns as in k_p2m_weights_img, 7R per leaf in S).  In the
// variables xb, with alpha = (lam + mu)/(lam + 2 mu), sc = (1 - alpha)/alpha:
//   anti-image  u_A  = the free-space recombination with c1 = 2 - alpha
//   B piece     u_B  = (sc / mu) grad W
//   C piece     u_C  = (x3 / mu) P,  P = (d1 Phi_a, d2 Phi_a, -d3 Phi_a - (2 - alpha) Phi_c)
// and the strain of u(x) = u(xb(x)) uses d/dx_j = s_j d/dxb_j, s = (1, 1, -1).
template <class TS>
__global__ void k_l2t_finish_img(const L2TArgs a, int R, const int* __restrict__ wleaves,
                                 const long long* __restrict__ soff, const TS* __restrict__ S) {
  const int box = a.leaves[wleaves[blockIdx.x]];
  const int P = a.tcount[box];
  const size_t ldc = (size_t)l2t_ld(P);
  const int lev = a.level[box];
  const double s = a.size / (double)(1ull << lev), is = 1.0 / s, is2 = is * is;
  const double c1 = a.c1, al = a.alpha, imu = 1.0 / a.mu, sc = (1.0 - al) / al;
  double org[3];
  lame_origin(a.ijk, a.level, box, a.c0, a.size, a.flev, org);
  for (int q = threadIdx.x; q < P * R; q += blockDim.x) {
    const int e = q % P, r = q / P;
    const int pidx = a.tstart[box] + e;
    const double* X = a.tgt_pts + 3 * (size_t)pidx;
    const double x[3] = {X[0], X[1], X[2]};
    double pot[7], g[7][3], H[7][3][3];
    for (int cidx7 = 0; cidx7 < 7; cidx7++) {
      const int col = cidx7 * R + r;
      const TS* sv = S + soff[blockIdx.x] + (size_t)col * ldc + 9 * (size_t)e;
      pot[cidx7] = sv[0];
      g[cidx7][0] = sv[3] * is;
      g[cidx7][1] = sv[4] * is;
      g[cidx7][2] = sv[1] * is;
      const double hzz = sv[2];
      const double hxx = 0.5 * (sv[7] - hzz), hyy = 0.5 * (-sv[7] - hzz), hxy = 0.5 * sv[8];
      const double hxz = sv[5], hyz = sv[6];
      H[cidx7][0][0] = hxx * is2; H[cidx7][1][1] = hyy * is2; H[cidx7][2][2] = hzz * is2;
      H[cidx7][0][1] = H[cidx7][1][0] = hxy * is2;
      H[cidx7][0][2] = H[cidx7][2][0] = hxz * is2;
      H[cidx7][1][2] = H[cidx7][2][1] = hyz * is2;
    }
    img_recombine(x, org, pot, g, H, c1, al, imu, sc, a.u_tgt + 3 * (a.ntgt * r + pidx),
                  a.dostrain_tgt ? a.e_tgt + 6 * (a.ntgt * r + pidx) : nullptr);
  }
}

bool launch_l2t_img(cudaStream_t st, int nleaf, const L2TArgs& a, int R, long long ubase) {
  const size_t smem = sizeof(double) * 7 * 2 * (size_t)ncoef(a.p) + sizeof(cplx) * L2T_WARPS * ncoef(a.p);
  if (smem > 227 * 1024) return false;  // high orders: the two-stage form
  if (nleaf <= 0 || R <= 0) return true;
  EFMM_CUDA_TRY(smem_raise(k_l2t_img, (int)smem));
  k_l2t_img<<<dim3(nleaf, R), L2T_WARPS * 32, smem, st>>>(a, R, ubase);
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
  return true;
}

template <class T>
void launch_l2t_twostage(cudaStream_t st, const L2TArgs& a, int R, int nwleaf, const int* wleaves,
                         const long long* goff, const long long* soff, int max_pts, T* Gbuf, T* Sbuf,
                         int ntask, const GemmTask* tasks, const T* local, bool image, bool do_g) {
  if (nwleaf <= 0) return;
  const int nc = ncoef(a.p);
  const int smem = (int)(sizeof(cplx) * 8 * nc);
  if (do_g) {
    EFMM_CUDA_TRY(smem_raise(k_l2t_features<T>, (int)(smem)));
    k_l2t_features<T><<<dim3(nwleaf, (max_pts + 7) / 8), 256, smem, st>>>(a, wleaves, goff, Gbuf, 0);
    count_launch();
  }
  gemm_product<T>(st, ntask, tasks, Gbuf, local, Sbuf);
  if (image)
    k_l2t_finish_img<T><<<nwleaf, 256, 0, st>>>(a, R, wleaves, soff, Sbuf);
  else
    k_l2t_finish<T><<<nwleaf, 256, 0, st>>>(a, R, wleaves, soff, Sbuf);
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}
void launch_l2t_bulk(cudaStream_t st, const L2TArgs& a, int R, int nwleaf, const int* wleaves, const long long* goff,
                     const long long* soff, const long long* boff, int max_pts, float* scratch, int ntask,
                     const BulkTask* tasks, const float* local, long long nb, bool image, bool do_g, int* err) {
  if (nwleaf <= 0) return;
  const int nc = ncoef(a.p), nkt = (2 * nc + 31) / 32;
  const int smem = (int)(sizeof(cplx) * 8 * nc);
  if (do_g) {
    EFMM_CUDA_TRY(smem_raise(k_l2t_features<float>, (int)(smem)));
    k_l2t_features<float><<<dim3(nwleaf, (max_pts + 7) / 8), 256, smem, st>>>(a, wleaves, goff, scratch, nkt);
    count_launch();
  }
  k_l2t_local_split<<<dim3(nwleaf, 16), 256, 0, st>>>(a, R, image ? 1 : 0, nb, wleaves, boff, local, scratch);
  count_launch();
  launch_tc_bulk<float>(st, ntask, tasks, scratch, scratch, scratch, err, 128);
  if (image)
    k_l2t_finish_img<float><<<nwleaf, 256, 0, st>>>(a, R, wleaves, soff, scratch);
  else
    k_l2t_finish<float><<<nwleaf, 256, 0, st>>>(a, R, wleaves, soff, scratch);
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}

template void launch_l2t_twostage<double>(cudaStream_t, const L2TArgs&, int, int, const int*, const long long*,
                                          const long long*, int, double*, double*, int, const GemmTask*,
                                          const double*, bool, bool);
template void launch_l2t_twostage<float>(cudaStream_t, const L2TArgs&, int, int, const int*, const long long*,
                                         const long long*, int, float*, float*, int, const GemmTask*,
                                         const float*, bool, bool);

// Stage 1 of the factored P2M for one wave of leaves: unit-density
// multipoles H (nk = 4 or 7 kinds, per leaf at hoff: [kind][ns tn][D]) and
// the density operand S (per leaf at soff: R rows of ns tn rounded up to 4).
// FP32 (T = float) runs k_p2m_unit_f and needs the basis normalisation.
// False (nothing launched) when the order is too high for the kernel's
// shared memory.
template <class T>
bool launch_p2m_unit(cudaStream_t st, const P2MArgs& a, int R, int nk, int nwleaf, int maxtn, const int* wleaves,
                     const long long* hoff, const long long* soff, int sbase, int ns, T* H, T* S, bool do_h,
                     bool split) {
  const int nc = ncoef(a.p);
  const bool fp32 = sizeof(T) == 4;
  const size_t smem = p2m_unit_smem(a.p, fp32);
  if (smem > 227 * 1024 || (fp32 && !a.wnorm)) return false;
  if (nwleaf <= 0) return true;
  auto sigma = [&]() {
    if constexpr (sizeof(T) == 4) {
      if (split) {
        k_p2m_sigma_split<<<dim3(nwleaf, 8), 256, 0, st>>>(a, R, wleaves, soff, sbase, ns, S);
        return;
      }
    }
    k_p2m_sigma<T><<<dim3(nwleaf, 8), 256, 0, st>>>(a, R, wleaves, soff, sbase, ns, S);
  };
  if (!do_h) {
    sigma();
    count_launch();
    EFMM_CUDA_TRY(cudaGetLastError());
    return true;
  }
  const dim3 grid(nwleaf, (maxtn + UNIT_TB - 1) / UNIT_TB);
  // the fewest threads (whole warp quadruples) that cover the coefficients in ceil(nc / NT) rounds
  const int NT = fp32 ? UNITF_THREADS : unit_threads<T>();
  const int rounds = (nc + NT - 1) / NT;
  const int nthr = std::max(128, std::min(NT, (((nc + rounds - 1) / rounds) + 127) / 128 * 128));
  if constexpr (sizeof(T) == 4) {
    float* Hf = reinterpret_cast<float*>(H);
    if (nk == 7) {
      EFMM_CUDA_TRY(smem_raise(k_p2m_unit_f<7>, (int)smem));
      k_p2m_unit_f<7><<<grid, nthr, smem, st>>>(a, wleaves, hoff, sbase, ns, Hf, split ? 1 : 0);
    } else {
      EFMM_CUDA_TRY(smem_raise(k_p2m_unit_f<4>, (int)smem));
      k_p2m_unit_f<4><<<grid, nthr, smem, st>>>(a, wleaves, hoff, sbase, ns, Hf, split ? 1 : 0);
    }
  } else {
    constexpr int NTD = unit_threads<T>();
    if (nk == 7) {
      EFMM_CUDA_TRY(smem_raise(k_p2m_unit<T, 7, NTD>, (int)smem));
      k_p2m_unit<T, 7, NTD><<<grid, nthr, smem, st>>>(a, wleaves, hoff, sbase, ns, H);
    } else {
      EFMM_CUDA_TRY(smem_raise(k_p2m_unit<T, 4, NTD>, (int)smem));
      k_p2m_unit<T, 4, NTD><<<grid, nthr, smem, st>>>(a, wleaves, hoff, sbase, ns, H);
    }
  }
  count_launch();
  sigma();
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
  return true;
}
size_t p2m_unit_smem(int p, bool fp32) {
  if (fp32) return unitf_smem(p);
  const size_t nc = ncoef(p);
  return 12 * (size_t)unit_ylen(p) * sizeof(cplx) + nc * sizeof(double) + (nc + 1) * sizeof(int) +
         (18 + 12 * 4) * sizeof(double);
}
template bool launch_p2m_unit<double>(cudaStream_t, const P2MArgs&, int, int, int, int, const int*,
                                      const long long*, const long long*, int, int, double*, double*, bool, bool);
template bool launch_p2m_unit<float>(cudaStream_t, const P2MArgs&, int, int, int, int, const int*,
                                     const long long*, const long long*, int, int, float*, float*, bool, bool);

// The batched product of the two-stage P2M: FP32 on the tensor cores
// (tc_gemm.cu) unless ELFMM3D_TC=0, FP64 (and FP32 when disabled) on the
// CUDA cores.
template <class T>
void gemm_product(cudaStream_t st, int ntask, const GemmTask* tasks, const T* F, const T* W, T* C, int bn) {
  if (ntask <= 0) return;
  if (sizeof(T) == 4 && tc_enabled()) {
    launch_gemm_tc(st, ntask, tasks, reinterpret_cast<const float*>(F), reinterpret_cast<const float*>(W),
                   reinterpret_cast<float*>(C), tc_err_ptr(), bn);
    return;
  }
  const int gsm = (int)(sizeof(T) * 4 * 16 * 128);
  EFMM_CUDA_TRY(smem_raise(k_gemm_tn<T>, (int)(gsm)));
  k_gemm_tn<T><<<ntask, 256, gsm, st>>>(tasks, F, W, C);
  count_launch();
}

template void gemm_product<double>(cudaStream_t, int, const GemmTask*, const double*, const double*, double*, int);
template void gemm_product<float>(cudaStream_t, int, const GemmTask*, const float*, const float*, float*, int);

template <class T>
void launch_p2m_img_twostage(cudaStream_t st, const P2MArgs& a, int R, int nwleaf, const int* wleaves,
                             const long long* foff, const long long* woff, const long long* noff, double* nrec,
                             int max_nodes, T* F, T* W, int ntask, const GemmTask* tasks, T* mpole,
                             bool do_product) {
  if (nwleaf <= 0) return;
  const int nc = ncoef(a.p);
  const int smem = (int)(sizeof(cplx) * 8 * nc);
  EFMM_CUDA_TRY(smem_raise(k_p2m_features<T, 9>, (int)(smem)));
  k_p2m_features<T, 9><<<dim3(nwleaf, (max_nodes + 7) / 8), 256, smem, st>>>(a, wleaves, foff, noff, nrec, F);
  count_launch();
  k_p2m_weights_img<T><<<dim3(nwleaf, 16), 256, 0, st>>>(a, R, wleaves, woff, noff, nrec, W); count_launch();
  if (do_product) gemm_product<T>(st, ntask, tasks, F, W, mpole);
  EFMM_CUDA_TRY(cudaGetLastError());
}
template <class T>
void launch_p2m_img(cudaStream_t st, int nleaf, const P2MArgs& a, int R, long long ubase, T* mpole) {
  if (nleaf <= 0 || R <= 0) return;
  const size_t smem = sizeof(double) * (2 * (size_t)P2M_NODES * ncoef(a.p) + 63 * P2M_NODES);
  EFMM_CUDA_TRY(smem_raise(k_p2m_img<T>, (int)smem));
  k_p2m_img<T><<<dim3(nleaf, R), P2M_THREADS, smem, st>>>(a, R, ubase, mpole);
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}
template void launch_p2m_img<double>(cudaStream_t, int, const P2MArgs&, int, long long, double*);
template void launch_p2m_img<float>(cudaStream_t, int, const P2MArgs&, int, long long, float*);
template void launch_p2m_img_twostage<double>(cudaStream_t, const P2MArgs&, int, int, const int*,
                                              const long long*, const long long*, const long long*, double*, int,
                                              double*, double*, int, const GemmTask*, double*, bool);
template void launch_p2m_img_twostage<float>(cudaStream_t, const P2MArgs&, int, int, const int*,
                                             const long long*, const long long*, const long long*, double*, int,
                                             float*, float*, int, const GemmTask*, float*, bool);

// ---------------------------------------------------------------- launchers
void launch_build_ops(cudaStream_t st, int nop, const OpDesc* ops, double* mats, int maxp) {
  if (nop <= 0) return;
  size_t smem = sizeof(cplx) * (size_t)ncoef(2 * maxp);
  if (smem > 48 * 1024)
    EFMM_CUDA_TRY(smem_raise(k_build_ops, (int)smem));
  k_build_ops<<<nop, 256, smem, st>>>(nop, ops, mats); count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}

void launch_p2m(cudaStream_t st, int nleaf, const P2MArgs& a, int nrhs) {
  if (nleaf <= 0) return;
  size_t smem = sizeof(double) * (2 * (size_t)P2M_NODES * ncoef(a.p) + 16 * P2M_NODES);
  if (smem > 48 * 1024)
    EFMM_CUDA_TRY(smem_raise(k_p2m, (int)smem));
  k_p2m<<<dim3(nleaf, nrhs), P2M_THREADS, smem, st>>>(a); count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}

template <class T>
void launch_p2m_twostage(cudaStream_t st, const P2MArgs& a, int R, int nwleaf, const int* wleaves,
                         const long long* foff, const long long* woff, const long long* noff, double* nrec,
                         int max_nodes, T* F, T* W, int ntask, const GemmTask* tasks, T* mpole,
                         bool do_product) {
  if (nwleaf <= 0) return;
  const int nc = ncoef(a.p);
  const int smem = (int)(sizeof(cplx) * 8 * nc);
  EFMM_CUDA_TRY(smem_raise(k_p2m_features<T, 4>, (int)(smem)));
  k_p2m_features<T, 4><<<dim3(nwleaf, (max_nodes + 7) / 8), 256, smem, st>>>(a, wleaves, foff, noff, nrec, F);
  count_launch();
  k_p2m_weights<T><<<dim3(nwleaf, 16), 256, 0, st>>>(a, R, wleaves, woff, noff, nrec, W); count_launch();
  if (do_product) gemm_product<T>(st, ntask, tasks, F, W, mpole);
  EFMM_CUDA_TRY(cudaGetLastError());
}
template void launch_p2m_twostage<double>(cudaStream_t, const P2MArgs&, int, int, const int*, const long long*,
                                          const long long*, const long long*, double*, int, double*, double*, int,
                                          const GemmTask*, double*, bool);
template void launch_p2m_twostage<float>(cudaStream_t, const P2MArgs&, int, int, const int*, const long long*,
                                         const long long*, const long long*, double*, int, float*, float*, int,
                                         const GemmTask*, float*, bool);

template <class TB>
bool launch_l2t_gemm(cudaStream_t st, int nchunk, const int* chunk_leaf, const int* chunk_e0, const L2TArgs& a,
                     int R, const TB* local, const double* wnorm) {
  const int nc = ncoef(a.p);
  size_t smem = sizeof(cplx) * LG_PTS * nc + sizeof(double) * (LG_K * LG_PTS * 9 + LG_K * LG_CP);
  if (smem > 227 * 1024) return false;
  if (nchunk <= 0 || R <= 0) return true;
  EFMM_CUDA_TRY(smem_raise(k_l2t_gemm<TB>, (int)smem));
  dim3 grid(nchunk, (4 * R + LG_C - 1) / LG_C);
  k_l2t_gemm<TB><<<grid, 256, smem, st>>>(a, chunk_leaf, chunk_e0, R, local, wnorm); count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
  return true;
}
template bool launch_l2t_gemm<double>(cudaStream_t, int, const int*, const int*, const L2TArgs&, int,
                                      const double*, const double*);
template bool launch_l2t_gemm<float>(cudaStream_t, int, const int*, const int*, const L2TArgs&, int,
                                     const float*, const double*);

template <class T>
bool launch_p2m_gemm(cudaStream_t st, int nleaf, const P2MArgs& a, int R, T* mpole) {
  const int nc = ncoef(a.p), D = 2 * nc, C = 4 * R;
  size_t smem = sizeof(cplx) * PG_NODES * nc + sizeof(double) * PG_NODES * 8 + sizeof(int) * (PG_NODES + 2) +
                sizeof(T) * PG_K * (PG_R + PG_C);
  smem = (smem + 15) / 16 * 16;
  if (smem > 227 * 1024) return false;  // high orders: the caller uses k_p2m
  if (nleaf <= 0 || R <= 0) return true;
  EFMM_CUDA_TRY(smem_raise(k_p2m_gemm<T>, (int)smem));
  dim3 grid(nleaf, (D + PG_R - 1) / PG_R, (C + PG_C - 1) / PG_C);
  k_p2m_gemm<T><<<grid, 256, smem, st>>>(a, R, mpole); count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
  return true;
}
template bool launch_p2m_gemm<double>(cudaStream_t, int, const P2MArgs&, int, double*);
template bool launch_p2m_gemm<float>(cudaStream_t, int, const P2MArgs&, int, float*);

template <class T>
void launch_translate(cudaStream_t st, int ntask, const TransTask* tasks, const TransPair* pairs,
                      const T* mats, const long long* mat_off, const int* mat_dim, int D, int C,
                      const T* src, T* dst) {
  if (ntask <= 0) return;
  const int smem = (int)(sizeof(T) * 2 * TR_K * (TR_R + TR_C));
  static bool attr_set[64] = {};  // per T instantiation and device
  int dev = 0;
  EFMM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= 64 || !attr_set[dev]) {
    EFMM_CUDA_TRY(smem_raise(k_translate<T>, (int)(smem)));
    if (dev < 64) attr_set[dev] = true;
  }
  k_translate<T><<<ntask, 256, smem, st>>>(tasks, pairs, mats, mat_off, mat_dim, D, C, src, dst); count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}
template void launch_translate<double>(cudaStream_t, int, const TransTask*, const TransPair*, const double*,
                                       const long long*, const int*, int, int, const double*, double*);
template void launch_translate<float>(cudaStream_t, int, const TransTask*, const TransPair*, const float*,
                                      const long long*, const int*, int, int, const float*, float*);

void launch_l2t(cudaStream_t st, int nleaf, const L2TArgs& a, int nrhs) {
  if (nleaf <= 0) return;
  int nw = L2T_WARPS;
  auto need = [&](int w) {
    return sizeof(double) * 4 * 2 * (size_t)ncoef(a.p) + sizeof(cplx) * w * (size_t)ncoef(a.p);
  };
  while (nw > 1 && need(nw) > 220 * 1024) nw /= 2;
  size_t smem = need(nw);
  if (smem > 48 * 1024)
    EFMM_CUDA_TRY(smem_raise(k_l2t, (int)smem));
  k_l2t<<<dim3(nleaf, nrhs), nw * 32, smem, st>>>(a); count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}

}  // namespace efmm
