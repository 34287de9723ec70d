// halfspace.cu -- image part of the Mindlin half-space layer potentials.
//
// elhfmm3dtriatargiter (src/elhfmm3dtria_iter.f:46) returns, at targets in
// z < 0, the image part of the half-space single / double layer potentials
// of piecewise-constant densities on flat triangles (the direct arrival is
// the free-space evaluation, a separate call).  Here the image part is
// summed directly over all (target, triangle) pairs on the GPU: the
// integrand (mindlin_gen.cuh, generated by gen_mindlin.py) is smooth on the
// triangle except near the reflected target, so each pair is integrated with
// the 12-node degree-6 rule on sub-triangles refined by distance to the
// reflected target: a sub-triangle is accepted once the reflected target is
// more than HS_RATIO diameters away (rule error ~ (1 / (2 HS_RATIO))^7
// relative), and one still closer after HS_MAXDEPTH halvings (the pair is
// near-singular: a target close to the image of its triangle, as for faults
// that reach the surface) is integrated adaptively with error control, the
// scheme of the reference's tria3adam (src/tria3adamar.f:33-395): the rule
// on the sub-triangle against the sum over its four children, accepted when
// every output of each unit direction agrees to eps times that direction's
// largest, else the children are refined in turn, at most HS_ADAPT_DEPTH
// more halvings.  eps comes from iprec: min(1e-6 (the reference's
// tolerance, src/elhfmm3dtria_iter.f:2728), eps(iprec) / 10).
//
// This direct sum (O(N M) pair integrals) is the check of the image FMM
// (image.cu); the FMM's near field uses the same refined quadrature
// (k_hs_store).
#include "common.cuh"
#include "mindlin_gen.cuh"
#include "halfspace.h"

namespace efmm {

double iprec_eps(int iprec);  // plan.cu

// sub-triangle accepted for the 12-node rule when the reflected target is
// farther than HS_RATIO x its diameter (rule error ~ (1 / (2 HS_RATIO))^7)
constexpr double HS_RATIO = 8.0;
constexpr int HS_MAXDEPTH = 8;
constexpr int HS_STACK = 3 * HS_MAXDEPTH + 1;
constexpr int HS_TILE = 64;
constexpr int HS_ADAPT_DEPTH = 16;  // halvings of a near-singular sub-triangle (path codes of 2 bits each)
constexpr int HS_ASTACK = 3 * HS_ADAPT_DEPTH + 1;

double hs_quad_eps(int iprec) {
  const double e = iprec_eps(iprec);
  return e > 0.0 ? fmin(1e-6, 0.1 * e) : 1e-16;
}

// Adaptive integration of NOUT outputs (NG groups of NOUT / NG, each with its
// own relative tolerance) over the sub-triangle v0 (9 doubles); ev(y, w, out)
// adds w x the integrand at y into out.  acc += the integral; *ncap counts
// sub-triangles kept at the depth cap without meeting the tolerance.
template <int NOUT, int NG, class Ev>
__device__ __noinline__ void hs_adapt(const double* v0, double eps, const Quad12& Q, Ev ev, double* acc, int* ncap) {
  unsigned int code[HS_ASTACK];
  unsigned char dep[HS_ASTACK];
  int top = 1;
  code[0] = 0;
  dep[0] = 0;
  auto rule = [&](const double* a, const double* b, const double* c, double* out) {
    const double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    const double v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    const double cr[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
    const double area = 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    for (int q = 0; q < 12; q++) {
      double y[3];
      for (int d = 0; d < 3; d++) y[d] = Q.b[q][0] * a[d] + Q.b[q][1] * b[d] + Q.b[q][2] * c[d];
      ev(y, Q.w[q] * area, out);
    }
  };
  while (top > 0) {
    --top;
    const unsigned int cd = code[top];
    const int depth = dep[top];
    // the sub-triangle: descend from v0 along the path (2 bits per halving,
    // the first halving in the highest bits)
    double a[3], b[3], c[3];
    for (int d = 0; d < 3; d++) {
      a[d] = v0[d];
      b[d] = v0[3 + d];
      c[d] = v0[6 + d];
    }
    for (int l = depth - 1; l >= 0; l--) {
      const int k = (cd >> (2 * l)) & 3;
      double ab[3], bc[3], ca[3];
      for (int d = 0; d < 3; d++) {
        ab[d] = 0.5 * (a[d] + b[d]);
        bc[d] = 0.5 * (b[d] + c[d]);
        ca[d] = 0.5 * (c[d] + a[d]);
      }
      for (int d = 0; d < 3; d++) {
        if (k == 0) { b[d] = ab[d]; c[d] = ca[d]; }
        else if (k == 1) { a[d] = ab[d]; c[d] = bc[d]; }
        else if (k == 2) { a[d] = ca[d]; b[d] = bc[d]; }
        else { a[d] = ab[d]; b[d] = bc[d]; c[d] = ca[d]; }
      }
    }
    double ab[3], bc[3], ca[3];
    for (int d = 0; d < 3; d++) {
      ab[d] = 0.5 * (a[d] + b[d]);
      bc[d] = 0.5 * (b[d] + c[d]);
      ca[d] = 0.5 * (c[d] + a[d]);
    }
    double I[NOUT], S[NOUT];
    for (int k = 0; k < NOUT; k++) I[k] = S[k] = 0.0;
    rule(a, b, c, I);
    rule(a, ab, ca, S);
    rule(ab, b, bc, S);
    rule(ca, bc, c, S);
    rule(ab, bc, ca, S);
    bool ok = true;
    constexpr int GS = NOUT / NG;
    for (int g = 0; g < NG; g++) {
      double dmax = 0.0, dif = 0.0;
      for (int k = g * GS; k < (g + 1) * GS; k++) {
        dmax = fmax(dmax, fabs(I[k]));
        dif = fmax(dif, fabs(S[k] - I[k]));
      }
      ok = ok && dif <= eps * dmax;
    }
    if (ok || depth >= HS_ADAPT_DEPTH || top + 4 > HS_ASTACK) {
      for (int k = 0; k < NOUT; k++) acc[k] += S[k];
      if (!ok && ncap) atomicAdd(ncap, 1);
      continue;
    }
    for (int k = 3; k >= 0; k--) {
      code[top] = (cd << 2) | (unsigned int)k;
      dep[top] = (unsigned char)(depth + 1);
      top++;
    }
  }
}

struct HsSub {
  double v[9];
  int depth;
};

__global__ void k_hs_prep(int n, const double* __restrict__ tri, const double* __restrict__ nrm,
                          const double* __restrict__ ssl, const double* __restrict__ sdl, HsTri* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  HsTri t;
  for (int c = 0; c < 9; c++) t.v[c] = tri[9 * (size_t)i + c];
  for (int c = 0; c < 3; c++) {
    t.n[c] = nrm[3 * (size_t)i + c];
    t.sl[c] = ssl ? ssl[3 * (size_t)i + c] : 0.0;
    t.dl[c] = sdl ? sdl[3 * (size_t)i + c] : 0.0;
  }
  out[i] = t;
}

__device__ void hs_pair(const HsTri& T, const double X[3], int dosl, int dodl, double lam, double mu,
                        const Quad12& Q, double eps, int* ncap, double acc[9]) {
  const double Xr[3] = {X[0], X[1], -X[2]};
  HsSub stk[HS_STACK];
  int top = 0;
  for (int c = 0; c < 9; c++) stk[0].v[c] = T.v[c];
  stk[0].depth = 0;
  top = 1;
  while (top > 0) {
    const HsSub s = stk[--top];
    const double* a = s.v;
    const double* b = s.v + 3;
    const double* c = s.v + 6;
    double cen[3], diam = 0.0;
    for (int d = 0; d < 3; d++) cen[d] = (a[d] + b[d] + c[d]) / 3.0;
    {
      double e0 = 0, e1 = 0, e2 = 0;
      for (int d = 0; d < 3; d++) {
        e0 += (b[d] - a[d]) * (b[d] - a[d]);
        e1 += (c[d] - b[d]) * (c[d] - b[d]);
        e2 += (a[d] - c[d]) * (a[d] - c[d]);
      }
      diam = sqrt(fmax(e0, fmax(e1, e2)));
    }
    double dist2 = 0;
    for (int d = 0; d < 3; d++) dist2 += (Xr[d] - cen[d]) * (Xr[d] - cen[d]);
    const bool far = dist2 > HS_RATIO * HS_RATIO * diam * diam;
    if (!far && (s.depth >= HS_MAXDEPTH || top + 4 > HS_STACK)) {
      // near-singular: adaptive with error control
      hs_adapt<9, 1>(s.v, eps, Q,
                     [&](const double* y, double w, double* out) {
                       double o[9];
                       if (dosl) {
                         mindlin_image_sl(lam, mu, X[0], X[1], X[2], y[0], y[1], y[2], T.sl[0], T.sl[1], T.sl[2],
                                          o);
                         for (int k = 0; k < 9; k++) out[k] += w * o[k];
                       }
                       if (dodl) {
                         mindlin_image_dl(lam, mu, X[0], X[1], X[2], y[0], y[1], y[2], T.dl[0], T.dl[1], T.dl[2],
                                          T.n[0], T.n[1], T.n[2], o);
                         for (int k = 0; k < 9; k++) out[k] += w * o[k];
                       }
                     },
                     acc, ncap);
    } else if (far) {
      const double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
      const double v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
      const double cr[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
      const double area = 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
      for (int q = 0; q < 12; q++) {
        double y[3];
        for (int d = 0; d < 3; d++) y[d] = Q.b[q][0] * a[d] + Q.b[q][1] * b[d] + Q.b[q][2] * c[d];
        const double w = Q.w[q] * area;
        double o[9];
        if (dosl) {
          mindlin_image_sl(lam, mu, X[0], X[1], X[2], y[0], y[1], y[2], T.sl[0], T.sl[1], T.sl[2], o);
          for (int k = 0; k < 9; k++) acc[k] += w * o[k];
        }
        if (dodl) {
          mindlin_image_dl(lam, mu, X[0], X[1], X[2], y[0], y[1], y[2], T.dl[0], T.dl[1], T.dl[2], T.n[0],
                           T.n[1], T.n[2], o);
          for (int k = 0; k < 9; k++) acc[k] += w * o[k];
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
      for (int k = 0; k < 4; k++) {
        HsSub t;
        for (int vtx = 0; vtx < 3; vtx++)
          for (int d = 0; d < 3; d++) t.v[3 * vtx + d] = kids[k][vtx][d];
        t.depth = s.depth + 1;
        stk[top++] = t;
      }
    }
  }
}

// One thread per target and chunk of HS_CHUNK triangles (grid.y), the
// triangles streamed through shared memory; partial sums are added to the
// zeroed outputs.
constexpr int HS_CHUNK = 512;

__global__ void __launch_bounds__(128, 1)  // one CTA: let the generated kernel keep 255 registers
k_hs_image(int n, const HsTri* __restrict__ tris, int m, const double* __restrict__ tgt, int dosl, int dodl,
           double lam, double mu, double eps, int* __restrict__ ncap, double* __restrict__ u,
           double* __restrict__ e6) {
  __shared__ HsTri tile[HS_TILE];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = i < m;
  double X[3] = {0, 0, 0};
  if (ok)
    for (int d = 0; d < 3; d++) X[d] = tgt[3 * (size_t)i + d];
  Quad12 Q;
  quad12(Q);
  double acc[9];
  for (int k = 0; k < 9; k++) acc[k] = 0.0;
  const int c0 = blockIdx.y * HS_CHUNK, c1 = min(n, c0 + HS_CHUNK);
  for (int t0 = c0; t0 < c1; t0 += HS_TILE) {
    const int cnt = min(HS_TILE, c1 - t0);
    __syncthreads();
    for (int q = threadIdx.x; q < cnt; q += blockDim.x) tile[q] = tris[t0 + q];
    __syncthreads();
    if (ok)
      for (int t = 0; t < cnt; t++) hs_pair(tile[t], X, dosl, dodl, lam, mu, Q, eps, ncap, acc);
  }
  if (!ok) return;
  for (int d = 0; d < 3; d++) atomicAdd(u + 3 * (size_t)i + d, acc[d]);
  for (int d = 0; d < 6; d++) atomicAdd(e6 + 6 * (size_t)i + d, acc[3 + d]);
}

// Unit-density blocks of one (target, triangle) pair with the refinement of
// hs_pair: acc[0..26] single layer (unit force e_k at 9k), acc[27..53]
// double layer (unit jump e_p at 27 + 9p); displacement then strain.
__device__ void hs_pair_blk(const double* tv, const double nrm[3], const double X[3], int dosl, int dodl,
                            double lam, double mu, const Quad12& Q, double eps, int* ncap, double* acc) {
  const double Xr[3] = {X[0], X[1], -X[2]};
  HsSub stk[HS_STACK];
  for (int c = 0; c < 9; c++) stk[0].v[c] = tv[c];
  stk[0].depth = 0;
  int top = 1;
  while (top > 0) {
    const HsSub s = stk[--top];
    const double* a = s.v;
    const double* b = s.v + 3;
    const double* c = s.v + 6;
    double cen[3], diam;
    for (int d = 0; d < 3; d++) cen[d] = (a[d] + b[d] + c[d]) / 3.0;
    {
      double e0 = 0, e1 = 0, e2 = 0;
      for (int d = 0; d < 3; d++) {
        e0 += (b[d] - a[d]) * (b[d] - a[d]);
        e1 += (c[d] - b[d]) * (c[d] - b[d]);
        e2 += (a[d] - c[d]) * (a[d] - c[d]);
      }
      diam = sqrt(fmax(e0, fmax(e1, e2)));
    }
    double dist2 = 0;
    for (int d = 0; d < 3; d++) dist2 += (Xr[d] - cen[d]) * (Xr[d] - cen[d]);
    const bool far = dist2 > HS_RATIO * HS_RATIO * diam * diam;
    if (!far && (s.depth >= HS_MAXDEPTH || top + 4 > HS_STACK)) {
      // near-singular: each layer adaptively with error control per unit direction
      if (dosl)
        hs_adapt<27, 3>(s.v, eps, Q,
                        [&](const double* y, double w, double* out) {
                          double o[27];
                          mindlin_image_sl_blk(lam, mu, X[0], X[1], X[2], y[0], y[1], y[2], o);
                          for (int k = 0; k < 27; k++) out[k] += w * o[k];
                        },
                        acc, ncap);
      if (dodl)
        hs_adapt<27, 3>(s.v, eps, Q,
                        [&](const double* y, double w, double* out) {
                          double o[27];
                          mindlin_image_dl_blk(lam, mu, X[0], X[1], X[2], y[0], y[1], y[2], nrm[0], nrm[1], nrm[2],
                                               o);
                          for (int k = 0; k < 27; k++) out[k] += w * o[k];
                        },
                        acc + 27, ncap);
    } else if (far) {
      const double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
      const double v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
      const double cr[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
      const double area = 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
      for (int q = 0; q < 12; q++) {
        double y[3];
        for (int d = 0; d < 3; d++) y[d] = Q.b[q][0] * a[d] + Q.b[q][1] * b[d] + Q.b[q][2] * c[d];
        const double w = Q.w[q] * area;
        double o[27];
        if (dosl) {
          mindlin_image_sl_blk(lam, mu, X[0], X[1], X[2], y[0], y[1], y[2], o);
          for (int k = 0; k < 27; k++) acc[k] += w * o[k];
        }
        if (dodl) {
          mindlin_image_dl_blk(lam, mu, X[0], X[1], X[2], y[0], y[1], y[2], nrm[0], nrm[1], nrm[2], o);
          for (int k = 0; k < 27; k++) acc[27 + k] += w * o[k];
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
      for (int k = 0; k < 4; k++) {
        HsSub t;
        for (int vtx = 0; vtx < 3; vtx++)
          for (int d = 0; d < 3; d++) t.v[3 * vtx + d] = kids[k][vtx][d];
        t.depth = s.depth + 1;
        stk[top++] = t;
      }
    }
  }
}

constexpr int HSS_PTS = 8;  // targets per CTA (the batched near-field chunks)

__global__ void __launch_bounds__(128, 1)
k_hs_store(const HsStoreArgs a, const int* __restrict__ chunk_leaf, const int* __restrict__ chunk_e0,
           double* __restrict__ store) {
  const int li = chunk_leaf[blockIdx.x], e0 = chunk_e0[blockIdx.x];
  const int leaf = a.leaves[li];
  const int tn = a.box_tgt_count[leaf], t0 = a.box_tgt_start[leaf];
  const int ne = min(HSS_PTS, tn - e0);
  const int nt = a.ntri[li];
  double* out = store + a.base[li];
  Quad12 Q;
  quad12(Q);
  for (int q = threadIdx.x; q < ne * nt; q += blockDim.x) {
    const int e = e0 + q / nt, t = q % nt;
    // triangle of near position t: the concatenated ranges of the paired boxes
    int tri = -1, pos = 0;
    for (int b = a.nb_start[li]; b < a.nb_start[li + 1]; b++) {
      const int sb = a.nb_items[b], cnt = a.box_src_count[sb];
      if (t < pos + cnt) {
        tri = a.box_src_start[sb] + (t - pos);
        break;
      }
      pos += cnt;
    }
    if (tri < 0) continue;
    const double* xb = a.tgt + 3 * (size_t)(t0 + e);
    const double X[3] = {xb[0], xb[1], -xb[2]};
    double acc[54];
    for (int k = 0; k < 54; k++) acc[k] = 0.0;
    if (a.points) {  // a particle: the kernel blocks at the point
      const double* y = a.pts + 3 * (size_t)tri;
      const double* nv = a.nrm + 3 * (size_t)tri;
      if (a.dosl) mindlin_image_sl_blk(a.lam, a.mu, X[0], X[1], X[2], y[0], y[1], y[2], acc);
      if (a.dodl) mindlin_image_dl_blk(a.lam, a.mu, X[0], X[1], X[2], y[0], y[1], y[2], nv[0], nv[1], nv[2], acc + 27);
    } else {
      hs_pair_blk(a.tri + 9 * (size_t)tri, a.nrm + 3 * (size_t)tri, X, a.dosl, a.dodl, a.lam, a.mu, Q, a.eps,
                  a.ncap, acc);
    }
    double* o = out + ((size_t)e * nt + t) * a.K;
    int w = 0;
    for (int layer = 0; layer < 2; layer++) {
      if ((layer == 0 && !a.dosl) || (layer == 1 && !a.dodl)) continue;
      for (int c = 0; c < 3; c++) {
        const double* blk = acc + 27 * layer + 9 * c;
        o[w] = blk[0]; o[w + 1] = blk[1]; o[w + 2] = blk[2];
        w += 3;
        if (a.dstr) {
          for (int k = 0; k < 6; k++) o[w + k] = blk[3 + k];
          w += 6;
        }
      }
    }
  }
}

// per-device counter of sub-triangles kept at the adaptive depth cap
namespace {
__device__ int g_hs_ncap;
int* g_hs_ncap_addr[64] = {};
}  // namespace

int* hs_ncap_ptr() {
  int dev = 0;
  EFMM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw CudaError{(int)cudaErrorInvalidDevice};
  if (!g_hs_ncap_addr[dev]) {
    void* p = nullptr;
    EFMM_CUDA_TRY(cudaGetSymbolAddress(&p, g_hs_ncap));
    g_hs_ncap_addr[dev] = static_cast<int*>(p);
  }
  return g_hs_ncap_addr[dev];
}

int hs_take_ncap() {
  int* p = hs_ncap_ptr();
  int h = 0;
  EFMM_CUDA_TRY(cudaMemcpy(&h, p, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) EFMM_CUDA_TRY(cudaMemset(p, 0, sizeof(int)));
  return h;
}

void launch_hs_store(cudaStream_t st, const HsStoreArgs& a, int nchunk, const int* chunk_leaf,
                     const int* chunk_e0, double* store) {
  if (nchunk <= 0) return;
  k_hs_store<<<nchunk, 128, 0, st>>>(a, chunk_leaf, chunk_e0, store);
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}

// The half-space particle direct sum of the image part: one thread per
// target, all points (the reference's elh3dpartdirecttarg image terms).
__global__ void __launch_bounds__(128, 1)
k_part_image(int n, const double* __restrict__ src, const double* __restrict__ sl, const double* __restrict__ dl,
             const double* __restrict__ nu, int m, const double* __restrict__ tgt, double lam, double mu,
             double* __restrict__ u, double* __restrict__ e6) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const double X[3] = {tgt[3 * (size_t)i], tgt[3 * (size_t)i + 1], tgt[3 * (size_t)i + 2]};
  double acc[9];
  for (int k = 0; k < 9; k++) acc[k] = 0.0;
  for (int j = 0; j < n; j++) {
    const double* y = src + 3 * (size_t)j;
    double o[9];
    if (sl) {
      mindlin_image_sl(lam, mu, X[0], X[1], X[2], y[0], y[1], y[2], sl[3 * (size_t)j], sl[3 * (size_t)j + 1],
                       sl[3 * (size_t)j + 2], o);
      for (int k = 0; k < 9; k++) acc[k] += o[k];
    }
    if (dl) {
      const double* nv = nu + 3 * (size_t)j;
      mindlin_image_dl(lam, mu, X[0], X[1], X[2], y[0], y[1], y[2], dl[3 * (size_t)j], dl[3 * (size_t)j + 1],
                       dl[3 * (size_t)j + 2], nv[0], nv[1], nv[2], o);
      for (int k = 0; k < 9; k++) acc[k] += o[k];
    }
  }
  for (int d = 0; d < 3; d++) u[3 * (size_t)i + d] = acc[d];
  for (int d = 0; d < 6; d++) e6[6 * (size_t)i + d] = acc[3 + d];
}

void launch_part_image(cudaStream_t st, int n, const double* src, const double* sl, const double* dl,
                       const double* nu, int m, const double* tgt, double lam, double mu, double* u, double* e6) {
  if (n <= 0 || m <= 0) return;
  k_part_image<<<(m + 127) / 128, 128, 0, st>>>(n, src, sl, dl, nu, m, tgt, lam, mu, u, e6);
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}

void launch_hs_image(cudaStream_t st, int n, const double* tri, const double* nrm, const double* ssl,
                     const double* sdl, int m, const double* tgt, double lam, double mu, double eps, int* ncap,
                     HsTri* work, double* u, double* e6) {
  if (n <= 0 || m <= 0) return;
  k_hs_prep<<<(n + 127) / 128, 128, 0, st>>>(n, tri, nrm, ssl, sdl, work); count_launch();
  EFMM_CUDA_TRY(cudaMemsetAsync(u, 0, 3 * sizeof(double) * (size_t)m, st));
  EFMM_CUDA_TRY(cudaMemsetAsync(e6, 0, 6 * sizeof(double) * (size_t)m, st));
  dim3 grid((m + 127) / 128, (n + HS_CHUNK - 1) / HS_CHUNK);
  k_hs_image<<<grid, 128, 0, st>>>(n, work, m, tgt, ssl != nullptr, sdl != nullptr, lam, mu, eps, ncap, u, e6);
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}

}  // namespace efmm
