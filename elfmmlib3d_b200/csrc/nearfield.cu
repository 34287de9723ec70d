// nearfield.cu -- analytic near-field kernels (FP64).
//
// The near field of the reference (src/elfmm3dtria.f:968 _evalloc and the
// ITER variant src/elfmm3dtria_iter_1.f:1240-1419) sums, for each evaluation
// point, the exact single/double layer potential of every triangle in the
// source boxes paired with the point's leaf box.  Here one CTA owns one leaf
// box: the paired triangles stream through shared memory in tiles, each warp
// takes one evaluation point against a tile (lanes split the triangles), and
// the per-point partial sums are reduced with warp shuffles into shared-memory
// accumulators that are written once at the end.
#include "common.cuh"
#include "kernels.h"
#include "tc_common.cuh"

namespace efmm {

// Build the per-triangle frame records in tree order and rotate the densities
// into each triangle frame.
__global__ void k_tri_prep(int n, const double* __restrict__ tri, const int* __restrict__ perm,
                           const double* __restrict__ ssl, const double* __restrict__ sdl,
                           int dosl, int dodl, TriRec* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int j = perm ? perm[i] : i;
  double t[9];
#pragma unroll
  for (int c = 0; c < 9; c++) t[c] = tri[9 * (size_t)j + c];
  TriRec r;
  tri_frame(t, r.f);
  double a[3] = {0, 0, 0}, b[3] = {0, 0, 0};
  if (dosl) { a[0] = ssl[3 * (size_t)j]; a[1] = ssl[3 * (size_t)j + 1]; a[2] = ssl[3 * (size_t)j + 2]; }
  if (dodl) { b[0] = sdl[3 * (size_t)j]; b[1] = sdl[3 * (size_t)j + 1]; b[2] = sdl[3 * (size_t)j + 2]; }
  const double* ax[3] = {r.f.e1, r.f.e2, r.f.e3};
#pragma unroll
  for (int c = 0; c < 3; c++) {
    r.ssl[c] = ax[c][0] * a[0] + ax[c][1] * a[1] + ax[c][2] * a[2];
    r.sdl[c] = ax[c][0] * b[0] + ax[c][1] * b[1] + ax[c][2] * b[2];
  }
  r.pad[0] = r.pad[1] = 0.0;
  out[i] = r;
}

constexpr int NF_TILE = 64;    // triangles staged per tile
constexpr int NF_WARPS = 4;    // warps per CTA
constexpr int NF_MAXEP = 512;  // max evaluation points per leaf held in shared memory
#ifndef NF_MINB
#define NF_MINB 2               // resident CTAs per SM the register budget targets
#endif

__device__ __forceinline__ void stage_tile(TriRec* sm, const TriRec* __restrict__ g, int cnt) {
  const double2* src = reinterpret_cast<const double2*>(g);
  double2* dst = reinterpret_cast<double2*>(sm);
  int nv = cnt * (int)(sizeof(TriRec) / sizeof(double2));
  for (int q = threadIdx.x; q < nv; q += blockDim.x) dst[q] = src[q];
}

// One CTA per leaf box.  Evaluation points of the leaf: its sources (sorted
// centroids, self-aware) then its targets.  nb_start/nb_items: CSR of the
// source boxes paired with the leaf; box_src_start/count give their triangle
// ranges.  Outputs are ADDED to u (3/pt) and e (6/pt, xx yy zz xy xz yz).
__global__ void __launch_bounds__(NF_WARPS * 32, NF_MINB)
k_near_leaf(int nleaf, const int* __restrict__ leaves, const int* __restrict__ nb_start,
            const int* __restrict__ nb_items, const int* __restrict__ box_src_start,
            const int* __restrict__ box_src_count, const int* __restrict__ box_tgt_start,
            const int* __restrict__ box_tgt_count, const TriRec* __restrict__ trir,
            const double* __restrict__ src_pts, const double* __restrict__ tgt_pts, int dosl,
            int dodl, int dostrain_src, int dostrain_tgt, int do_src, int do_tgt, double rlam,
            double rmu, double* __restrict__ u_src, double* __restrict__ e_src,
            double* __restrict__ u_tgt, double* __restrict__ e_tgt) {
  __shared__ TriRec tile[NF_TILE];
  __shared__ double acc[NF_MAXEP][9];
  int leaf = leaves[blockIdx.x];
  int s0 = box_src_start[leaf], sn = do_src ? box_src_count[leaf] : 0;
  int t0 = box_tgt_start[leaf], tn = do_tgt ? box_tgt_count[leaf] : 0;
  int nep = sn + tn;
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // process evaluation points in chunks of NF_MAXEP
  for (int ep0 = 0; ep0 < nep; ep0 += NF_MAXEP) {
    int nepc = min(NF_MAXEP, nep - ep0);
    for (int q = threadIdx.x; q < nepc * 9; q += blockDim.x) (&acc[0][0])[q] = 0.0;
    __syncthreads();
    for (int b = nb_start[blockIdx.x]; b < nb_start[blockIdx.x + 1]; b++) {
      int sb = nb_items[b];
      int tr0 = box_src_start[sb], trn = box_src_count[sb];
      for (int k0 = 0; k0 < trn; k0 += NF_TILE) {
        int cnt = min(NF_TILE, trn - k0);
        __syncthreads();
        stage_tile(tile, trir + tr0 + k0, cnt);
        __syncthreads();
        for (int e = warp; e < nepc; e += NF_WARPS) {
          int ep = ep0 + e;
          bool is_src = ep < sn;
          int pidx = is_src ? s0 + ep : t0 + (ep - sn);
          const double* P = is_src ? src_pts + 3 * (size_t)pidx : tgt_pts + 3 * (size_t)pidx;
          double X[3] = {P[0], P[1], P[2]};
          bool dostrain = is_src ? dostrain_src : dostrain_tgt;
          double u[3] = {0, 0, 0}, ee[6] = {0, 0, 0, 0, 0, 0};
          for (int k = lane; k < cnt; k += 32) {
            int tidx = tr0 + k0 + k;
            bool self = is_src && (tidx == pidx);
            const TriRec& r = tile[k];
            pair_eval(r.f, r.ssl, r.sdl, dosl, dodl, dostrain, X, self, rlam, rmu, u, ee);
          }
#pragma unroll
          for (int c = 0; c < 3; c++) u[c] = warp_sum(u[c]);
          if (dostrain) {
#pragma unroll
            for (int c = 0; c < 6; c++) ee[c] = warp_sum(ee[c]);
          }
          if (lane == 0) {
            acc[e][0] += u[0]; acc[e][1] += u[1]; acc[e][2] += u[2];
            if (dostrain)
              for (int c = 0; c < 6; c++) acc[e][3 + c] += ee[c];
          }
        }
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nepc; e += blockDim.x) {
      int ep = ep0 + e;
      bool is_src = ep < sn;
      int pidx = is_src ? s0 + ep : t0 + (ep - sn);
      double* U = is_src ? u_src : u_tgt;
      double* E = is_src ? e_src : e_tgt;
      U[3 * (size_t)pidx] += acc[e][0];
      U[3 * (size_t)pidx + 1] += acc[e][1];
      U[3 * (size_t)pidx + 2] += acc[e][2];
      bool dostrain = is_src ? dostrain_src : dostrain_tgt;
      if (dostrain)
        for (int c = 0; c < 6; c++) E[6 * (size_t)pidx + c] += acc[e][3 + c];
    }
    __syncthreads();
  }
}

// All-pairs direct sum (el3dtriadirecttarg, src/elfmm3dtria.f:1483): one warp
// per evaluation point, all triangles streamed through shared memory.
// Points [0, nsrc) are the centroids (self pair when the indices match),
// [nsrc, nsrc+ntgt) the targets.  Outputs are overwritten.
__global__ void __launch_bounds__(NF_WARPS * 32, NF_MINB)
k_direct_all(int ntri, const TriRec* __restrict__ trir, int nsrc, const double* __restrict__ src_pts,
             int ntgt, const double* __restrict__ tgt_pts, int dosl, int dodl, int dostrain_src,
             int dostrain_tgt, double rlam, double rmu, double* __restrict__ u_src,
             double* __restrict__ e_src, double* __restrict__ u_tgt, double* __restrict__ e_tgt) {
  __shared__ TriRec tile[NF_TILE];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int ep = blockIdx.x * NF_WARPS + warp;
  int nep = nsrc + ntgt;
  bool active = ep < nep;
  bool is_src = ep < nsrc;
  int pidx = is_src ? ep : ep - nsrc;
  double X[3] = {0, 0, 0};
  if (active) {
    const double* P = is_src ? src_pts + 3 * (size_t)pidx : tgt_pts + 3 * (size_t)pidx;
    X[0] = P[0]; X[1] = P[1]; X[2] = P[2];
  }
  bool dostrain = is_src ? dostrain_src : dostrain_tgt;
  double u[3] = {0, 0, 0}, ee[6] = {0, 0, 0, 0, 0, 0};
  for (int k0 = 0; k0 < ntri; k0 += NF_TILE) {
    int cnt = min(NF_TILE, ntri - k0);
    __syncthreads();
    stage_tile(tile, trir + k0, cnt);
    __syncthreads();
    if (active) {
      for (int k = lane; k < cnt; k += 32) {
        bool self = is_src && (k0 + k == pidx);
        const TriRec& r = tile[k];
        pair_eval(r.f, r.ssl, r.sdl, dosl, dodl, dostrain, X, self, rlam, rmu, u, ee);
      }
    }
  }
  if (!active) return;
#pragma unroll
  for (int c = 0; c < 3; c++) u[c] = warp_sum(u[c]);
#pragma unroll
  for (int c = 0; c < 6; c++) ee[c] = warp_sum(ee[c]);
  if (lane == 0) {
    double* U = is_src ? u_src : u_tgt;
    double* E = is_src ? e_src : e_tgt;
    U[3 * (size_t)pidx] = u[0];
    U[3 * (size_t)pidx + 1] = u[1];
    U[3 * (size_t)pidx + 2] = u[2];
    if (dostrain)
      for (int c = 0; c < 6; c++) E[6 * (size_t)pidx + c] = ee[c];
  }
}

// ITER mode, first call: compute and store the unit-density response blocks
// of every near (point, triangle) pair of each leaf.  Layout per leaf:
// [evaluation point][near triangle][K doubles], at base[leaf]; near triangles
// are the concatenated source ranges of the leaf's paired boxes.
__global__ void __launch_bounds__(NF_WARPS * 32, NF_MINB)
k_near_store(const NearArgs a, const long long* __restrict__ base, const int* __restrict__ ntri,
             int K, int dodisp, double* __restrict__ store) {
  __shared__ TriRec tile[NF_TILE];
  int leaf = a.leaves[blockIdx.x];
  int s0 = a.box_src_start[leaf], sn = a.do_src ? a.box_src_count[leaf] : 0;
  int t0 = a.box_tgt_start[leaf], tn = a.do_tgt ? a.box_tgt_count[leaf] : 0;
  int nep = sn + tn;
  int nt = ntri[blockIdx.x];
  double* out = store + base[blockIdx.x];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int pos = 0;  // running index of the leaf's near triangles
  for (int b = a.nb_start[blockIdx.x]; b < a.nb_start[blockIdx.x + 1]; b++) {
    int sb = a.nb_items[b];
    int tr0 = a.box_src_start[sb], trn = a.box_src_count[sb];
    for (int k0 = 0; k0 < trn; k0 += NF_TILE) {
      int cnt = min(NF_TILE, trn - k0);
      __syncthreads();
      stage_tile(tile, a.trir + tr0 + k0, cnt);
      __syncthreads();
      for (int e = warp; e < nep; e += NF_WARPS) {
        bool is_src = e < sn;
        int pidx = is_src ? s0 + e : t0 + (e - sn);
        const double* P = is_src ? a.src_pts + 3 * (size_t)pidx : a.tgt_pts + 3 * (size_t)pidx;
        double X[3] = {P[0], P[1], P[2]};
        bool dostrain = is_src ? a.dostrain_src : a.dostrain_tgt;
        for (int k = lane; k < cnt; k += 32) {
          int tidx = tr0 + k0 + k;
          bool self = is_src && (tidx == pidx);
          double blk[54];
          pair_blocks(tile[k].f, a.dosl, a.dodl, dodisp, dostrain, X, self, a.rlam, a.rmu, blk);
          double* o = out + ((size_t)e * nt + (pos + k0 + k)) * K;
          for (int q = 0; q < K; q++) o[q] = blk[q];
        }
      }
    }
    pos += trn;
  }
}

// ITER mode, later calls: replay the stored blocks against new densities
// (tree order, global frame) and ADD to the outputs.  One CTA per leaf, one
// warp per evaluation point, lanes over the point's near triangles so each
// warp reads one contiguous row of blocks.
__global__ void __launch_bounds__(256)
k_near_replay(const NearArgs a, const long long* __restrict__ base, const int* __restrict__ ntri,
              int K, int dodisp, const double* __restrict__ ssl, const double* __restrict__ sdl,
              const double* __restrict__ store) {
  int leaf = a.leaves[blockIdx.x];
  int s0 = a.box_src_start[leaf], sn = a.do_src ? a.box_src_count[leaf] : 0;
  int t0 = a.box_tgt_start[leaf], tn = a.do_tgt ? a.box_tgt_count[leaf] : 0;
  int nep = sn + tn;
  int nt = ntri[blockIdx.x];
  const double* blocks = store + base[blockIdx.x];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int e = warp; e < nep; e += nw) {
    bool is_src = e < sn;
    int pidx = is_src ? s0 + e : t0 + (e - sn);
    bool dostrain = is_src ? a.dostrain_src : a.dostrain_tgt;
    double u[3] = {0, 0, 0}, ee[6] = {0, 0, 0, 0, 0, 0};
    const double* row = blocks + (size_t)e * nt * K;
    int pos = 0;
    for (int b = a.nb_start[blockIdx.x]; b < a.nb_start[blockIdx.x + 1]; b++) {
      int sb = a.nb_items[b];
      int tr0 = a.box_src_start[sb], trn = a.box_src_count[sb];
      for (int k = lane; k < trn; k += 32) {
        int t = tr0 + k;
        const double* B = row + (size_t)(pos + k) * K;
        int w = 0;
        for (int layer = 0; layer < 2; layer++) {
          if ((layer == 0 && !a.dosl) || (layer == 1 && !a.dodl)) continue;
          const double* sg = (layer == 0 ? ssl : sdl) + 3 * (size_t)t;
          double sv[3] = {sg[0], sg[1], sg[2]};
          for (int c = 0; c < 3; c++) {
            if (dodisp) {
              u[0] += B[w] * sv[c]; u[1] += B[w + 1] * sv[c]; u[2] += B[w + 2] * sv[c];
              w += 3;
            }
            if (dostrain) {
              for (int q = 0; q < 6; q++) ee[q] += B[w + q] * sv[c];
              w += 6;
            }
          }
        }
      }
      pos += trn;
    }
#pragma unroll
    for (int c = 0; c < 3; c++) u[c] = warp_sum(u[c]);
#pragma unroll
    for (int c = 0; c < 6; c++) ee[c] = warp_sum(ee[c]);
    if (lane == 0) {
      double* U = is_src ? a.u_src : a.u_tgt;
      double* E = is_src ? a.e_src : a.e_tgt;
      if (dodisp)
        for (int c = 0; c < 3; c++) U[3 * (size_t)pidx + c] += u[c];
      if (dostrain)
        for (int c = 0; c < 6; c++) E[6 * (size_t)pidx + c] += ee[c];
    }
  }
}

// Many right-hand sides at once (densities tree order, right-hand side
// innermost: sigma[(tri * 3 + component) * R + r]).  The pair response to unit densities
// (pair_blocks, as stored by the ITER mode) does not depend on the densities,
// so it is computed once per (point, triangle) pair and contracted with all
// R right-hand sides: per tile of NB_PTS points x NB_TRI triangles, phase 1
// writes the pair blocks to shared memory (one pair per thread), phase 2 is a
// small dense product  out[point][9][R] += block[point][tri][9 x 6] *
// sigma[tri][6][R]  with the outputs held in registers (9 x RB per thread;
// R <= 16 RB).  One CTA per (near leaf, chunk of NB_PTS evaluation points).
constexpr int NB_PTS = 8, NB_TRI = 16, NB_THREADS = NB_PTS * NB_TRI;

// REPLAY: the pair blocks are read from the stored near field (k_near_store
// layout: per leaf at base[leaf], [point][near triangle][K]) instead of
// computed -- the ITER store applied to many right-hand sides at once.
template <int RB, bool REPLAY>
__global__ void __launch_bounds__(NB_THREADS)
k_near_batch(const NearArgs a, const int* __restrict__ chunk_leaf, const int* __restrict__ chunk_e0,
             int R, int K, int dostrain, const double* __restrict__ ssl, const double* __restrict__ sdl,
             int ntri_all, int nsrc, int ntgt, const long long* __restrict__ sbase, const int* __restrict__ sntri,
             const double* __restrict__ store) {
  constexpr int RW = 16 * RB;  // right-hand sides held per tile
  __shared__ TriRec tile[NB_TRI];
  extern __shared__ __align__(16) double nb_sm[];
  double* Bk = nb_sm;                            // [NB_PTS][NB_TRI][K]
  double* Sg = Bk + NB_PTS * NB_TRI * K;         // [NB_TRI][6][RW]
  const int li = chunk_leaf[blockIdx.x], e0 = chunk_e0[blockIdx.x];
  const int leaf = a.leaves[li];
  const int s0 = a.box_src_start[leaf], sn = a.do_src ? a.box_src_count[leaf] : 0;
  const int t0 = a.box_tgt_start[leaf], tn = a.do_tgt ? a.box_tgt_count[leaf] : 0;
  const int nep = sn + tn;
  const int tid = threadIdx.x;
  const int pp = tid / NB_TRI, tt = tid % NB_TRI;  // phase 1: (point, triangle)
  const int rr = tid % 16, pq = tid / 16;          // phase 2: (point, rhs lane)
  // phase-1 point
  const int e1 = e0 + pp;
  const bool ok1 = e1 < nep;
  const bool src1 = e1 < sn;
  const int pid1 = ok1 ? (src1 ? s0 + e1 : t0 + (e1 - sn)) : 0;
  double X[3] = {0, 0, 0};
  if (ok1) {
    const double* P = src1 ? a.src_pts + 3 * (size_t)pid1 : a.tgt_pts + 3 * (size_t)pid1;
    X[0] = P[0]; X[1] = P[1]; X[2] = P[2];
  }
  double acc[9][RB];
#pragma unroll
  for (int c = 0; c < 9; c++)
#pragma unroll
    for (int k = 0; k < RB; k++) acc[c][k] = 0.0;
  const int nl = a.dosl + a.dodl;
  int pos = 0;  // running index of the leaf's near triangles (store layout)
  for (int b = a.nb_start[li]; b < a.nb_start[li + 1]; b++) {
    const int sb = a.nb_items[b];
    const int tr0 = a.box_src_start[sb], trn = a.box_src_count[sb];
    for (int k0 = 0; k0 < trn; k0 += NB_TRI) {
      const int cnt = min(NB_TRI, trn - k0);
      __syncthreads();
      if (!REPLAY) stage_tile(tile, a.trir + tr0 + k0, cnt);
      for (int q = tid; q < NB_TRI * 6 * RW; q += NB_THREADS) {
        int t = q / (6 * RW), j = (q / RW) % 6, r = q % RW;
        int layer = j / 3, d = j % 3;
        double v = 0.0;
        if (t < cnt && r < R && (layer == 0 ? a.dosl : a.dodl)) {
          const double* sg = layer == 0 ? ssl : sdl;
          v = sg[((size_t)(tr0 + k0 + t) * 3 + d) * R + r];
        }
        Sg[q] = v;
      }
      __syncthreads();
      if (REPLAY) {
        // the tile's blocks of the chunk's points: contiguous K-runs per point
        const int nt = sntri[li];
        const double* src = store + sbase[li];
        for (int q = tid; q < NB_PTS * NB_TRI * K; q += NB_THREADS) {
          const int pt = q / (NB_TRI * K), rem = q % (NB_TRI * K), t = rem / K, c = rem % K;
          const int e = e0 + pt;
          double v = 0.0;
          if (e < nep && t < cnt) v = src[((size_t)e * nt + (pos + k0 + t)) * K + c];
          Bk[q] = v;
        }
      } else {
        double* o = Bk + (pp * NB_TRI + tt) * K;
        if (ok1 && tt < cnt) {
          const int tidx = tr0 + k0 + tt;
          pair_blocks(tile[tt].f, a.dosl, a.dodl, true, dostrain, X, src1 && tidx == pid1, a.rlam, a.rmu, o);
        } else {
          for (int q = 0; q < K; q++) o[q] = 0.0;
        }
      }
      __syncthreads();
      for (int t = 0; t < cnt; t++) {
        const double* Bt = Bk + (pq * NB_TRI + t) * K;
        int w = 0;
        for (int j = 0; j < 6; j++) {
          if ((j < 3 && !a.dosl) || (j >= 3 && !a.dodl)) continue;
          double sv[RB];
#pragma unroll
          for (int k = 0; k < RB; k++) sv[k] = Sg[(t * 6 + j) * RW + rr + 16 * k];
#pragma unroll
          for (int c = 0; c < 3; c++)
#pragma unroll
            for (int k = 0; k < RB; k++) acc[c][k] += Bt[w + c] * sv[k];
          w += 3;
          if (dostrain) {
#pragma unroll
            for (int c = 0; c < 6; c++)
#pragma unroll
              for (int k = 0; k < RB; k++) acc[3 + c][k] += Bt[w + c] * sv[k];
            w += 6;
          }
        }
      }
    }
    pos += trn;
  }
  (void)nl;
  const int e2 = e0 + pq;
  if (e2 >= nep) return;
  const bool src2 = e2 < sn;
  const int pid2 = src2 ? s0 + e2 : t0 + (e2 - sn);
  const size_t np = src2 ? (size_t)nsrc : (size_t)ntgt;
  const bool ds2 = src2 ? a.dostrain_src : a.dostrain_tgt;
#pragma unroll
  for (int k = 0; k < RB; k++) {
    const int r = rr + 16 * k;
    if (r >= R) continue;
    double* U = (src2 ? a.u_src : a.u_tgt) + 3 * (np * r + pid2);
#pragma unroll
    for (int c = 0; c < 3; c++) U[c] += acc[c][k];
    if (ds2) {
      double* E = (src2 ? a.e_src : a.e_tgt) + 6 * (np * r + pid2);
#pragma unroll
      for (int c = 0; c < 6; c++) E[c] += acc[3 + c][k];
    }
  }
}

// Batched replay of the stored near field, specialised on the layer count
// NLAY (1: one layer, 2: both) and strain STR: compile-time block size
// K = 3 NLAY (3 + 6 STR), only the enabled layers' densities staged, every
// inner loop unrolled.  Same tiling as k_near_batch (CTA per 8 points of a
// leaf, 16 triangles per tile, 9 x RB outputs per thread).
template <int RB, int NLAY, int STR>
__global__ void __launch_bounds__(NB_THREADS)
k_near_replay_batch(const NearArgs a, const int* __restrict__ chunk_leaf, const int* __restrict__ chunk_e0, int R,
                    const double* __restrict__ sg0, const double* __restrict__ sg1, int nsrc, int ntgt,
                    const long long* __restrict__ sbase, const int* __restrict__ sntri,
                    const double* __restrict__ store) {
  constexpr int RW = 16 * RB, NJ = 3 * NLAY, KB = 3 + 6 * STR, K = NJ * KB;
  extern __shared__ __align__(16) double rb_sm[];
  double* Bk = rb_sm;                     // [NB_PTS][NB_TRI][K]
  double* Sg = Bk + NB_PTS * NB_TRI * K;  // [NB_TRI][NJ][RW]
  const int li = chunk_leaf[blockIdx.x], e0 = chunk_e0[blockIdx.x];
  const int leaf = a.leaves[li];
  const int s0 = a.box_src_start[leaf], sn = a.do_src ? a.box_src_count[leaf] : 0;
  const int t0 = a.box_tgt_start[leaf], tn = a.do_tgt ? a.box_tgt_count[leaf] : 0;
  const int nep = sn + tn;
  const int tid = threadIdx.x;
  const int rr = tid % 16, pq = tid / 16;
  const int nt = sntri[li];
  const double* src = store + sbase[li];
  double acc[KB][RB];
#pragma unroll
  for (int c = 0; c < KB; c++)
#pragma unroll
    for (int k = 0; k < RB; k++) acc[c][k] = 0.0;
  int pos = 0;
  for (int b = a.nb_start[li]; b < a.nb_start[li + 1]; b++) {
    const int sb = a.nb_items[b];
    const int tr0 = a.box_src_start[sb], trn = a.box_src_count[sb];
    for (int k0 = 0; k0 < trn; k0 += NB_TRI) {
      const int cnt = min(NB_TRI, trn - k0);
      __syncthreads();
      for (int q = tid; q < NB_TRI * NJ * RW; q += NB_THREADS) {
        const int t = q / (NJ * RW), j = (q / RW) % NJ, r = q % RW;
        const double* sg = (NLAY == 2 && j >= 3) ? sg1 : sg0;
        double v = 0.0;
        if (t < cnt && r < R) v = sg[((size_t)(tr0 + k0 + t) * 3 + (j % 3)) * R + r];
        Sg[q] = v;
      }
      for (int q = tid; q < NB_PTS * NB_TRI * K; q += NB_THREADS) {
        const int pt = q / (NB_TRI * K), rem = q % (NB_TRI * K), t = rem / K, c = rem % K;
        const int e = e0 + pt;
        double v = 0.0;
        if (e < nep && t < cnt) v = src[((size_t)e * nt + (pos + k0 + t)) * K + c];
        Bk[q] = v;
      }
      __syncthreads();
      const double* Bp = Bk + pq * NB_TRI * K;
#pragma unroll 2
      for (int t = 0; t < cnt; t++) {
        const double* Bt = Bp + t * K;
#pragma unroll
        for (int j = 0; j < NJ; j++) {
          double sv[RB];
#pragma unroll
          for (int k = 0; k < RB; k++) sv[k] = Sg[(t * NJ + j) * RW + rr + 16 * k];
#pragma unroll
          for (int c = 0; c < KB; c++) {
            const double bv = Bt[j * KB + c];
#pragma unroll
            for (int k = 0; k < RB; k++) acc[c][k] += bv * sv[k];
          }
        }
      }
    }
    pos += trn;
  }
  const int e2 = e0 + pq;
  if (e2 >= nep) return;
  const bool src2 = e2 < sn;
  const int pid2 = src2 ? s0 + e2 : t0 + (e2 - sn);
  const size_t np = src2 ? (size_t)nsrc : (size_t)ntgt;
  const bool ds2 = src2 ? a.dostrain_src : a.dostrain_tgt;
#pragma unroll
  for (int k = 0; k < RB; k++) {
    const int r = rr + 16 * k;
    if (r >= R) continue;
    double* U = (src2 ? a.u_src : a.u_tgt) + 3 * (np * r + pid2);
#pragma unroll
    for (int c = 0; c < 3; c++) U[c] += acc[c][k];
    if (STR && ds2) {
      double* E = (src2 ? a.e_src : a.e_tgt) + 6 * (np * r + pid2);
#pragma unroll
      for (int c = 0; c < 6; c++) E[c] += acc[3 + c][k];
    }
  }
}

// ------------------------------------- stored near field on the tensor cores
// Mixed-precision replay of the ITER store as one dense product per leaf:
// out[row][r] = sum_k A[k][row] S[r][k] with k = NJ t + j (near triangle t,
// density component j of the NJ = 3 x layers stored) and row = KB e + c
// (evaluation point e, output c of KB = 3 (+ 6 strain)).  A is the FP64
// store converted once to FP32 in this layout (same per-leaf offsets, lda =
// KB x points); S the leaf's near densities gathered per right-hand side;
// the product runs on the tensor cores (gemm_product<float>) and the
// results are added to the FP64 outputs.

// Position of the leaf's own triangles in its near list (-1 if absent):
// the self pairs (source point e, near triangle self + e) are applied in
// FP64 from the FP64 store (k_near_self64), not through the FP32 copy.
__device__ __forceinline__ int near_self_pos(const NearArgs& a, int i, int leaf) {
  int pos = 0;
  for (int b = a.nb_start[i]; b < a.nb_start[i + 1]; b++) {
    const int sb = a.nb_items[b];
    if (sb == leaf) return pos;
    pos += a.box_src_count[sb];
  }
  return -1;
}

// FP64 store [point][near triangle][K] -> FP32 [NJ t + j][KB e + c], per leaf
// at fbase[i] with rows of ceil4(KB x points) floats (padding zero; self
// pairs zero).
__global__ void __launch_bounds__(256)
k_near_store_tc(const NearArgs a, const long long* __restrict__ base, const long long* __restrict__ fbase,
                const int* __restrict__ ntri, int K, int KB, const double* __restrict__ store,
                float* __restrict__ out) {
  const int i = blockIdx.x, leaf = a.leaves[i];
  const int sn = a.do_src ? a.box_src_count[leaf] : 0;
  const int nep = sn + (a.do_tgt ? a.box_tgt_count[leaf] : 0);
  const long long nt = ntri[i], M = (long long)KB * nep, Mp = (M + 3) & ~3LL, NJ = K / KB, tot = nep * nt * K;
  const int self = near_self_pos(a, i, leaf);
  const double* src = store + base[i];
  float* dst = out + fbase[i];
  for (long long q = blockIdx.y * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.y * blockDim.x) {
    const long long e = q / (nt * K), rem = q % (nt * K), t = rem / K, jc = rem % K;
    const long long j = jc / KB, c = jc % KB;
    const bool is_self = e < sn && self >= 0 && t == self + e;
    dst[(t * NJ + j) * Mp + e * KB + c] = is_self ? 0.0f : (float)src[q];
  }
  // the padding of each row
  const long long pad = Mp - M, rows = nt * NJ;
  for (long long q = blockIdx.y * (long long)blockDim.x + threadIdx.x; q < rows * pad;
       q += (long long)gridDim.y * blockDim.x)
    dst[(q / pad) * Mp + M + q % pad] = 0.0f;
}

// FP64 store [point][near triangle][K] -> tiles of the pre-split store: per
// leaf at tbase[i], tile (mt, kt) at (mt nkt + kt) 8192 floats holding rows
// 128 mt.. (KB e + c) and k 32 kt.. (NJ t + j) of A, the TF32 head of each
// element then its tail, in the canonical K-major layout (element (row, k)
// at (k % 4) + 4 (row % 8) + 32 (k / 4) + 256 (row / 8)); zero past M and K
// and at the self pairs (applied in FP64).  CTAs (leaf, blockIdx.y) over the
// leaf's tiles; the stores are coalesced, the loads gather from runs of the
// pair blocks.
__global__ void __launch_bounds__(256)
k_near_split_store(const NearArgs a, const long long* __restrict__ base, const long long* __restrict__ tbase,
                   const int* __restrict__ ntri, int K, int KB, const double* __restrict__ store,
                   float* __restrict__ out) {
  const int i = blockIdx.x, leaf = a.leaves[i];
  const int sn = a.do_src ? a.box_src_count[leaf] : 0;
  const int nep = sn + (a.do_tgt ? a.box_tgt_count[leaf] : 0);
  const long long nt = ntri[i], NJ = K / KB, M = (long long)KB * nep, KK = NJ * nt;
  const long long nmt = (M + 127) / 128, nkt = (KK + 31) / 32;
  const int self = near_self_pos(a, i, leaf);
  const double* src = store + base[i];
  float* dst = out + tbase[i];
  for (long long tile = blockIdx.y; tile < nmt * nkt; tile += gridDim.y) {
    const long long mt = tile / nkt, kt = tile % nkt;
    float* o = dst + tile * 8192;
    for (int q = threadIdx.x; q < 4096; q += blockDim.x) {
      const int k = (q & 3) | (((q >> 5) & 7) << 2), m = ((q >> 2) & 7) | ((q >> 8) << 3);
      const long long row = 128 * mt + m, kk = 32 * kt + k;
      float v = 0.0f;
      if (row < M && kk < KK) {
        const long long e = row / KB, c = row % KB, t = kk / NJ, j = kk % NJ;
        if (!(e < sn && self >= 0 && t == self + e)) v = (float)src[(e * nt + t) * K + j * KB + c];
      }
      const float h = tf32_head(v);
      o[q] = h;
      o[4096 + q] = v - h;
    }
  }
}

// Near densities of each leaf as pre-split tiles of 64 columns (right-hand
// sides) x 32 k (k = NJ t + j over the leaf's near triangles t, components
// j), TF32 head then tail, canonical layout: per leaf at sbase[i], tile (ct,
// kt) at (ct nkt + kt) 4096 floats; positions past R or K written as zeros.
// CTAs (leaf, blockIdx.y) over the leaf's tiles: the triangle of each k is
// found by walking the leaf's near boxes, the densities are read 64
// right-hand sides at a time (coalesced) into shared memory (rows of 72
// floats: neither phase has bank conflicts) and written in tile order.
__global__ void __launch_bounds__(256)
k_near_sigma_split(const NearArgs a, int R, int NJ, const double* __restrict__ g0, const double* __restrict__ g1,
                   const long long* __restrict__ sbase, const int* __restrict__ ntri, float* __restrict__ S) {
  __shared__ float sv[32][72];
  __shared__ int tri_k[32];
  const int i = blockIdx.x;
  const int K = NJ * ntri[i], nkt = (K + 31) / 32, nct = (R + 63) / 64;
  float* o = S + sbase[i];
  for (int tile = blockIdx.y; tile < nct * nkt; tile += gridDim.y) {
    const int ct = tile / nkt, kt = tile % nkt;
    __syncthreads();  // the previous tile's reads of sv and tri_k are done
    if (threadIdx.x < 32) {
      const int kk = 32 * kt + threadIdx.x;
      int tri = -1;
      if (kk < K) {
        int u = kk / NJ;
        for (int b = a.nb_start[i]; b < a.nb_start[i + 1]; b++) {
          const int sb = a.nb_items[b], cnt = a.box_src_count[sb];
          if (u < cnt) {
            tri = a.box_src_start[sb] + u;
            break;
          }
          u -= cnt;
        }
      }
      tri_k[threadIdx.x] = tri;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < 2048; q += blockDim.x) {
      const int n = q & 63, k = q >> 6, r = 64 * ct + n, tri = tri_k[k];
      float v = 0.0f;
      if (tri >= 0 && r < R) {
        const int j = (32 * kt + k) % NJ;
        v = (float)(j >= 3 ? g1 : g0)[((size_t)tri * 3 + (j % 3)) * R + r];
      }
      sv[k][n] = v;
    }
    __syncthreads();
    float* t = o + (long long)tile * 4096;
    for (int q = threadIdx.x; q < 2048; q += blockDim.x) {
      const int k = (q & 3) | (((q >> 5) & 7) << 2), n = ((q >> 2) & 7) | ((q >> 8) << 3);
      const float v = sv[k][n], h = tf32_head(v);
      t[q] = h;
      t[2048 + q] = v - h;
    }
  }
}

// The self pairs of the mixed replay in FP64: per source point of the leaf
// (thread) and group of SELF_RB right-hand sides (blockIdx.y), the FP64
// stored block (NJ density components x KB outputs, read once into
// registers) times the FP64 densities of the point's own triangle, ADDED to
// the outputs.
constexpr int SELF_RB = 8;
template <int NJ, int KB>
__global__ void __launch_bounds__(128)
k_near_self64(const NearArgs a, int R, const double* __restrict__ g0, const double* __restrict__ g1,
              const long long* __restrict__ base, const int* __restrict__ ntri, const double* __restrict__ store,
              int nsrc) {
  constexpr int K = NJ * KB;
  const int i = blockIdx.x, r0 = blockIdx.y * SELF_RB, leaf = a.leaves[i];
  const int s0 = a.box_src_start[leaf], sn = a.do_src ? a.box_src_count[leaf] : 0;
  const int self = near_self_pos(a, i, leaf);
  if (self < 0) return;
  const long long nt = ntri[i];
  const int rn = min(SELF_RB, R - r0);
  for (int e = threadIdx.x; e < sn; e += blockDim.x) {
    const int pid = s0 + e;
    const double* blk = store + base[i] + ((long long)e * nt + self + e) * K;
    double bk[K];
#pragma unroll
    for (int k = 0; k < K; k++) bk[k] = blk[k];
    for (int rr = 0; rr < rn; rr++) {
      const int r = r0 + rr;
      double out[KB];
#pragma unroll
      for (int c = 0; c < KB; c++) out[c] = 0.0;
#pragma unroll
      for (int j = 0; j < NJ; j++) {
        const double sv = (j >= 3 ? g1 : g0)[((size_t)pid * 3 + (j % 3)) * R + r];
#pragma unroll
        for (int c = 0; c < KB; c++) out[c] += bk[j * KB + c] * sv;
      }
      double* U = a.u_src + 3 * ((size_t)nsrc * r + pid);
#pragma unroll
      for (int c = 0; c < 3; c++) U[c] += out[c];
      if (KB == 9 && a.dostrain_src) {
        double* E = a.e_src + 6 * ((size_t)nsrc * r + pid);
#pragma unroll
        for (int c = 0; c < 6; c++) E[c] += out[3 + c];
      }
    }
  }
}

static void launch_near_self64(cudaStream_t st, const NearArgs& a, int R, int NJ, int KB, const double* g0,
                               const double* g1, const long long* base, const int* ntri, const double* store,
                               int nsrc) {
  const dim3 grid(a.nleaf, (R + SELF_RB - 1) / SELF_RB);
  if (NJ == 3 && KB == 3)
    k_near_self64<3, 3><<<grid, 128, 0, st>>>(a, R, g0, g1, base, ntri, store, nsrc);
  else if (NJ == 3 && KB == 9)
    k_near_self64<3, 9><<<grid, 128, 0, st>>>(a, R, g0, g1, base, ntri, store, nsrc);
  else if (NJ == 6 && KB == 3)
    k_near_self64<6, 3><<<grid, 128, 0, st>>>(a, R, g0, g1, base, ntri, store, nsrc);
  else if (NJ == 6 && KB == 9)
    k_near_self64<6, 9><<<grid, 128, 0, st>>>(a, R, g0, g1, base, ntri, store, nsrc);
  else
    throw CudaError{(int)cudaErrorInvalidValue};
  count_launch();
}

// Near densities of each leaf as the B operand: S[r][NJ t + j] at soff[leaf]
// (row length ntri NJ rounded up to 4), from sigma[(tri 3 + comp) R + r]
// (g0: the first layer stored, g1: the double layer when both are).
__global__ void __launch_bounds__(256)
k_near_sigma_tc(const NearArgs a, int R, int NJ, const double* __restrict__ g0, const double* __restrict__ g1,
                const long long* __restrict__ soff, const int* __restrict__ ntri, float* __restrict__ S) {
  const int i = blockIdx.x;
  const int K = NJ * ntri[i], Kp = (K + 3) & ~3;
  float* o = S + soff[i];
  int pos = 0;
  for (int b = a.nb_start[i]; b < a.nb_start[i + 1]; b++) {
    const int sb = a.nb_items[b];
    const int tr0 = a.box_src_start[sb], trn = a.box_src_count[sb];
    for (int q = threadIdx.x; q < trn * NJ * R; q += blockDim.x) {
      const int r = q / (trn * NJ), k = q % (trn * NJ), t = k / NJ, j = k % NJ;
      const double* sg = j >= 3 ? g1 : g0;
      o[(size_t)r * Kp + (size_t)(pos + t) * NJ + j] = (float)sg[((size_t)(tr0 + t) * 3 + (j % 3)) * R + r];
    }
    pos += trn;
  }
}

// Add the products C[r][KB e + c] (per leaf at coff) to the outputs.
__global__ void __launch_bounds__(256)
k_near_scatter_tc(const NearArgs a, int R, int KB, const long long* __restrict__ coff, const double* __restrict__ C,
                  int nsrc, int ntgt) {
  const int i = blockIdx.x, r = blockIdx.y, leaf = a.leaves[i];
  const int s0 = a.box_src_start[leaf], sn = a.do_src ? a.box_src_count[leaf] : 0;
  const int t0 = a.box_tgt_start[leaf], tn = a.do_tgt ? a.box_tgt_count[leaf] : 0;
  const int M = KB * (sn + tn);
  const double* Cr = C + coff[i] + (size_t)r * M;
  for (int row = threadIdx.x; row < M; row += blockDim.x) {
    const int e = row / KB, c = row % KB;
    const bool src = e < sn;
    const int pid = src ? s0 + e : t0 + (e - sn);
    const size_t np = src ? (size_t)nsrc : (size_t)ntgt;
    const double v = Cr[row];
    if (c < 3) {
      (src ? a.u_src : a.u_tgt)[3 * (np * r + pid) + c] += v;
    } else if (src ? a.dostrain_src : a.dostrain_tgt) {
      (src ? a.e_src : a.e_tgt)[6 * (np * r + pid) + (c - 3)] += v;
    }
  }
}

void launch_near_store_tc(cudaStream_t st, const NearArgs& a, const long long* base, const long long* fbase,
                          const int* ntri, int K, int KB, const double* store, float* out) {
  if (a.nleaf <= 0) return;
  k_near_store_tc<<<dim3(a.nleaf, 64), 256, 0, st>>>(a, base, fbase, ntri, K, KB, store, out);
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}

void launch_near_split_store(cudaStream_t st, const NearArgs& a, const long long* base, const long long* tbase,
                             const int* ntri, int K, int KB, const double* store, float* out) {
  if (a.nleaf <= 0) return;
  k_near_split_store<<<dim3(a.nleaf, 32), 256, 0, st>>>(a, base, tbase, ntri, K, KB, store, out);
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}

void launch_near_split(cudaStream_t st, const NearArgs& a, int R, int NJ, int KB, const double* g0,
                       const double* g1, const long long* sbase, const int* ntri, float* S, int ntask,
                       const BulkTask* tasks, const float* A, const long long* coff, double* C, int nsrc, int ntgt,
                       const long long* base, const double* store, int* err, cudaEvent_t* ev) {
  if (a.nleaf <= 0 || R <= 0) return;
  k_near_sigma_split<<<dim3(a.nleaf, 8), 256, 0, st>>>(a, R, NJ, g0, g1, sbase, ntri, S);
  count_launch();
  if (ev) EFMM_CUDA_TRY(cudaEventRecord(ev[0], st));
  launch_tc_bulk<double>(st, ntask, tasks, A, S, C, err, 64);
  if (ev) EFMM_CUDA_TRY(cudaEventRecord(ev[1], st));
  k_near_scatter_tc<<<dim3(a.nleaf, R), 256, 0, st>>>(a, R, KB, coff, C, nsrc, ntgt);
  count_launch();
  if (a.do_src) {
    launch_near_self64(st, a, R, NJ, KB, g0, g1, base, ntri, store, nsrc);
  }
  EFMM_CUDA_TRY(cudaGetLastError());
}

void launch_near_tc(cudaStream_t st, const NearArgs& a, int R, int NJ, int KB, const double* g0, const double* g1,
                    const long long* soff, const int* ntri, float* S, int ntask, const GemmTask* tasks,
                    const float* A, const long long* coff, double* C, int nsrc, int ntgt, const long long* base,
                    const double* store) {
  if (a.nleaf <= 0 || R <= 0) return;
  k_near_sigma_tc<<<a.nleaf, 256, 0, st>>>(a, R, NJ, g0, g1, soff, ntri, S);
  count_launch();
  launch_gemm_tc(st, ntask, tasks, A, S, C, tc_err_ptr(), R <= 64 ? 64 : 128);
  k_near_scatter_tc<<<dim3(a.nleaf, R), 256, 0, st>>>(a, R, KB, coff, C, nsrc, ntgt);
  count_launch();
  if (a.do_src) {
    launch_near_self64(st, a, R, NJ, KB, g0, g1, base, ntri, store, nsrc);
  }
  EFMM_CUDA_TRY(cudaGetLastError());
}

// ---------------------------------------------------------------- launchers
void launch_tri_prep(cudaStream_t st, int n, const double* tri, const int* perm, const double* ssl,
                     const double* sdl, int dosl, int dodl, TriRec* out) {
  if (n <= 0) return;
  k_tri_prep<<<(n + 127) / 128, 128, 0, st>>>(n, tri, perm, ssl, sdl, dosl, dodl, out); count_launch();
}

void launch_near_leaf(cudaStream_t st, const NearArgs& a) {
  if (a.nleaf <= 0) return;
  k_near_leaf<<<a.nleaf, NF_WARPS * 32, 0, st>>>(
      a.nleaf, a.leaves, a.nb_start, a.nb_items, a.box_src_start, a.box_src_count,
      a.box_tgt_start, a.box_tgt_count, a.trir, a.src_pts, a.tgt_pts, a.dosl, a.dodl,
      a.dostrain_src, a.dostrain_tgt, a.do_src, a.do_tgt, a.rlam, a.rmu, a.u_src, a.e_src,
      a.u_tgt, a.e_tgt); count_launch();
}

void launch_near_store(cudaStream_t st, const NearArgs& a, const long long* base, const int* ntri, int K,
                       int dodisp, double* store) {
  if (a.nleaf <= 0) return;
  k_near_store<<<a.nleaf, NF_WARPS * 32, 0, st>>>(a, base, ntri, K, dodisp, store); count_launch();
}

void launch_near_replay(cudaStream_t st, const NearArgs& a, const long long* base, const int* ntri, int K,
                        int dodisp, const double* ssl, const double* sdl, const double* store) {
  if (a.nleaf <= 0) return;
  k_near_replay<<<a.nleaf, 256, 0, st>>>(a, base, ntri, K, dodisp, ssl, sdl, store); count_launch();
}

void launch_near_batch(cudaStream_t st, const NearArgs& a, int nchunk, const int* chunk_leaf,
                       const int* chunk_e0, int R, int dostrain, const double* ssl, const double* sdl,
                       int ntri_all, int nsrc, int ntgt, const long long* sbase, const int* sntri,
                       const double* store) {
  if (nchunk <= 0 || R <= 0) return;
  if (R > 64) throw CudaError{(int)cudaErrorInvalidValue};
  const int nl = a.dosl + a.dodl;
  const int K = nl * 3 * (3 + 6 * dostrain);
  const int RB = (R + 15) / 16;
  const int smem = (int)(sizeof(double) * (NB_PTS * NB_TRI * K + NB_TRI * 6 * 16 * RB));
  auto go = [&](auto kern) {
    EFMM_CUDA_TRY(smem_raise(kern, (int)(smem)));
    kern<<<nchunk, NB_THREADS, smem, st>>>(a, chunk_leaf, chunk_e0, R, K, dostrain, ssl, sdl, ntri_all, nsrc,
                                           ntgt, sbase, sntri, store);
    count_launch();
  };
  if (store) {
    const int nlay = nl, str = dostrain;
    const double* g0 = a.dosl ? ssl : sdl;
    const double* g1 = sdl;
    const int smem2 = (int)(sizeof(double) * (NB_PTS * NB_TRI * K + NB_TRI * 3 * nlay * 16 * RB));
    auto go2 = [&](auto kern) {
      EFMM_CUDA_TRY(smem_raise(kern, (int)(smem2)));
      kern<<<nchunk, NB_THREADS, smem2, st>>>(a, chunk_leaf, chunk_e0, R, g0, g1, nsrc, ntgt, sbase, sntri, store);
      count_launch();
    };
#define EFMM_RB(RBV)                                                         \
  if (nlay == 1 && !str) go2(k_near_replay_batch<RBV, 1, 0>);                \
  else if (nlay == 1) go2(k_near_replay_batch<RBV, 1, 1>);                   \
  else if (!str) go2(k_near_replay_batch<RBV, 2, 0>);                        \
  else go2(k_near_replay_batch<RBV, 2, 1>);
    switch (RB) {
      case 1: EFMM_RB(1) break;
      case 2: EFMM_RB(2) break;
      case 3: EFMM_RB(3) break;
      default: EFMM_RB(4) break;
    }
#undef EFMM_RB
  } else {
    switch (RB) {
      case 1: go(k_near_batch<1, false>); break;
      case 2: go(k_near_batch<2, false>); break;
      case 3: go(k_near_batch<3, false>); break;
      default: go(k_near_batch<4, false>); break;
    }
  }
  EFMM_CUDA_TRY(cudaGetLastError());
}

void launch_direct_all(cudaStream_t st, int ntri, const TriRec* trir, int nsrc, const double* src_pts,
                       int ntgt, const double* tgt_pts, int dosl, int dodl, int dostrain_src,
                       int dostrain_tgt, double rlam, double rmu, double* u_src, double* e_src,
                       double* u_tgt, double* e_tgt) {
  int nep = nsrc + ntgt;
  if (nep <= 0) return;
  k_direct_all<<<(nep + NF_WARPS - 1) / NF_WARPS, NF_WARPS * 32, 0, st>>>(
      ntri, trir, nsrc, src_pts, ntgt, tgt_pts, dosl, dodl, dostrain_src, dostrain_tgt, rlam, rmu,
      u_src, e_src, u_tgt, e_tgt); count_launch();
}

}  // namespace efmm
