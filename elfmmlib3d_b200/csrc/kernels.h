// kernels.h -- host-side launchers for the device kernels (internal header).
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

namespace efmm {

struct NearArgs {
  int nleaf;
  const int *leaves, *nb_start, *nb_items;
  const int *box_src_start, *box_src_count, *box_tgt_start, *box_tgt_count;
  const TriRec* trir;
  const double *src_pts, *tgt_pts;
  int dosl, dodl, dostrain_src, dostrain_tgt, do_src, do_tgt;
  double rlam, rmu;
  double *u_src, *e_src, *u_tgt, *e_tgt;
};

void launch_tri_prep(cudaStream_t st, int n, const double* tri, const int* perm, const double* ssl,
                     const double* sdl, int dosl, int dodl, TriRec* out);
void launch_near_leaf(cudaStream_t st, const NearArgs& a);
void launch_near_store(cudaStream_t st, const NearArgs& a, const long long* base, const int* ntri, int K,
                       int dodisp, double* store);
void launch_near_replay(cudaStream_t st, const NearArgs& a, const long long* base, const int* ntri, int K,
                        int dodisp, const double* ssl, const double* sdl, const double* store);
// R <= 64 right-hand sides; densities (ntri_all, 3, R) tree order, outputs
// (R, nsrc or ntgt, 3 or 6) tree order, ADDED to.  With store != NULL the
// pair blocks come from the ITER store (per leaf at sbase, sntri near
// triangles) instead of being computed.
void launch_near_batch(cudaStream_t st, const NearArgs& a, int nchunk, const int* chunk_leaf,
                       const int* chunk_e0, int R, int dostrain, const double* ssl, const double* sdl,
                       int ntri_all, int nsrc, int ntgt, const long long* sbase = nullptr,
                       const int* sntri = nullptr, const double* store = nullptr);
void launch_direct_all(cudaStream_t st, int ntri, const TriRec* trir, int nsrc, const double* src_pts,
                       int ntgt, const double* tgt_pts, int dosl, int dodl, int dostrain_src,
                       int dostrain_tgt, double rlam, double rmu, double* u_src, double* e_src,
                       double* u_tgt, double* e_tgt);

}  // namespace efmm
