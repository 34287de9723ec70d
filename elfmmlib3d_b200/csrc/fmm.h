// fmm.h -- far-field launchers (internal header).
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

namespace efmm {

// One translation operator: kind 0 = M2L (d = offset in box units),
// 1 = M2M, 2 = L2L (d = child centre - parent centre in parent units).
struct OpDesc {
  int kind, p;
  double d[3];
  long long off;  // offset of the matrix in the operator pool (doubles)
};

struct TransPair {
  int src, dst;
  double alpha;
};
// One 128 x 128 output tile: operator group, first row, the group's first
// pair, the group's column count (pairs x C) and the tile's first column.
struct TransTask {
  int group, row0, pair0, ncols, col0;
};

struct P2MArgs {
  const int* leaves;
  const int *level, *ijk, *sstart, *scount;
  double c0[3], size;
  const double *tri, *nrm, *ssl, *sdl;  // tree order
  int dosl, dodl, p;
  double c1, c2, inv2mu;
  double* mpole;
};

struct L2TArgs {
  const int* leaves;
  const int *level, *ijk, *sstart, *scount, *tstart, *tcount;
  double c0[3], size;
  const double* local;
  const double *src_pts, *tgt_pts;  // tree order
  int p, do_src, do_tgt, dostrain_src, dostrain_tgt;
  double c1;
  double *u_src, *e_src, *u_tgt, *e_tgt;
};

void launch_build_ops(cudaStream_t st, int nop, const OpDesc* ops, double* mats, int maxp);
void launch_p2m(cudaStream_t st, int nleaf, const P2MArgs& a);
template <class T>
void launch_translate(cudaStream_t st, int ntask, const TransTask* tasks, const TransPair* pairs,
                      const T* mats, const long long* mat_off, const int* mat_dim, int D, int C,
                      const T* src, T* dst);
void launch_l2t(cudaStream_t st, int nleaf, const L2TArgs& a);

}  // namespace efmm
