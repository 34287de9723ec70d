// particles.h -- near field and direct sum of the particle FMM (internal
// header; particles.cu).
#pragma once
#include <cuda_runtime.h>
#include "kernels.h"

namespace efmm {

// Near field of the particle FMM over the plan's near lists: NearArgs with
// part_sl / part_dl (tree order), nu the dipole orientations (tree order);
// results ADDED to the tree-order outputs (strain as 6 entries).
void launch_near_points(cudaStream_t st, const NearArgs& a, const double* nu, double rlam, double rmu);
// Direct O(N^2) sum: all n sources act, the first ne sources and the m
// targets are evaluated; user order, outputs overwritten (null skips one).
void launch_part_direct(cudaStream_t st, int n, int ne, const double* src, const double* sl, const double* dl,
                        const double* nu, int m, const double* tgt, double rlam, double rmu, double* u_src,
                        double* e_src, double* u_tgt, double* e_tgt);

}  // namespace efmm
