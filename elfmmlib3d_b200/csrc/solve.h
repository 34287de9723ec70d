// solve.h -- the iterative solver loop over the layer-potential operator
// (internal header; solve.cu).
#pragma once

namespace efmm {

class Plan;

// The minimal-residual iteration of the reference's matlab/gmres_simple.m on
// the device, R right-hand sides at once (rhs and x: (R, n, 3) device
// arrays).  F: the free-space plan (geometry set with iter = true, no
// targets); I: the half-space image plan (iter = true, mindlin = true,
// targets = the reflected centroids) or null for free space.  kind 0: the
// traction at the centroids of the double layer (nrm (n, 3) device, the
// normals the traction is taken on); 1: the displacement at the centroids of
// the single layer.  precision as in evaluate_batch.  Per column: iterations,
// final |r| / |b|, and 0 converged / 4 maxit reached / 8 stagnated.
// Returns an ier code (a failed operator application).
int solve_layers(Plan* F, Plan* I, int kind, double rlam, double rmu, int R, const double* d_nrm,
                 const double* d_rhs, double* d_x, double tol, int maxit, int precision, int* iters,
                 double* relres, int* ier_cols);

}  // namespace efmm
