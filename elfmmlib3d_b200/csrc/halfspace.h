// halfspace.h -- image part of the half-space layer potentials (internal header).
#pragma once
#include <cuda_runtime.h>

namespace efmm {

// One triangle with its normal and densities (user order).
struct HsTri {
  double v[9], n[3], sl[3], dl[3];
};

// Image displacement u (m,3) and strain e6 (m,6: xx yy zz xy xz yz) at
// targets tgt (m,3) of the single (ssl) and double (sdl, normals nrm)
// layers on triangles tri (n,3,3); NULL disables a layer.  work: n records.
void launch_hs_image(cudaStream_t st, int n, const double* tri, const double* nrm, const double* ssl,
                     const double* sdl, int m, const double* tgt, double lam, double mu, HsTri* work, double* u,
                     double* e6);

}  // namespace efmm
