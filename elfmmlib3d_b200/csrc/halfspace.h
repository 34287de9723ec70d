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
// eps: relative tolerance of the adaptive integration of near-singular
// sub-triangles (hs_quad_eps); *ncap (may be null) counts sub-triangles kept
// at the depth cap without meeting it.
void launch_hs_image(cudaStream_t st, int n, const double* tri, const double* nrm, const double* ssl,
                     const double* sdl, int m, const double* tgt, double lam, double mu, double eps, int* ncap,
                     HsTri* work, double* u, double* e6);
// tolerance of the image quadrature for iprec: min(1e-6, eps(iprec) / 10)
double hs_quad_eps(int iprec);
// The image part at targets (m,3) of point forces sl and point jumps dl
// with orientations nu at the n points src (user order; null disables a
// layer): u (m,3), e6 (m,6), overwritten.  The half-space particle direct sum.
void launch_part_image(cudaStream_t st, int n, const double* src, const double* sl, const double* dl,
                       const double* nu, int m, const double* tgt, double lam, double mu, double* u, double* e6);

// Near field of the image FMM: the unit-density image responses of every
// (target, near triangle) pair of each near leaf, written in the stored
// near-field layout (per leaf at base[leaf]: [target][near triangle][K],
// K = layers x 3 directions x (3 displacement + 6 strain if dstr)), so that
// the batched replay contracts them with any number of right-hand sides.
// Targets are the reflected points (x1, x2, -x3) in tree order; triangles,
// normals tree order.
struct HsStoreArgs {
  const int *leaves, *nb_start, *nb_items;
  const int *box_src_start, *box_src_count, *box_tgt_start, *box_tgt_count;
  const double *tri, *nrm, *tgt;
  const long long* base;
  const int* ntri;
  int dosl, dodl, dstr, K;
  double lam, mu;
  double eps = 1e-6;     // adaptive tolerance of near-singular sub-triangles
  int* ncap = nullptr;   // sub-triangles kept at the depth cap (counter, may be null)
  // particles: sources are the points pts (tree order), nrm their dipole
  // orientations; a pair block is the image kernel at the point
  int points = 0;
  const double* pts = nullptr;
};
// The per-device counter of sub-triangles kept at the adaptive depth cap
// (device address, for HsStoreArgs::ncap and launch_hs_image), and its value
// read and cleared (blocking).
int* hs_ncap_ptr();
int hs_take_ncap();
// One CTA per chunk of (near leaf, first of 8 targets).
void launch_hs_store(cudaStream_t st, const HsStoreArgs& a, int nchunk, const int* chunk_leaf,
                     const int* chunk_e0, double* store);

}  // namespace efmm
