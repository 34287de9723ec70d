/*
 * elfmm3d_b200.h -- C ABI of the B200 elastostatic triangle-layer FMM.
 *
 * Two families of entry points:
 *
 * 1. Drop-in replacements for the reference's Fortran subroutines.  Every
 *    argument is passed by reference, arrays are Fortran column-major
 *    (triangle(3,3,n), sigma(3,n), ptfrc(3,n), strain(3,3,n)), integers are
 *    32-bit and no hidden string lengths exist.  The symbols carry the
 *    gfortran/ifort trailing underscore, so an unmodified Fortran caller links
 *    against libelfmm3d_b200.so in place of the reference objects.  Host
 *    arrays in, host arrays out; device memory is managed internally (the
 *    reference likewise allocates its own scratch).  Outputs carry no 1/(4 pi)
 *    factor, exactly like the reference.
 *
 * 2. A native device API (efmm_*) taking device pointers and returning ier,
 *    used for resident-data pipelines, benchmarking and tests.
 *
 * Error codes (ier): 0 ok, 4 tree construction failed, 8 device allocation
 * failed, 16 invalid argument; 256 CUDA error, 512 stored-operator handle
 * mismatch, 1024 no CUDA device.
 */
#ifndef ELFMM3D_B200_H
#define ELFMM3D_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- reference-compatible entry points ------------------------------- */

/* Replaces elfmm3dtria (src/elfmm3dtria.f:71-74): on-surface evaluation at the
 * n source points (triangle centroids). */
void elfmm3dtria_(int *ier, const int *iprec, const double *rlam, const double *rmu,
                  const double *triangle, const double *trinorm, const int *nparts,
                  const double *source, const int *ifsingle, const double *sigma_sl,
                  const int *ifdouble, const double *sigma_dl, const int *ifptfrc, double *ptfrc,
                  const int *ifstrain, double *strain);

/* Replaces elfmm3dtriatarg (src/elfmm3dtria.f:162-167): on-surface and
 * off-surface targets. */
void elfmm3dtriatarg_(int *ier, const int *iprec, const double *rlam, const double *rmu,
                      const double *triangle, const double *trinorm, const int *nparts,
                      const double *source, const int *ifsingle, const double *sigma_sl,
                      const int *ifdouble, const double *sigma_dl, const int *ifptfrc,
                      double *ptfrc, const int *ifstrain, double *strain, const int *ntargs,
                      const double *target, const int *ifptfrctarg, double *ptfrctarg,
                      const int *ifstraintarg, double *straintarg);

/* Replaces el3dtriadirecttarg (src/elfmm3dtria.f:1483-1487): O(N^2) direct
 * evaluation with the analytic triangle integrals.  (No ier, as in the
 * reference; failures are reported on stderr and leave outputs at zero.) */
void el3dtriadirecttarg_(const double *rlam, const double *rmu, const double *triangle,
                         const double *trinorm, const int *nsource, const double *source,
                         const int *ifsingle, const double *sigma_sl, const int *ifdouble,
                         const double *sigma_dl, const int *ifptfrc, double *ptfrc,
                         const int *ifstrain, double *strain, const int *ntarget,
                         const double *target, const int *ifptfrctarg, double *ptfrctarg,
                         const int *ifstraintarg, double *straintarg);

/* Replaces elfmm3dtriatargiter (src/elfmm3dtria_iter_1.f:160-165): the
 * iterative-solver variant that keeps the near-field interactions between
 * calls on the same geometry.  icomp_type as in the reference
 * (src/elfmm3dtria_iter_1.f:95-107): 1 evaluate without storage, 2 evaluate
 * and store, 3 evaluate with the stored near field (same geometry, iprec,
 * layers and outputs as the store; new densities), 4 tree only (sets lused),
 * 5 store and evaluate the near field alone, 0 nothing.  The stored operator
 * lives in device memory owned by the library; wsave receives an 8-word
 * handle naming it, so lused is always 8.  With lwsave < 8, icomp_type 2 and 3
 * evaluate without storage, as the reference does when wsave is too short.
 * A handle that no longer matches (other geometry, iprec, layers, outputs or
 * Lame constants, released or evicted store) gives ier 512.  At most four
 * stores are live; a fifth evicts the least recently used. */
void elfmm3dtriatargiter_(int *ier, const int *iprec, const double *rlam, const double *rmu,
                          const double *triangle, const double *trinorm, const int *nparts,
                          const double *source, const int *ifsingle, const double *sigma_sl,
                          const int *ifdouble, const double *sigma_dl, const int *ifptfrc,
                          double *ptfrc, const int *ifstrain, double *strain, const int *ntargs,
                          const double *target, const int *ifptfrctarg, double *ptfrctarg,
                          const int *ifstraintarg, double *straintarg, const int *icomp_type,
                          double *wsave, const int *lwsave, int *lused);

/* Replaces elfmm3dtriaiter (src/elfmm3dtria_iter_1.f:43-47): the ITER variant
 * without off-surface targets. */
void elfmm3dtriaiter_(int *ier, const int *iprec, const double *rlam, const double *rmu,
                      const double *triangle, const double *trinorm, const int *nparts,
                      const double *source, const int *ifsingle, const double *sigma_sl,
                      const int *ifdouble, const double *sigma_dl, const int *ifptfrc,
                      double *ptfrc, const int *ifstrain, double *strain, const int *icomp_type,
                      double *wsave, const int *lwsave, int *lused);

/* Replaces elfmm3dparttarg (src/elfmm3dpart.f:104-218): the particle FMM in
 * free space.  Point forces sigma_sl(3,n) and point displacement
 * discontinuities sigma_dl(3,n) with orientations sigma_dv(3,n) at
 * source(3,n); displacement ptfrc(3,n) and strain(3,3,n) at the sources
 * (self-interaction excluded) and at target(3,nt).  Same decomposition,
 * tree and translations as the triangle FMM (one P2M node per source; near
 * field by point pairs).  ier as elfmm3dtriatarg_. */
void elfmm3dparttarg_(int *ier, const int *iprec, const double *rlam, const double *rmu, const int *nparts,
                      const double *source, const int *ifsingle, const double *sigma_sl, const int *ifdouble,
                      const double *sigma_dl, const double *sigma_dv, const int *ifptfrc, double *ptfrc,
                      const int *ifstrain, double *strain, const int *ntargs, const double *target,
                      const int *ifptfrctarg, double *ptfrctarg, const int *ifstraintarg, double *straintarg);

/* Replaces elfmm3dpart (src/elfmm3dpart.f:52-102): as above, no targets. */
void elfmm3dpart_(int *ier, const int *iprec, const double *rlam, const double *rmu, const int *nparts,
                  const double *source, const int *ifsingle, const double *sigma_sl, const int *ifdouble,
                  const double *sigma_dl, const double *sigma_dv, const int *ifptfrc, double *ptfrc,
                  const int *ifstrain, double *strain);

/* Replaces el3dpartdirecttarg (src/elfmm3dpart.f:506-712): the O(N^2)
 * particle direct sum, on the GPU. */
void el3dpartdirecttarg_(const double *rlam, const double *rmu, const int *nsource, const double *source,
                         const int *ifsingle, const double *sigma_sl, const int *ifdouble, const double *sigma_dl,
                         const double *sigma_dv, const int *ifptfrc, double *ptfrc, const int *ifstrain,
                         double *strain, const int *ntarget, const double *target, const int *ifptfrctarg,
                         double *ptfrctarg, const int *ifstraintarg, double *straintarg);

/* Replaces elhfmm3dparttarg (src/elhfmm3dpart.f:99-498): the particle FMM
 * in the Mindlin half space z <= 0 (traction-free z = 0), arguments as
 * elfmm3dparttarg_: the free-space particle FMM plus the image part (image
 * FMM, one P2M node per source, the image kernels at the points as its near
 * field).  Sources and targets in z <= 0, else ier 16. */
void elhfmm3dparttarg_(int *ier, const int *iprec, const double *rlam, const double *rmu, const int *nparts,
                       const double *source, const int *ifsingle, const double *sigma_sl, const int *ifdouble,
                       const double *sigma_dl, const double *sigma_dv, const int *ifptfrc, double *ptfrc,
                       const int *ifstrain, double *strain, const int *ntargs, const double *target,
                       const int *ifptfrctarg, double *ptfrctarg, const int *ifstraintarg, double *straintarg);

/* Replaces elhfmm3dpart (src/elhfmm3dpart.f:47-97): as above, no targets. */
void elhfmm3dpart_(int *ier, const int *iprec, const double *rlam, const double *rmu, const int *nparts,
                   const double *source, const int *ifsingle, const double *sigma_sl, const int *ifdouble,
                   const double *sigma_dl, const double *sigma_dv, const int *ifptfrc, double *ptfrc,
                   const int *ifstrain, double *strain);

/* Replaces elh3dpartdirecttarg (listed in src/elfmm3dpart.f:33-36): the
 * half-space particle direct sum (free-space pairs plus the image kernels
 * of every source), on the GPU. */
void elh3dpartdirecttarg_(const double *rlam, const double *rmu, const int *nsource, const double *source,
                          const int *ifsingle, const double *sigma_sl, const int *ifdouble, const double *sigma_dl,
                          const double *sigma_dv, const int *ifptfrc, double *ptfrc, const int *ifstrain,
                          double *strain, const int *ntarget, const double *target, const int *ifptfrctarg,
                          double *ptfrctarg, const int *ifstraintarg, double *straintarg);

/* Host evaluation of one (point, particle) pair of the particle near field
 * (the decomposition the device uses): u[3], strain e6[6] (xx yy zz xy xz
 * yz) at x of a point force sl and a point jump dl with orientation nu at y
 * (either layer may be NULL).  No counterpart in the reference; the CPU
 * check of the particle kernels. */
int efmm_part_pair_host(double rlam, double rmu, const double *x, const double *y, const double *sl,
                        const double *dl, const double *nu, double *u, double *e6);

/* nrhs right-hand sides from host arrays (no counterpart in the reference):
 * geometry as in elfmm3dtriatarg_, sigma_sl/sigma_dl (3,n,nrhs) column-major
 * (NULL disables a layer), outputs ptfrc (3,n,nrhs), strain (3,3,n,nrhs),
 * ptfrctarg (3,nt,nrhs), straintarg (3,3,nt,nrhs) (NULL disables one).
 * precision as in efmm_plan_evaluate_batch.  Blocking; returns ier. */
int efmm_batch_host(int iprec, double rlam, double rmu, int n, const double *triangle,
                    const double *trinorm, const double *source, int nt, const double *target,
                    int nrhs, const double *sigma_sl, const double *sigma_dl, double *ptfrc,
                    double *strain, double *ptfrctarg, double *straintarg, int precision);

/* Half-space self-evaluation of nrhs right-hand sides from host arrays (no
 * single counterpart in the reference: it replaces the loop of
 * elfmm3dtriatargiter + elhfmm3dtriatargiter call pairs over slip vectors,
 * icomp_type 2 then 3, and the drivers' sum of direct arrival and image,
 * examples/elhfmm3dtria_self_iter_dr.f:222-385).  Geometry as in
 * elfmm3dtria_ (z <= 0), sigma_sl/sigma_dl (3,n,nrhs) column-major (NULL
 * disables a layer); outputs the total displacement ptfrc (3,n,nrhs) and
 * strain (3,3,n,nrhs) at the centroids (NULL disables one).  precision 0
 * FP64, 1 mixed.  icomp_type 1 evaluates; 2 evaluates and stores both near
 * fields on the device behind the 8-word handle in wsave (lwsave >= 8);
 * 3 replays them with new densities (same geometry, iprec, nrhs, precision,
 * layers and outputs, else 512), each of the two passes replayed as one
 * CUDA graph for nrhs <= 64.  One store is live at a time: a new store
 * invalidates the previous handle.  Blocking; returns ier. */
int elhfmm3dtria_batch_host(int iprec, double rlam, double rmu, int n, const double *triangle,
                            const double *trinorm, const double *source, int nrhs,
                            const double *sigma_sl, const double *sigma_dl, double *ptfrc,
                            double *strain, int precision, int icomp_type, double *wsave,
                            int lwsave);

/* Replaces elhfmm3dtriatargiter (src/elhfmm3dtria_iter.f:46-51): the image
 * part of the half-space (z <= 0, traction-free surface z = 0) single and
 * double layer potentials at targets, Mindlin's solution (the direct
 * arrival is the free-space evaluation, elfmm3dtriatarg_ / elfmm3dtria_).
 * Evaluated by the image FMM (anti-image and Mindlin B/C far field, image
 * near field by refined quadrature) on the sources and the reflected
 * targets, to the accuracy of iprec.  icomp_type 1 evaluates; 2 evaluates
 * and stores the image near field on the device behind the 8-word handle in
 * wsave (lwsave >= 8; shorter: a plain evaluation); 3 reuses that store
 * with new densities on the same geometry (512 for a handle that does not
 * match); 5 behaves as 2; 0 and 4 only set lused = 8.  Sources or targets
 * above z = 0 give ier 16. */
void elhfmm3dtriatargiter_(int *ier, const int *iprec, const double *rlam, const double *rmu,
                           const double *triangle, const double *trinorm, const int *nparts,
                           const double *source, const int *ifsingle, const double *sigma_sl,
                           const int *ifdouble, const double *sigma_dl, const int *ntargs,
                           const double *target, const int *ifptfrctarg, double *ptfrctarg,
                           const int *ifstraintarg, double *straintarg, const int *icomp_type,
                           double *wsave, const int *lwsave, int *lused);

/* Half-space total field (no single counterpart in the reference, whose
 * drivers add the two calls, examples/elhfmm3dtria_self_iter_dr.f:331-385):
 * the direct arrival (elfmm3dtriatarg_, on-surface at the centroids) plus
 * the image part (elhfmm3dtriatargiter_, icomp_type 1) at the centroids
 * (ptfrc, strain) and at the targets (ptfrctarg, straintarg), arguments as
 * in elfmm3dtriatarg_.  The image part of both point sets is one image-FMM
 * pass.  Sources, centroids or targets above z = 0 give ier 16 (nothing
 * evaluated). */
void elhfmm3dtria_total_(int *ier, const int *iprec, const double *rlam, const double *rmu,
                         const double *triangle, const double *trinorm, const int *nparts,
                         const double *source, const int *ifsingle, const double *sigma_sl,
                         const int *ifdouble, const double *sigma_dl, const int *ifptfrc, double *ptfrc,
                         const int *ifstrain, double *strain, const int *ntargs, const double *target,
                         const int *ifptfrctarg, double *ptfrctarg, const int *ifstraintarg,
                         double *straintarg);

/* Frees the device store named by an ITER handle (no counterpart in the
 * reference, whose store is the caller's wsave array), including the two
 * plans of an elhfmm3dtria_batch_host store.  512 if the handle names no
 * live store. */
int efmm_iter_release(const double *wsave, int lwsave);

/* Device bytes held by the store an ITER handle names; -1 if none. */
long long efmm_iter_stored_bytes(const double *wsave, int lwsave);

/* ---- native device API ----------------------------------------------- */

typedef struct efmm_plan efmm_plan;

int efmm_device_count(void);

/* Create a plan on CUDA device `device` (its own stream).  NULL on failure. */
efmm_plan *efmm_plan_create(int device);
void efmm_plan_destroy(efmm_plan *plan);

/* Geometry (device pointers, user order): tri (n,3,3), nrm (n,3), src (n,3),
 * tgt (nt,3).  iter != 0 selects the ITER leaf capacity (2x), mindlin != 0
 * the half-space root box (centred on z = 0).  Builds the tree, the lists,
 * the work lists and the translation operators. */
int efmm_plan_set_geometry(efmm_plan *plan, int n, const double *tri, const double *nrm,
                           const double *src, int nt, const double *tgt, int iprec, int iter,
                           int mindlin);

/* Leaf capacity of the plan's following set_geometry calls (boxes split
 * while they hold more than nbox sources or targets); nbox <= 0 restores the
 * iprec table (src/elfmm3dtria.f:702-722).  Another capacity gives another
 * tree (not the reference's) with the same accuracy contract. */
int efmm_plan_set_leaf(efmm_plan *plan, int nbox);

/* A forest of independent problems for the plan's following set_geometry
 * calls (no counterpart in the reference): forest = {root centre x, y, z,
 * root side, level L} -- the tree's root is this cube instead of the
 * points' bounding cube, every box above level L splits, and boxes of
 * different columns of level L (grid positions (i, j), any k) are never
 * neighbours, so the problems placed one per column do not interact.  A
 * Mindlin plan needs centre z = 0.  NULL: one problem (the default).  L in
 * 1..15; ier 16 otherwise. */
int efmm_plan_set_forest(efmm_plan *plan, const double *forest);

/* Evaluate with device densities ssl/sdl (n,3; NULL disables a layer) into
 * device outputs u_src (n,3), e_src (n,3,3), u_tgt (nt,3), e_tgt (nt,3,3)
 * (NULL disables an output).  Blocks until the results are complete. */
int efmm_plan_evaluate(efmm_plan *plan, double rlam, double rmu, const double *ssl,
                       const double *sdl, double *u_src, double *e_src, double *u_tgt,
                       double *e_tgt);

/* nrhs right-hand sides in one pass (no counterpart in the reference, which
 * takes one density pair per call): ssl/sdl (nrhs,n,3), outputs
 * u_src (nrhs,n,3), e_src (nrhs,n,3,3), u_tgt (nrhs,nt,3), e_tgt (nrhs,nt,3,3),
 * device pointers, NULL disables as in efmm_plan_evaluate.  The near-field
 * pair responses are computed once for all right-hand sides and the
 * P2M and translations run as products over boxes x passes x right-hand
 * sides.  precision 0: FP64 throughout, the same results as nrhs calls of
 * efmm_plan_evaluate; precision 1: mixed, P2M products, expansions and
 * translations in FP32, near field and local evaluation in FP64. */
int efmm_plan_evaluate_batch(efmm_plan *plan, double rlam, double rmu, int nrhs, const double *ssl,
                             const double *sdl, double *u_src, double *e_src, double *u_tgt,
                             double *e_tgt, int precision);

/* Useful flops per expansion column (one Laplace pass of one right-hand
 * side) of the current geometry: P2M, M2M, M2L, L2L, L2T. */
void efmm_plan_flops(const efmm_plan *plan, double *f5);

/* Device-resident ITER evaluation (the plan's geometry must have been set
 * with iter != 0): mode 1 computes and stores the near-field interactions
 * and evaluates, mode 2 evaluates with the stored interactions (same layers,
 * outputs and Lame constants as the store, else 512).  Arguments as in
 * efmm_plan_evaluate. */
int efmm_plan_evaluate_iter(efmm_plan *plan, double rlam, double rmu, const double *ssl,
                            const double *sdl, double *u_src, double *e_src, double *u_tgt,
                            double *e_tgt, int mode);

/* Batched ITER evaluation: efmm_plan_evaluate_batch with the stored
 * near-field interactions of efmm_plan_evaluate_iter (mode 1 stores them,
 * mode 2 reuses them; the same store serves both entry points when the
 * layers, outputs and Lame constants agree, else 512).  The replay is one
 * sparse-block product of the stored pair responses with all right-hand
 * sides (the ITER store of src/elfmm3dtria_iter_1.f:1240-1419 applied to
 * nrhs density pairs at once). */
int efmm_plan_evaluate_batch_iter(efmm_plan *plan, double rlam, double rmu, int nrhs, const double *ssl,
                                  const double *sdl, double *u_src, double *e_src, double *u_tgt,
                                  double *e_tgt, int precision, int mode);

/* Half-space image part as an FMM (replaces the direct image sum of
 * elhfmm3dtriatargiter, src/elhfmm3dtria_iter.f:544-840: anti-image elastic
 * FMM, Mindlin B/C FMM, image near field).  The plan's geometry must have
 * been set with mindlin != 0 and, as targets, the reflections (x1, x2, -x3)
 * of the points x (z <= 0) where the field is wanted; sources in z <= 0.
 * ssl/sdl (nrhs,n,3) device, NULL disables a layer; outputs at the points
 * x: u_tgt (nrhs,nt,3), e_tgt (nrhs,nt,3,3).  precision 0 FP64, 1 mixed
 * (FP32 expansions and translations); mode 0 plain, 1 store the image
 * near-field blocks and use them, 2 reuse them (512 on mismatch). */
int efmm_plan_evaluate_image(efmm_plan *plan, double rlam, double rmu, int nrhs, const double *ssl,
                             const double *sdl, double *u_tgt, double *e_tgt, int precision, int mode);

/* The image part by direct summation over all (target, triangle) pairs with
 * the quadrature of the image near field (host arrays as in
 * elhfmm3dtriatargiter; u (nt,3), e (nt,3,3), NULL skips an output): the
 * O(n nt) check of the image FMM.  The quadrature refines sub-triangles by
 * distance to the reflected target and integrates the near-singular ones
 * adaptively to relative tolerance min(1e-6, eps(iprec) / 10), the scheme
 * of tria3adam (src/tria3adamar.f:33-395), with a depth cap. */
int efmm_hs_image_direct(int iprec, double rlam, double rmu, const double *tri, const double *nrm, int n,
                         const double *ssl, const double *sdl, int nt, const double *tgt, double *u, double *e);

/* Sub-triangles of the image quadrature (direct sum or image near-field
 * store) kept at the adaptive depth cap without meeting the tolerance since
 * the last call, on the current device (the reference reports the same
 * event as ier 4 of tria3adam, src/tria3adamar.f:65-67); clears the count.
 * -1 on a CUDA error. */
int efmm_hs_capped(void);

/* Host check (no GPU) of the image FMM's M2L for the kernel
 * U = z log(r + z) - r (src/mindlinpieces.f:29): order-p local expansion at
 * offset X (box units, X2 >= 0) of nsrc random unit-box sources against
 * their direct sum; returns the largest relative error (-1 on bad input). */
double efmm_u_m2l_selfcheck(int p, double X0, double X1, double X2, int nsrc, unsigned seed);

/* Host evaluation of one (triangle, point) interaction of the free-space
 * analytic near field, the closed-form triangle integrals the device near
 * field runs (the role of elust3triadirecttarg_one / eltst3triadirecttarg_one,
 * src/elfmm3dtria.f:1689-2015, 2368-2911): displacement u[3] and strain
 * e6[6] (xx yy zz xy xz yz) at x of the single layer ssl[3] and/or double
 * layer sdl[3] (global components; NULL disables one; the double layer's
 * normal is the vertex-order normal) on triangle tri[9]; self = 1 when x is
 * the triangle's own centroid (principal value / finite part).  For checks;
 * no device is used.  Returns 0, or 16 for NULL arguments. */
int efmm_pair_eval_host(double rlam, double rmu, const double *tri, const double *ssl, const double *sdl,
                        const double *x, int self, double *u, double *e6);

/* Host evaluation of the image kernels that the half-space image near field
 * and direct image sum integrate (no counterpart in the reference, whose
 * kernels are src/el3greenh.f:643-787 with src/mindlinpieces.f): responses
 * at target x (3) to the three unit point forces (layer 0) or the three
 * unit displacement jumps with normal nrm (layer 1) at source s (3), both in
 * z < 0; out[27] = per direction displacement (3) then strain (xx yy zz xy
 * xz yz), no 1/(4 pi).  For checks of the kernels; no device is used.
 * Returns 0, or 16 for a bad layer or a NULL pointer. */
int efmm_mindlin_image_kernel(int layer, double lam, double mu, const double *x, const double *s,
                              const double *nrm, double *out);

/* Device check of the tensor-core FP32 product (tcgen05.mma kind::tf32,
 * 3-term split) that carries the batched P2M: random A (K x M) and B
 * (N x K) against an FP64 host product; *rel = relative l2 error, *timeout
 * != 0 if a bounded wait in the kernel ran out.  Returns 0 or an ier. */
int efmm_tc_gemm_selfcheck(int M, int N, int K, unsigned seed, double *rel, int *timeout);
/* The same check with output tiles bn = 64 or 128 columns wide (the 64-wide
 * tiles carry the factored P2M product, N = number of right-hand sides);
 * aligned != 0: leading dimensions rounded up to multiples of 4 (16-byte
 * rows, vector loads), else odd ones. */
int efmm_tc_gemm_selfcheck_tile(int M, int N, int K, int bn, int aligned, unsigned seed, double *rel,
                                int *timeout);

/* Repeated batched evaluations as one CUDA graph (no counterpart in the
 * reference): the same arguments as efmm_plan_evaluate_batch_iter /
 * efmm_plan_evaluate_image.  The first call with new arguments (parameters
 * and device pointers) runs the pass, captures a second identical pass and
 * launches it; later calls with the same arguments launch the captured
 * graph only, so new densities must be written into the same buffers.
 * Batch: mode 0 (analytic near field) or 2 (a store made by an earlier
 * mode-1 call); image: the stored near field of an earlier mode-1 call.
 * nrhs <= 64 (one pass per call; else IER 16).
 * The first call should not run while another capture on the plan's stream
 * is in progress.  A new geometry drops the graph. */
int efmm_plan_evaluate_batch_graph(efmm_plan *plan, double rlam, double rmu, int nrhs, const double *ssl,
                                   const double *sdl, double *u_src, double *e_src, double *u_tgt,
                                   double *e_tgt, int precision, int mode);
int efmm_plan_evaluate_image_graph(efmm_plan *plan, double rlam, double rmu, int nrhs, const double *ssl,
                                   const double *sdl, double *u_tgt, double *e_tgt, int precision);

/* Device bytes of the plan's stored near field (0 if none). */
long long efmm_plan_stored_bytes(const efmm_plan *plan);

/* Orders of the mixed form (precision 1; no counterpart in the reference):
 * its expansions and translations are truncated at max(eps(iprec), eps)
 * -- by default eps = 5e-8, about the FP32 rounding of the result, so that
 * no truncation is finer than the arithmetic; eps <= 0 keeps the iprec
 * orders.  *order (if not NULL) receives the mixed form's expansion order.
 * Applies to later calls on the plan's current geometry. */
int efmm_plan_set_mixed_floor(efmm_plan *plan, double eps, int *order);

/* Flops of one pass's translation launches (M2M, M2L, L2L into f3) for
 * nrhs right-hand sides at the orders of the form `precision` selects
 * (1: the mixed form's), counted as the kernels run them (factored: two
 * rotations and the shift along z per pair and column).  Measurement
 * support, no counterpart in the reference. */
int efmm_plan_translation_flops(efmm_plan *plan, int nrhs, int precision, double *f3);

/* Direct sum at the first nsub source points only (centroids 0..nsub-1,
 * self-aware), outputs u_src (nsub,3), e_src (nsub,3,3): the FP64 check of a
 * large evaluation on a subset. */
int efmm_plan_evaluate_direct_subset(efmm_plan *plan, double rlam, double rmu, int nsub,
                                     const double *ssl, const double *sdl, double *u_src,
                                     double *e_src);

/* Same outputs from the all-pairs direct sum on the plan's geometry. */
int efmm_plan_evaluate_direct(efmm_plan *plan, double rlam, double rmu, const double *ssl,
                              const double *sdl, double *u_src, double *e_src, double *u_tgt,
                              double *e_tgt);

/* CPU self-check (no device): builds the factored translation operators
 * (rotation, shift along z, rotation back) of the 316 M2L offsets and the
 * 8 M2M and 8 L2L shifts at order p and tolerance eps and stores in *worst
 * the largest relative difference to the dense operators over every
 * stride-th of them.  Returns the number of operators built. */
int efmm_factored_selfcheck(int p, double eps, int stride, double *worst);

/* Number of this library's kernels launched so far in the process. */
long long efmm_kernel_launches(void);

/* CUDA events on the plan's stream: record slot (0..7); elapsed time in ms
 * between two recorded slots (waits for the second). */
int efmm_plan_record(efmm_plan *plan, int slot);
float efmm_plan_elapsed(efmm_plan *plan, int a, int b);

/* Direct sum without device allocation.  No counterpart in the reference: it
 * is for callers that cannot allocate device memory when they need the
 * result (a memory pool that already holds the free device memory, or a
 * latency-bound loop that cannot afford an allocation's synchronisation).
 * Same result as el3dtriadirecttarg_ for device-resident inputs (user order):
 * tri (n,3,3), src (n,3), ssl/sdl (n,3; NULL disables a layer), tgt (nt,3);
 * outputs u_src (n,3), e_src (n,3,3), u_tgt (nt,3), e_tgt (nt,3,3), NULL
 * disables one.  Intermediates live in fixed file-scope device arrays
 * (about 11 MB per GPU, held until exit once loaded): at most 32768
 * triangles and 65536 evaluation points (n + nt) per call; larger sizes
 * return 16 with a message on stderr.  Enqueues on `stream` (a cudaStream_t,
 * NULL = legacy default stream) and returns.  The first call on a device
 * loads the scratch (CUDA loads modules lazily by default) and looks up its
 * address: make it (n = 1 is enough) before a memory pool reserves the
 * device's free memory and before any stream capture.  Calls that overlap on
 * the GPU share the scratch and race.  Not usable after cudaDeviceReset in
 * the same process.  A launch error already pending in the calling thread
 * makes the call return 256 without running and without clearing it. */
int efmm_direct_noalloc(double rlam, double rmu, int n, const double *tri, const double *src,
                        const double *ssl, const double *sdl, int nt, const double *tgt,
                        double *u_src, double *e_src, double *u_tgt, double *e_tgt, void *stream);

/* Per-stage device times (ms) of the last evaluate: total, prep, p2m, m2m,
 * m2l, l2l, l2t, near. */
void efmm_plan_timings(const efmm_plan *plan, float *ms8);

/* The batched P2M product stage of the last evaluate_batch / evaluate_image
 * (the largest kernel of the mixed form): out2[0] device ms (CUDA events
 * around each product launch), out2[1] its useful FP32 flops. */
void efmm_plan_product_stats(const efmm_plan *plan, double *out2);

/* The tensor-core product of the last mixed replay of the stored near field
 * from its split (outside CUDA-graph capture): out2[0] device ms (CUDA
 * events around the launch), out2[1] the bytes of its operands and results
 * (split store, split densities, FP64 products); zeros when the last mixed
 * replay did not use the split.  No counterpart in the reference. */
void efmm_plan_near_stats(const efmm_plan *plan, double *out2);

/* Host wall-clock ms of the last set_geometry: tree, lists, work lists
 * (with the tree-order gathers), translation operators. */
void efmm_plan_setup_timings(const efmm_plan *plan, float *ms4);

/* info[0..7] = nboxes, nlev, expansion order p, leaf capacity nbox,
 * near-field point pairs, M2L box pairs, kernels launched by the last
 * evaluate, far field enabled. */
void efmm_plan_info(const efmm_plan *plan, long long *info8);

/* Export the tree in the reference layout (1-based, src/d3tstrcr.f:1292-1310):
 * boxes (nboxes,20), iz (n), iztarg (nt), laddr (nlev+1,2), center (3), size,
 * and lists 1..5 as CSR: lstart (5, nboxes+1) and litems (sum of counts).
 * With litems == NULL only lcount[5] is filled. */
int efmm_plan_tree_export(const efmm_plan *plan, int *boxes, int *iz, int *iztarg, int *laddr,
                          double *center_size4, int *lstart, int *litems, long long *lcount5);

/* Iterative solution over the layer-potential operator (the reference's
 * solver loop is MATLAB over a function handle, matlab/gmres_simple.m and
 * matlab/Contents.m:32-33; this is its minimal-residual iteration on the
 * device): nrhs right-hand sides rhs (nrhs,n,3) -> densities x (nrhs,n,3),
 * device arrays, each column with its own coefficients.  free_plan: geometry
 * set with iter = 1 and no targets; image_plan: NULL (free space) or the
 * half-space image plan (iter = 1, mindlin = 1, targets = the reflected
 * centroids (x1, x2, -x3)).  kind 0: x is a double-layer density (slip),
 * the operator the traction (lam tr(e) I + 2 mu e) nrm at the centroids
 * (nrm (n,3) device); kind 1: x is a single-layer density (traction), the
 * operator the displacement at the centroids.  The first application stores
 * the near fields if the plans hold none; later ones replay them (CUDA
 * graphs for nrhs <= 64).  Stops a column at |r| < tol |b| (ier_cols 0),
 * when |r| stops decreasing (8) or after maxit steps (4); iters and the
 * final |r| / |b| per column (each may be NULL).  Returns ier. */
int efmm_plan_solve(efmm_plan *free_plan, efmm_plan *image_plan, int kind, double rlam, double rmu, int nrhs,
                    const double *nrm, const double *rhs, double *x, double tol, int maxit, int precision,
                    int *iters, double *relres, int *ier_cols);

/* The same iteration on the host for a dense row-major n x n matrix A and
 * nrhs right-hand sides B (nrhs,n) -> X (nrhs,n): the CPU check of the
 * algorithm (no device used). */
int efmm_gcr_dense_host(int n, int nrhs, const double *A, const double *B, double *X, double tol, int maxit,
                        int *iters, double *relres, int *ier_cols);

/* The form of the tensor-core FP32 product for this process: 1 (default)
 * operands streamed by cp.async into a ring of raw tiles, 0 staged through
 * registers (also ELFMM3D_TC_RING=0).  Returns the previous form.  No
 * counterpart in the reference. */
int efmm_tc_variant(int ring);

/* Form of the mixed-precision products whose one operand depends on the
 * geometry only (the stored near field's replay, the resident L2T
 * functionals) for this process: 1 (default) that operand split once into
 * TF32 head / tail tiles, the other split per call, both streamed by bulk
 * copies into the tensor cores (8 bytes per element; used where it fits), 0
 * FP32 operands split in shared memory on every call (also
 * ELFMM3D_SPLIT=0).  Returns the previous form.  No counterpart in the
 * reference. */
int efmm_split_variant(int split);

/* Self-check of the bulk-copy product of split operands on random A (K x M)
 * and B (N x K) in [-1, 1) (M <= 8192, N <= 1024, bn 64 or 128 columns per
 * tile, fp64 != 0: FP64 K-tile sums): relative l2 error against an FP64 host
 * product in *rel, the kernel's error flag (a wait that ran out) in
 * *timeout.  Returns 0, 16 (bad sizes) or 256 (device error).  Test entry;
 * no counterpart in the reference. */
int efmm_tc_bulk_selfcheck(int M, int N, int K, int bn, int fp64, unsigned seed, double *rel, int *timeout);

/* The autotuner (no counterpart in the reference, whose tuning is the fixed
 * iprec tables, src/elfmm3dtria.f:702-722): per key (knob, expansion order,
 * leaf capacity, expansion columns per box, precision, plan kind) the first
 * passes time every candidate implementation of the knob's stage
 * (TUNE_VISITS = 2 runs each, the faster kept) and later passes run the
 * fastest.  Knobs 0, 1, 2: the FP32 translations of the M2M, M2L, L2L
 * stages on the tensor cores (candidate 0) or the CUDA cores (1).  Decisions
 * persist in the file named by ELFMM3D_TUNE_FILE when it is set.  pick
 * returns the candidate to run; report records a timed run (ms); dump
 * writes "knob p nbox C prec kind decided ms..." lines into buf (len bytes)
 * and returns the full length. */
int efmm_tune_pick(int knob, int p, int nbox, int C, int prec, int kind, int ncand);
void efmm_tune_report(int knob, int p, int nbox, int C, int prec, int kind, int ncand, int cand, float ms);
void efmm_tune_reset(void);
int efmm_tune_dump(char *buf, int len);

/* Checks of the FP32 factored translations on the tensor cores (no
 * counterpart in the reference): one M2L, one M2M and one L2L group of order
 * p (1..31).  _selfcheck emulates the kernel's arithmetic on the host (tiles,
 * their layout, the padded rows, the row maps of the three factors, the
 * 3-term split); _device runs the kernel on the GPU for npair box pairs of C
 * columns each.  Both return 0 and the relative l2 difference from the FP64
 * product of the same FP32 operators in *rel (_device: *timeout != 0 if a
 * bounded wait ran out).  _bench times reps launches on the same inputs:
 * mean ms in *ms. */
int efmm_rot_tc_selfcheck(int p, unsigned seed, double *rel);
int efmm_rot_tc_selfcheck_device(int p, int C, int npair, unsigned seed, double *rel, int *timeout);
int efmm_rot_tc_bench(int p, int C, int npair, int reps, double *ms, int *timeout);

/* ---- many independent half-space problems in one pass -----------------
 * (no counterpart in the reference, whose drivers evaluate one fault per
 * call: the half-space self-evaluation of examples/elhfmm3dtria_self_iter_dr.f
 * :331-385, direct arrival plus image part, for every problem).  The
 * problems are moved side by side in x and y (z kept: the half-space kernels
 * depend on x and y through differences only), one per column of boxes of a
 * common root cube centred on z = 0, and one free-space plan and one image
 * plan are built over all of them as a forest (efmm_plan_set_forest): every
 * stage of both passes is one launch over the boxes of all problems. */
typedef struct efmm_forest efmm_forest;

efmm_forest *efmm_forest_create(int device);
void efmm_forest_destroy(efmm_forest *forest);

/* The problems' geometry, device arrays concatenated in problem order:
 * counts (host, nprob) triangles per problem, tri (n,3,3), nrm (n,3),
 * centroids cen (n,3), n = sum of counts, every vertex and centroid in
 * z <= 0 (else ier 16).  iter != 0: the ITER leaf capacity (for mode 1/2
 * evaluations).  Builds both plans. */
int efmm_forest_set_geometry(efmm_forest *forest, int nprob, const int *counts, const double *tri,
                             const double *nrm, const double *cen, int iprec, int iter);

/* Half-space displacement u (n,3) and strain e (n,3,3) at every problem's
 * centroids (device, problem order; NULL disables an output) of the
 * densities ssl / sdl (n,3; NULL disables a layer), each problem on its own.
 * precision 0 FP64, 1 mixed; mode 0, or 1 / 2 to store / replay both plans'
 * near fields (geometry set with iter != 0).  Blocks. */
int efmm_forest_evaluate(efmm_forest *forest, double rlam, double rmu, const double *ssl, const double *sdl,
                         double *u, double *e, int precision, int mode);

/* Leaf capacities of the forest's free-space and image plans for the next
 * efmm_forest_set_geometry (<= 0: the default, the plans' iprec table for
 * the free-space plan and half of it for the image plan, whose refined
 * image near field costs more per pair than its far field). */
int efmm_forest_set_leaf(efmm_forest *forest, int nbox_free, int nbox_image);

/* Tolerance floor of both plans' mixed-form orders (efmm_plan_set_mixed_floor;
 * eps <= 0 keeps the iprec orders).  No counterpart in the reference. */
int efmm_forest_set_mixed_floor(efmm_forest *forest, double eps);

/* The same for the forest behind elhfmm3dtria_many_host (its later calls).
 * No counterpart in the reference. */
int efmm_many_host_set_mixed_floor(double eps);

/* The forest's plans: which 0 the free-space (direct arrival) plan, 1 the
 * image plan (for efmm_plan_info, efmm_plan_tree_export, timings). */
efmm_plan *efmm_forest_plan(efmm_forest *forest, int which);

/* The placement (host code, no device): from each problem's centroid
 * bounding box bb (nprob,6: min x, y, z, max x, y, z) the root cube
 * root5 = {centre x, y, z = 0, side, level L} and the x and y shift of each
 * problem, shift (nprob,2), that moves its box to the centre of column
 * k = i + 2^L j.  ier 16 on nprob < 1, bad boxes or a box above z = 0. */
int efmm_forest_layout(int nprob, const double *bb, double *root5, double *shift);

/* Host arrays in and out: the problems of efmm_forest_set_geometry and the
 * outputs of efmm_forest_evaluate (mode 0) in one call, on a forest kept
 * between calls. */
int elhfmm3dtria_many_host(int iprec, double rlam, double rmu, int nprob, const int *counts, const double *tri,
                           const double *nrm, const double *cen, const double *ssl, const double *sdl, double *u,
                           double *e, int precision);

/* ---- flat-triangle geometry I/O (host code) ----------------------------
 * The Cart3D ".tri" format: "nverts nfaces", nverts vertices (3 reals),
 * nfaces vertex-index triples (1-based), free format.  Arrays in the
 * reference's layout: verts(3,nverts), ifaces(3,nfaces). */

/* Replaces atrireadchk (src/trilib.f:59-88), which reads from a Fortran
 * unit; here from a file name.  Reads the sizes into *nverts / *nfaces, then
 * the arrays if they fit: ier 0 ok, 1 the file cannot be opened, 2 lv <
 * nverts, 3 li < nfaces (the reference's codes; lv = li = 0 asks for the
 * sizes), 4 malformed file (not a number, index outside 1..nverts). */
int efmm_tri_read(const char *path, double *verts, int lv, int *nverts, int *ifaces, int li, int *nfaces);

/* Replaces atriwrite (src/trilib.f:113-128): writes the file (vertices
 * with 17 significant digits, so they read back bit for bit).  ier 0 / 1. */
int efmm_tri_write(const char *path, const double *verts, int nverts, const int *ifaces, int nfaces);

/* Replaces matlab/atrirefine.m: every face split into four at its edge
 * midpoints.  verts1 (3, nverts + 3 nfaces): the vertices, then the
 * midpoints of edges 1-2, 2-3, 3-1 of each face (three blocks in face order,
 * shared edges not merged); ifaces1 (3, 4 nfaces): the corner triangles of
 * vertex 1, 2, 3 of each face, then the middle triangles (four blocks).
 * ier 16 on an index outside 1..nverts. */
int efmm_tri_refine(const double *verts, int nverts, const int *ifaces, int nfaces, double *verts1,
                    int *ifaces1);

/* Replaces buildtri (src/trilib.f:192-240): triangle(3,3,ntri),
 * centroids(3,ntri), unit normals trinorm(3,ntri) and areas triarea(ntri)
 * (NULL skips one) from the vertex arrays; the normal and area formulas of
 * triangle_norm / triangle_area (src/trilib.f:245-318).  ier 16 on an index
 * outside 1..nverts. */
int efmm_tri_build(const double *verts, int nverts, int ntri, const int *itrivert, double *triangle,
                   double *centroids, double *trinorm, double *triarea);

#ifdef __cplusplus
}
#endif
#endif
