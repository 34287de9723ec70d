// fmm.h -- far-field launchers (internal header).
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

namespace efmm {

// One translation operator: kind 0 = M2L (d = offset in box units),
// 1 = M2M, 2 = L2L (d = child centre - parent centre in parent units),
// 3 = M2L of the half-space kernel U = z log(r + z) - r (d as for kind 0).
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

// One 128 x 128 tile of C[col][row] = sum_k A[k][row] B[col][k]
// (A: K rows of lda, B: N columns of ldb, C: N columns of ldc).
struct GemmTask {
  long long a_off, b_off, c_off;
  int M, N, K, lda, ldb, ldc, row0, col0;
};

struct P2MArgs {
  const int* leaves;
  const int *level, *ijk, *sstart, *scount;
  double c0[3], size;
  const double *tri, *nrm, *ssl, *sdl;  // tree order
  int dosl, dodl, p;
  double c1, c2, inv2mu;
  double* mpole;
  // right-hand side r = blockIdx.y: density component d of triangle t at
  // ssl/sdl[r * rstride + t * tstride + d * dstride]; expansion columns
  // 4r..4r+3 of C per box
  int C = 4;
  long long rstride = 0, tstride = 3, dstride = 1;
  const double* wnorm = nullptr;  // product form: rows scaled by wnorm[row] if set
  // half-space image columns: alpha = (lam + mu)/(lam + 2 mu) and the Lame
  // constants of the double-layer tensor
  double alpha = 0, lam = 0, mu = 0;
  // particles (k_p2m only): one node per source at pts (tree order), weight
  // 1, nrm = the dipole orientations (src/elfmm3dpart.f:319-420)
  int points = 0;
  const double* pts = nullptr;
  // level of the forest's problem columns (-1: one problem); sets the origin
  // of the linear pass (lame_origin)
  int flev = -1;
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
  // right-hand side blockIdx.y: expansion columns 4r..4r+3 of C per box,
  // outputs at r * (3 or 6) * (number of sources or targets)
  int C = 4;
  long long nsrc = 0, ntgt = 0;
  double alpha = 0, mu = 0;  // half-space image recombination
  const double* wnorm = nullptr;  // two-stage L2T in FP32: functionals x wnorm[row]
  int flev = -1;  // as P2MArgs::flev
};

// Leading dimension of the L2T functionals and sums of a leaf of P points:
// 9 P rounded up to a multiple of 4, so that every row starts on 16 bytes
// (the products' 16-byte copies in FP32 and FP64).
__host__ __device__ inline long long l2t_ld(int P) { return (9LL * P + 3) & ~3LL; }

void launch_build_ops(cudaStream_t st, int nop, const OpDesc* ops, double* mats, int maxp);
void launch_p2m(cudaStream_t st, int nleaf, const P2MArgs& a, int nrhs = 1);
// P2M of R right-hand sides as a product (columns 4R per box); writes mpole
// (T = double, or float for the mixed-precision form).  Returns false (and
// launches nothing) when the order is too high for its shared-memory tiles.
template <class T>
bool launch_p2m_gemm(cudaStream_t st, int nleaf, const P2MArgs& a, int R, T* mpole);
// L2T of R right-hand sides as a product over (chunks of 8 points of a leaf,
// 256 columns); local (boxes, 4R, D) in TB (float: normalised basis, rows
// rescaled by wnorm).  Returns false when the order is too high.
// Two-stage P2M of R right-hand sides for one wave of leaves: node features
// F (per leaf at foff: 4 x 12 x triangles rows of D), node weights W (per
// leaf at woff: 4R columns of 4 x 12 x triangles; node records of 8 doubles
// per node at noff), then the batched product
// into mpole (tasks cut by the caller).
template <class T>
void launch_p2m_twostage(cudaStream_t st, const P2MArgs& a, int R, int nwleaf, const int* wleaves,
                         const long long* foff, const long long* woff, const long long* noff, double* nrec,
                         int max_nodes, T* F, T* W, int ntask, const GemmTask* tasks, T* mpole,
                         bool do_product = true);
// Direct L2T of the image columns for few right-hand sides (one CTA per
// leaf and right-hand side, FP64 locals: columns kind * R + r of 6R per box,
// the U column at local + ubase + (box R + r) D).
// Returns false (nothing launched) when the order is too high for its tiles.
bool launch_l2t_img(cudaStream_t st, int nleaf, const L2TArgs& a, int R, long long ubase);
// The product stage alone (FP32: tensor cores unless ELFMM3D_TC=0).  Tasks
// cover 128 x 128 output tiles; bn = 64 runs the tensor-core tiles 64 columns
// wide (every task then has at most 64 columns).
template <class T>
void gemm_product(cudaStream_t st, int ntask, const GemmTask* tasks, const T* F, const T* W, T* C, int bn = 128);
template <class TB>
bool launch_l2t_gemm(cudaStream_t st, int nchunk, const int* chunk_leaf, const int* chunk_e0, const L2TArgs& a,
                     int R, const TB* local, const double* wnorm);
// Two-stage L2T of R right-hand sides for one wave of leaves: functionals G
// (per leaf at goff: D rows of 9 x points), the FP64 product into S (per leaf
// at soff: 4R columns of 9 x points; tasks cut by the caller, B = local),
// then the Lame recombination into the outputs.
// image = true: the half-space image columns (7R per leaf, targets only)
// and their recombination (k_l2t_finish_img).
// T = float: normalised-basis functionals (L2TArgs.wnorm) and FP32
// normalised local expansions, the product on the tensor cores.
// do_g = false: the functionals at goff are already there (resident from an
// earlier pass over the same geometry) and are not recomputed.
template <class T>
void launch_l2t_twostage(cudaStream_t st, const L2TArgs& a, int R, int nwleaf, const int* wleaves,
                         const long long* goff, const long long* soff, int max_pts, T* Gbuf, T* Sbuf,
                         int ntask, const GemmTask* tasks, const T* local, bool image = false, bool do_g = true);
// The two-stage L2T from split operands (mixed form, functionals resident):
// functionals as split A tiles (per leaf at goff, written when do_g), the
// wave's local expansions (FP32 normalised, free-space or image column
// layout, nb boxes) as split B tiles at boff, the bulk-copy product
// (k_tc_bulk, 128-column tiles) into S at soff (columns of l2t_ld(P)), then
// the Lame recombination.
struct BulkTask;
void launch_l2t_bulk(cudaStream_t st, const L2TArgs& a, int R, int nwleaf, const int* wleaves, const long long* goff,
                     const long long* soff, const long long* boff, int max_pts, float* scratch, int ntask,
                     const BulkTask* tasks, const float* local, long long nb, bool image, bool do_g, int* err);
// Two-stage P2M of the half-space image columns (7R per box, tasks cut by
// the caller): node features with second-derivative rows (9 x 12 x
// triangles rows of D per leaf at foff), node weights (7R columns of 9 x 12
// x triangles per leaf at woff), batched product into mpole.
// Stage 1 of the P2M factored through unit-density multipoles, for one wave
// of leaves (at most maxtn triangles each): H (nk = 4 free-space or
// anti-image kinds, 7 with the image columns; per leaf at hoff,
// [kind][ns x triangles][D], geometry only) for the ns density components
// sbase.. (0..2 single layer, 3..5 double layer), and the density operand S
// (per leaf at soff, R rows of ns x triangles rounded up to a multiple of 4).
// Stage 2 is gemm_product with K = ns x triangles, N = R.  False (nothing
// launched) when the order is too high for its shared memory
// (p2m_unit_smem(p, T is float) > 227 KB).  do_h = false: H is already
// there (resident from an earlier pass) and only S is formed.  split (T =
// float): H and S as split tiles for k_tc_bulk instead: per leaf and kind q,
// H's tile (row tile mt of ceil(D / 128), K tile kt of nkt = ceil(ns tn /
// 32)) at hoff + ((q ceil(D / 128) + mt) nkt + kt) 8192, S's tiles of 64
// right-hand sides at soff + (ct nkt + kt) 4096 (k_p2m_sigma_split).
template <class T>
bool launch_p2m_unit(cudaStream_t st, const P2MArgs& a, int R, int nk, int nwleaf, int maxtn, const int* wleaves,
                     const long long* hoff, const long long* soff, int sbase, int ns, T* H, T* S, bool do_h = true,
                     bool split = false);
size_t p2m_unit_smem(int p, bool fp32);
// Direct P2M of the image columns (one CTA per leaf and right-hand side):
// columns kind * R + r of 6R per box (kinds 0..5) and the U column at
// mpole + ubase + (box R + r) D.  For few right-hand sides.
template <class T>
void launch_p2m_img(cudaStream_t st, int nleaf, const P2MArgs& a, int R, long long ubase, T* mpole);
template <class T>
void launch_p2m_img_twostage(cudaStream_t st, const P2MArgs& a, int R, int nwleaf, const int* wleaves,
                             const long long* foff, const long long* woff, const long long* noff, double* nrec,
                             int max_nodes, T* F, T* W, int ntask, const GemmTask* tasks, T* mpole,
                             bool do_product = true);
template <class T>
void launch_translate(cudaStream_t st, int ntask, const TransTask* tasks, const TransPair* pairs,
                      const T* mats, const long long* mat_off, const int* mat_dim, int D, int C,
                      const T* src, T* dst);
void launch_l2t(cudaStream_t st, int nleaf, const L2TArgs& a, int nrhs = 1);
// The FP32 product of k_gemm_tn<float> on the tensor cores (tc_gemm.cu):
// tcgen05.mma kind::tf32 with the 3-term head/tail split (FP32 accuracy).
// *err is set when a bounded wait runs out (the tile is then not stored).
// bn: output tile width (64 or 128 columns).  The double-output form adds
// the tensor cores' K-tile sums in FP64.
void launch_gemm_tc(cudaStream_t st, int ntask, const GemmTask* tasks, const float* A, const float* B, float* C,
                    int* err, int bn = 128);
void launch_gemm_tc(cudaStream_t st, int ntask, const GemmTask* tasks, const float* A, const float* B, double* C,
                    int* err, int bn = 128);
// Per-device error flag of the tensor-core products; tc_take_error reads
// and clears it (blocking).
int* tc_err_ptr();
bool tc_take_error();
bool tc_enabled();

}  // namespace efmm
