// kernels.h -- host-side launchers for the device kernels (internal header).
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"
#include "fmm.h"

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
  const double* part_sl = nullptr;  // particles: densities (n, 3) in tree order
  const double* part_dl = nullptr;
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
// Mixed-precision replay of the stored near field on the tensor cores: the
// FP64 store converted once to FP32 in the product layout (per leaf at the
// store's offsets: A[NJ t + j][KB e + c], lda = KB x points, self pairs
// zero), then per call the near densities gathered per leaf (S at soff, rows
// of NJ x ntri rounded up to 4), the product tasks (per leaf and 128-row
// tile: C at coff, ldc = KB x points, FP64 sums), the results ADDED to the
// outputs, and the self pairs added in FP64 from the FP64 store at base.
void launch_near_store_tc(cudaStream_t st, const NearArgs& a, const long long* base, const long long* fbase,
                          const int* ntri, int K, int KB, const double* store, float* out);
void launch_near_tc(cudaStream_t st, const NearArgs& a, int R, int NJ, int KB, const double* g0, const double* g1,
                    const long long* soff, const int* ntri, float* S, int ntask, const GemmTask* tasks,
                    const float* A, const long long* coff, double* C, int nsrc, int ntgt, const long long* base,
                    const double* store);
// Products from pre-split operands (tc_bulk.cu): A as tiles of 128 rows x
// 32 k (8192 floats: TF32 head then tail, canonical K-major layout; tile kt
// of a task at a_off + 8192 kt), B as tiles of BN columns x 32 k (64 BN
// floats; tile kt at b_off + 64 BN kt), zeros past the matrices;
// C[c_off + col ldc + row] = sum_k A[k][row] B[col][k] stored for row < M,
// col < N of the task's tile (rows row0.., columns col0..), K-tile sums in
// TC (float or double).
struct BulkTask {
  long long a_off, b_off, c_off;  // floats, floats, elements of C
  int M, N, nkt, row0, col0, ldc;
};
template <class TC>
void launch_tc_bulk(cudaStream_t st, int ntask, const BulkTask* tasks, const float* A, const float* B, TC* C,
                    int* err, int bn);
int split_variant();  // 1: pre-split operands where they fit (default), 0: FP32 operands
// The mixed replay of the stored near field from its split: the FP64 store
// as A tiles per leaf (row tile mt, K tile kt at tbase[i] + (mt nkt + kt)
// 8192, nkt = ceil(NJ ntri / 32)), written once; per call the densities as
// B tiles of 64 columns (column tile ct at sbase[i] + (ct nkt + kt) 4096;
// positions past R or K must hold zeros), the product (tasks per leaf, row
// tile and column tile; C at coff, ldc = KB x points, FP64 sums), the
// results ADDED to the outputs, the self pairs in FP64; ev (two events, or
// null) recorded around the product.
void launch_near_split_store(cudaStream_t st, const NearArgs& a, const long long* base, const long long* tbase,
                             const int* ntri, int K, int KB, const double* store, float* out);
void launch_near_split(cudaStream_t st, const NearArgs& a, int R, int NJ, int KB, const double* g0,
                       const double* g1, const long long* sbase, const int* ntri, float* S, int ntask,
                       const BulkTask* tasks, const float* A, const long long* coff, double* C, int nsrc, int ntgt,
                       const long long* base, const double* store, int* err, cudaEvent_t* ev = nullptr);
void launch_direct_all(cudaStream_t st, int ntri, const TriRec* trir, int nsrc, const double* src_pts,
                       int ntgt, const double* tgt_pts, int dosl, int dodl, int dostrain_src,
                       int dostrain_tgt, double rlam, double rmu, double* u_src, double* e_src,
                       double* u_tgt, double* e_tgt);

}  // namespace efmm
