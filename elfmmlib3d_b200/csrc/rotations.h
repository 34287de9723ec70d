// rotations.h -- translations factored as rotation, shift along z, rotation
// back (internal header).
//
// A translation by offset d (M2L, M2M or L2L) equals
//   Bk(d) * Z(|d|) * Fw(d)
// with Fw rotating the input expansion into a frame whose z axis is along d,
// Z the same translation along z (block diagonal in the order m), and Bk the
// rotation back.  Rotations are block diagonal in the degree n, so the
// factored form costs O(p^3) per column instead of the O(p^4) of the dense
// per-offset operator; the reference translates the same way
// (src/l3dmplocfinal4.f:373-572, src/rotviarecur3.f:652-881).
#pragma once
#include <vector>
#include "devbuf.h"

namespace efmm {

// One factored operator: truncation order and offsets (elements) of its
// three parts in the pool.  Fw/Bk: degree blocks n = 0..p of (2n+2)^2,
// row-major, rows and columns in storage order within the degree.  Z: order
// blocks m = 0..p of (2(p-m+1))^2, rows and columns (n, m, re/im) for
// n = m..p.
struct RotOp {
  int p;
  long long fw, z, bk;
};

// Host construction of the factored operators of every translation group.
// kinds[g] (0 M2L, 1 M2M, 2 L2L), orders p[g] and offsets d[g] (box units as
// in the dense builder).  Pool in double, factorial basis.
void build_factored_ops(int pmax, const std::vector<int>& kinds, const std::vector<int>& orders,
                        const std::vector<double>& offsets, std::vector<RotOp>& ops,
                        std::vector<double>& pool);

// The same pool in the normalised basis (multipole coefficients x w, local
// coefficients / w, w[row] per real row), FP32.
void normalise_factored_ops(const std::vector<int>& kinds, const std::vector<RotOp>& ops,
                            const std::vector<double>& pool, const std::vector<double>& w,
                            std::vector<float>& out);

// Transpose every block in place (row-major -> column-major: the device
// layout).
void column_major_factored(const std::vector<RotOp>& ops, std::vector<double>& pool);

// Largest relative difference between the factored and the dense operators
// applied to random vectors, over the given groups (host computation).
double check_factored_ops(const std::vector<int>& kinds, const std::vector<int>& orders,
                          const std::vector<double>& offsets, const std::vector<RotOp>& ops,
                          const std::vector<double>& pool, int stride);

struct TransTask;
struct TransPair;

// Apply the factored translations of ntask column tiles (task.col0 counts
// columns of the group's pairs x C; task.row0 unused) and ADD into dst.
template <class T>
void launch_translate_rot(cudaStream_t st, int ntask, const TransTask* tasks, const TransPair* pairs,
                          const RotOp* ops, const T* pool, int D, int C, int maxdim, const T* src, T* dst);

// Columns per CTA of the factored kernel for a given largest operator size.
int rot_cols_per_cta(int maxdim, int elem_bytes);

// ---- the FP32 factored translations on the tensor cores (rot_tc.cu) ----
// A segment: the columns (npair x C) of one group's pairs, with the bases
// (floats) of its rows in the two intermediate arrays Y and W, laid out
// [row][column] (ncols per row).
struct RotTcSeg {
  int group, pair0, ncols, pad;
  long long ybase, wbase;
};
// A task: 128 consecutive columns of one segment.
struct RotTcTask {
  int seg, col0;
};
// Per group: the order and, per stage (0 Fw, 1 Z, 2 Bk), the offset (floats)
// of its first block tile; block tiles follow in block order, each the TF32
// head then tail of the block in the canonical K-major layout (ceil16(rows)
// x ceil8(rows) floats per part).
struct RotTcOp {
  int p, pad;
  long long tiles[3];
};
// Rows of block q of a stage at order p, and a stage's padded output rows
// (each block rounded up to a multiple of 8): the row count of Y (stage 0)
// and W (stage 1) per column.
int rot_tc_rows(int stage, int p, int q);
int rot_tc_pad_rows(int stage, int p);
size_t rot_tc_smem();
// Operator tiles from the normalised FP32 pool in row-major block layout
// (groups of order > 31 get no tiles: their blocks exceed 64 rows).
void build_rot_tc_tiles(const std::vector<RotOp>& ops, const std::vector<float>& pool_rowmajor,
                        std::vector<RotTcOp>& tops, std::vector<float>& tiles);
// One stage over ntask tasks: 0 reads the source expansions and writes Y,
// 1 reads Y and writes W, 2 reads W and adds alpha x the result into dst.
void launch_rot_tc(cudaStream_t st, int stage, int ntask, const RotTcTask* tasks, const RotTcSeg* segs,
                   const TransPair* pairs, const RotTcOp* ops, const float* tiles, int D, int C, const float* src,
                   float* ybuf, float* wbuf, float* dst, int* err);

}  // namespace efmm
