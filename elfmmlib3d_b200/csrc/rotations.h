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

// Parity-split factored form (FP32 device pool, normalised basis): the frame
// change as Ry(-theta) Rz(-phi); Rz a 2 x 2 per order m, Ry and the shift
// along z re / im blocks per degree / order.  Per group at `base` (floats):
// Rz forward [4 (p+1)], Ry forward blocks n = 0..p, shift blocks m = 0..p,
// Ry back blocks n = 0..p, Rz back [4 (p+1)]; a block of r rows holds, per
// input row k, ceil(r/2) float4 (re[2j][k], im[2j][k], re[2j+1][k],
// im[2j+1][k]), then one zero column.
struct RotSOp {
  int p, pad;
  long long base;
};
long long rots_group_size(int p);
// The split pool of every group; w: normalisation per real row at the
// largest order (2 ncoef(pmax)).
void build_split_ops(const std::vector<int>& kinds, const std::vector<int>& orders,
                     const std::vector<double>& offsets, const std::vector<double>& w,
                     std::vector<RotSOp>& ops, std::vector<float>& pool);
// Whether the split kernel serves a launch whose largest operator size is maxdim.
bool rot_split_ok(int maxdim);

// M2L of the half-space kernel U in the parity-split form (FP32 normalised
// pool): per group the order, the leading dimension of its blocks (ncoef
// rounded up to 4), the offsets (floats) of its re and im blocks (row-major,
// shared by the groups with the same (rho, dz, order)) and of its Rz in /
// out tables (4 per order m).
struct USOp {
  int p, ld;
  long long re, im, rzi, rzo;
};
// orders[g] and offsets d[g] (box units, dz >= 0) of the U groups; w:
// normalisation per real row; *cross: the largest re / im coupling dropped
// (relative to the block's largest entry).
void build_usplit_ops(const std::vector<int>& orders, const std::vector<double>& offsets, const std::vector<double>& w,
                      std::vector<USOp>& ops, std::vector<float>& pool, double* cross);

struct TransTask;
struct TransPair;

// Apply the factored translations of ntask column tiles (task.col0 counts
// columns of the group's pairs x C; task.row0 unused) and ADD into dst.
template <class T>
void launch_translate_rot(cudaStream_t st, int ntask, const TransTask* tasks, const TransPair* pairs,
                          const RotOp* ops, const T* pool, int D, int C, int maxdim, const T* src, T* dst);

// The same translations from the split pool (FP32, orders <= 31), tasks cut
// for rot_split_cols() columns; variant <= 0: the default kernel variant.
void launch_translate_rot_split(cudaStream_t st, int ntask, const TransTask* tasks, const TransPair* pairs,
                                const RotSOp* ops, const float* pool, int D, int C, int maxdim, const float* src,
                                float* dst, int variant = 0);
// Columns per CTA of the split kernel.
int rot_split_cols();

// The U-kernel M2L in the parity-split form: tasks (group, first coefficient
// row, pair0, columns, first column) of 64 x 128 tiles (both parts), orders
// <= 63; ADDS into dst.
void launch_translate_us(cudaStream_t st, int ntask, const TransTask* tasks, const TransPair* pairs, const USOp* ops,
                         const float* pool, int D, int C, const float* src, float* dst);

// Columns per CTA of the factored kernel for a given largest operator size.
int rot_cols_per_cta(int maxdim, int elem_bytes);

// ---- the FP32 factored translations on the tensor cores (rot_tc.cu) ----
// A segment: the columns (npair x C) of one group's pairs.
struct RotTcSeg {
  int group, pair0, ncols, pad;
};
// A task: 32 consecutive columns of one segment (RTC_COLS).
struct RotTcTask {
  int seg, col0;
};
constexpr int RTC_COLS = 32;
// Per group: the order and, per stage (0 Fw, 1 Z, 2 Bk), the offset (floats)
// of its first block tile.  Block tiles follow in block order; a block of b
// rows has ceil8(b) operator rows and K = ceil8(b) input rows, split into K
// chunks of 32, each chunk the TF32 head then tail of the block's columns in
// the chunk, in the canonical K-major layout (ceil8(b) x Kc floats per part).
struct RotTcOp {
  int p, pad;
  long long tiles[3];
};
// Rows of block q of a stage at order p.
int rot_tc_rows(int stage, int p, int q);
// Shared memory of a launch whose groups have orders <= pmax.
size_t rot_tc_smem(int pmax);
// Operator tiles from the normalised FP32 pool in row-major block layout
// (groups of order > 31 get no tiles: their blocks exceed 64 rows).
void build_rot_tc_tiles(const std::vector<RotOp>& ops, const std::vector<float>& pool_rowmajor,
                        std::vector<RotTcOp>& tops, std::vector<float>& tiles);
// The three factors of ntask tasks (groups of order <= pmax <= 31): alpha x
// Bk Z Fw of each column of src is ADDED into its destination column of dst.
void launch_rot_tc(cudaStream_t st, int ntask, const RotTcTask* tasks, const RotTcSeg* segs, const TransPair* pairs,
                   const RotTcOp* ops, const float* tiles, int D, int C, int pmax, const float* src, float* dst,
                   int* err);

}  // namespace efmm
