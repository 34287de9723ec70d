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

}  // namespace efmm
