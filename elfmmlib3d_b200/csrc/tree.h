// tree.h -- device oct-tree (internal header).
#pragma once
#include <vector>
#include <utility>
#include "devbuf.h"

namespace efmm {

// raw pointers for kernels
struct TreeDev {
  const int *level, *ijk, *parent, *kids, *nkids;
  const int *sstart, *scount, *tstart, *tcount;
  int *coll, *ncoll;
  double c0[3];
  double size;
  // forest of independent problems (flev >= 0): each column of boxes of
  // level flev (one (i, j) grid position, every k) holds one problem, and
  // only boxes of the same column below flev interact
  int flev;
};

// Device scratch of the tree and list builds, kept between builds so that a
// repeated set_geometry allocates nothing (cudaMalloc/cudaFree on every call
// stalled the host for up to a quarter second).
struct TreeScratch {
  DevBuf<char> tmp;
  DevBuf<double> bb;
  DevBuf<int> pbs, pbt, izs2, izt2, split, cs, ct, nch, off;
  DevBuf<unsigned long long> ks, ks2, kt, kt2, k0, k1;
  DevBuf<int> l2cnt, l2off, l2items, c1, c3, o1, o3, cnt, v0;
  DevBuf<int2> pairs, p1, p3, p4;
};

// Box ids are 0-based; ijk are the reference's 1-based grid indices; point
// ranges are 0-based offsets into the tree-ordered arrays; iz/izt map tree
// order -> user order (0-based).
struct Tree {
  int n = 0, nt = 0, nboxes = 0, nlev = 0;
  double c0[3] = {0, 0, 0}, size = 0;
  int flev = -1;  // forest level (TreeDev::flev), -1: one problem
  DevBuf<int> level, ijk, parent, kids, nkids, sstart, scount, tstart, tcount;
  DevBuf<int> iz, izt;
  std::vector<std::pair<int, int>> laddr;  // (first box, count) per level
  DevBuf<int> coll, ncoll;                 // list 5, 27 slots per box
  DevBuf<int> l1_start, l1_items, l2_start, l2_items, l3_start, l3_items, l4_start, l4_items;
  TreeScratch scr;

  TreeDev dev() const {
    TreeDev t;
    t.level = level.get(); t.ijk = ijk.get(); t.parent = parent.get(); t.kids = kids.get();
    t.nkids = nkids.get(); t.sstart = sstart.get(); t.scount = scount.get();
    t.tstart = tstart.get(); t.tcount = tcount.get(); t.coll = coll.get(); t.ncoll = ncoll.get();
    for (int c = 0; c < 3; c++) t.c0[c] = c0[c];
    t.size = size;
    t.flev = flev;
    return t;
  }
};

// forest (may be null): {c0x, c0y, c0z, size, level} -- the given root cube
// instead of the points' bounding cube, every box above `level` split, and
// the lists of build_lists restricted to the columns of that level.
int build_tree(cudaStream_t st, int n, const double* d_src, int nt, const double* d_tgt, int nbox,
               int mindlin, Tree& tr, const double* forest = nullptr);
int build_lists(cudaStream_t st, Tree& tr);

}  // namespace efmm
