// tree.cu -- adaptive oct-tree and interaction lists on the GPU.
//
// Reproduces the boxes, point orders and lists of the reference builder
// d3tstrcr (src/d3tstrcr.f:31, d3tallbem :1249, lists d3tlsts :702 / d3tlst31
// :919) for the same points:
//   * the root is the bounding cube of sources and targets (Mindlin variant:
//     centred on z = 0, side >= 2 max|z|, src/d3tstrcr_mindlin.f:1380);
//   * a box splits while it holds more than nbox sources or nbox targets;
//   * points are partitioned stably by z, then y, then x against the box
//     centre (coordinate > centre goes to the upper child), child digit
//     d = ix + 2 iy + 4 iz, empty children are skipped, boxes are numbered
//     breadth-first;
//   * box centres use the reference's floating-point expression (no FMA).
// One level at a time: every point gets the key (start of its box, digit), a
// stable radix sort reorders all points (points of boxes that do not split
// keep their place), and children are created from per-box digit counts.
// Lists: 5 (colleagues) and 2 from the parent's colleagues' children, 1 and 3
// from a depth-first walk below each leaf's colleagues, 4 as the dual of 3.
//
// Forest (no counterpart in the reference): many independent problems in one
// tree.  The caller places problem k in its own column of boxes of level L
// (grid position (i, j) of that level, all k) and gives the root cube; every
// box above level L splits, and boxes of different columns are never
// colleagues, so every list stays inside one problem and each problem sees
// the FMM of the subtree below its column.
#include <vector>
#include <algorithm>
#include "common.cuh"
#include "devbuf.h"
#include "sort.h"
#include "tree.h"

namespace efmm {

// reference box centre, src/d3tstrcr.f:1682 (d3tcentf) without contraction
__device__ __forceinline__ double centf(double c0, double size, double side, int i) {
  double x0 = __dsub_rn(c0, size / 2.0);
  double t = __dmul_rn((double)(i - 1), side);
  return __dadd_rn(__dadd_rn(x0, t), side / 2.0);
}

__global__ void k_bbox(int n, const double* __restrict__ p, double* out /* 6: mins, maxs */) {
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int c = 0; c < 3; c++) {
      double v = p[3 * (size_t)i + c];
      mn[c] = fmin(mn[c], v);
      mx[c] = fmax(mx[c], v);
    }
  for (int c = 0; c < 3; c++) {
    for (int o = 16; o > 0; o >>= 1) {
      mn[c] = fmin(mn[c], __shfl_xor_sync(0xffffffffu, mn[c], o));
      mx[c] = fmax(mx[c], __shfl_xor_sync(0xffffffffu, mx[c], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
    for (int c = 0; c < 3; c++) {
      // monotone integer images of doubles for atomic min/max
      unsigned long long* o = reinterpret_cast<unsigned long long*>(out);
      auto enc = [](double v) {
        unsigned long long b = __double_as_longlong(v);
        return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
      };
      atomicMin(o + c, enc(mn[c]));
      atomicMax(o + 3 + c, enc(mx[c]));
    }
  }
}

// every box of a level below `force` splits (the levels above a forest's
// problems), others while they hold more than nbox sources or targets
__global__ void k_split(int lo, int hi, int nbox, int force, const int* __restrict__ scount,
                        const int* __restrict__ tcount, int* __restrict__ split) {
  int b = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= hi) return;
  split[b - lo] = (force || scount[b] > nbox || tcount[b] > nbox) ? 1 : 0;
}

// digit + key for every point; counts per (split box, digit)
__global__ void k_digits(int n, const double* __restrict__ pts, const int* __restrict__ perm,
                         const int* __restrict__ pbox, const int* __restrict__ level, int lev,
                         int lo, const int* __restrict__ split, const int* __restrict__ ijk,
                         const int* __restrict__ bstart, double c0x, double c0y, double c0z,
                         double size, double side, unsigned long long* __restrict__ keys,
                         int* __restrict__ cnt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b = pbox[i];
  unsigned long long key = (unsigned long long)bstart[b] << 3;
  if (level[b] == lev && split[b - lo]) {
    int j = perm[i];
    double cx = centf(c0x, size, side, ijk[3 * b]);
    double cy = centf(c0y, size, side, ijk[3 * b + 1]);
    double cz = centf(c0z, size, side, ijk[3 * b + 2]);
    int ix = pts[3 * (size_t)j] > cx, iy = pts[3 * (size_t)j + 1] > cy, iz = pts[3 * (size_t)j + 2] > cz;
    int d = ix + 2 * iy + 4 * iz;
    key |= (unsigned long long)d;
    atomicAdd(&cnt[8 * (b - lo) + d], 1);
  }
  keys[i] = key;
}

__global__ void k_nchild(int nlev, const int* __restrict__ split, const int* __restrict__ cs,
                         const int* __restrict__ ct, int* __restrict__ nch) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nlev) return;
  int c = 0;
  if (split[k])
    for (int d = 0; d < 8; d++) c += (cs[8 * k + d] + ct[8 * k + d]) > 0;
  nch[k] = c;
}

__global__ void k_children(int lo, int hi, int lev, const int* __restrict__ split,
                           const int* __restrict__ cs, const int* __restrict__ ct,
                           const int* __restrict__ off, int* __restrict__ level, int* __restrict__ ijk,
                           int* __restrict__ parent, int* __restrict__ kids, int* __restrict__ nkids,
                           int* __restrict__ sstart, int* __restrict__ scount,
                           int* __restrict__ tstart, int* __restrict__ tcount) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  int b = lo + k;
  if (b >= hi || !split[k]) return;
  int id = hi + off[k];
  int s = sstart[b], t = tstart[b];
  int q = 0;
  for (int d = 0; d < 8; d++) {
    int a = cs[8 * k + d], c = ct[8 * k + d];
    if (a + c > 0) {
      int ch = id + q;
      level[ch] = lev + 1;
      ijk[3 * ch] = 2 * (ijk[3 * b] - 1) + 1 + (d & 1);
      ijk[3 * ch + 1] = 2 * (ijk[3 * b + 1] - 1) + 1 + ((d >> 1) & 1);
      ijk[3 * ch + 2] = 2 * (ijk[3 * b + 2] - 1) + 1 + ((d >> 2) & 1);
      parent[ch] = b;
      nkids[ch] = 0;
      for (int z = 0; z < 8; z++) kids[8 * ch + z] = -1;
      sstart[ch] = s;
      scount[ch] = a;
      tstart[ch] = t;
      tcount[ch] = c;
      kids[8 * b + q] = ch;
      q++;
    }
    s += a;
    t += c;
  }
  nkids[b] = q;
}

// point -> box for the new children (one warp per child)
__global__ void k_pbox(int lo, int hi, const int* __restrict__ start, const int* __restrict__ count,
                       int* __restrict__ pbox) {
  int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  int b = lo + w;
  if (b >= hi) return;
  int s = start[b], c = count[b];
  for (int i = lane; i < c; i += 32) pbox[s + i] = b;
}

// --------------------------------------------------------------------------
// lists
// --------------------------------------------------------------------------
// reference touch test d3tifint (src/d3tstrcr.f:1082) on box corners
__device__ __forceinline__ void box_corner(const double* c0, double size, int lev, const int* ijk,
                                           double* mn, double* mx) {
  double side = size / (double)(1ull << lev);
  for (int d = 0; d < 3; d++) {
    double c = centf(c0[d], size, side, ijk[d]);
    mn[d] = __dsub_rn(c, side / 2.0);
    mx[d] = __dadd_rn(mn[d], side);
  }
}
__device__ bool touch(const TreeDev& T, int a, int b) {
  double mn1[3], mx1[3], mn2[3], mx2[3];
  box_corner(T.c0, T.size, T.level[a], T.ijk + 3 * a, mn1, mx1);
  box_corner(T.c0, T.size, T.level[b], T.ijk + 3 * b, mn2, mx2);
  double eps = mx1[0] - mn1[0];
  eps = fmin(eps, mx2[0] - mn2[0]);
  eps = fmin(eps, mx2[1] - mn2[1]);
  eps = fmin(eps, mx2[2] - mn2[2]);
  eps = fmin(eps, mx1[1] - mn1[1]);
  eps = fmin(eps, mx1[2] - mn1[2]);
  eps = eps / 10000.0;
  for (int d = 0; d < 3; d++) {
    if (mn1[d] > mx2[d] + eps) return false;
    if (mn2[d] > mx1[d] + eps) return false;
  }
  return true;
}

// Problem of box b in a forest: its grid column (i, j) at level T.flev, -1
// above that level (boxes that hold several problems); 0 without a forest.
__device__ __forceinline__ int fcol(const TreeDev& T, int b) {
  if (T.flev < 0) return 0;
  const int l = T.level[b];
  if (l < T.flev) return -1;
  const int sh = l - T.flev;
  return ((T.ijk[3 * b] - 1) >> sh) + (((T.ijk[3 * b + 1] - 1) >> sh) << T.flev);
}

// lists 5 and 2 for boxes of one level.  coll: 27 slots per box.
// mode 0: count list-2 entries; mode 1: write them at l2_off.  In a forest,
// boxes of different problems are neither colleagues nor in list 2, and the
// boxes above the problems' level (colleagues among themselves, so that the
// level below finds its colleagues) have no list 2.
__global__ void k_list52(TreeDev T, int lo, int hi, int mode, int* __restrict__ l2cnt,
                         const int* __restrict__ l2off, int* __restrict__ l2items) {
  int b = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= hi) return;
  int dad = T.parent[b];
  int nc = 0, n2 = 0;
  int w = mode ? l2off[b] : 0;
  const int fb = fcol(T, b);
  for (int i = 0; i <= T.ncoll[dad]; i++) {
    int c = (i == 0) ? dad : T.coll[27 * dad + i - 1];
    for (int q = 0; q < T.nkids[c]; q++) {
      int kid = T.kids[8 * c + q];
      if (kid == b) continue;
      const int fk = fcol(T, kid);
      if (touch(T, kid, b)) {
        if (fk != fb) continue;
        if (mode == 0) T.coll[27 * b + nc] = kid;
        nc++;
      } else {
        if (fk != fb || fb < 0) continue;
        if (mode == 1) l2items[w + n2] = kid;
        n2++;
      }
    }
  }
  if (mode == 0) {
    T.ncoll[b] = nc;
    l2cnt[b] = n2;
  }
}

// d3tlst31: DFS below each colleague of a leaf.  mode 0 counts, mode 1 writes
// (ibox, jbox) pairs of list 1 (both directions when levels differ) and 3.
__global__ void k_list13(TreeDev T, int nb, int mode, int* __restrict__ c1, int* __restrict__ c3,
                         const int* __restrict__ o1, const int* __restrict__ o3,
                         int2* __restrict__ p1, int2* __restrict__ p3) {
  int ib = blockIdx.x * blockDim.x + threadIdx.x;
  if (ib >= nb) return;
  int n1 = 0, n3 = 0;
  int w1 = mode ? o1[ib] : 0, w3 = mode ? o3[ib] : 0;
  if (T.nkids[ib] == 0 && T.level[ib] != 0) {
    int stk_box[64], stk_n[64];
    for (int jj = 0; jj < T.ncoll[ib]; jj++) {
      int j0 = T.coll[27 * ib + jj];
      int is = 0, j = j0;
      stk_box[0] = j;
      stk_n[0] = T.nkids[j];
      for (int guard = 0; guard < (1 << 26); guard++) {
        if (!touch(T, ib, j)) {
          if (mode) p3[w3 + n3] = make_int2(ib, j);
          n3++;
          is--;
          stk_n[is]--;
          j = stk_box[is];
          continue;
        }
        if (T.nkids[j] == 0) {
          if (mode) p1[w1 + n1] = make_int2(ib, j);
          n1++;
          if (T.level[j] != T.level[ib]) {
            if (mode) p1[w1 + n1] = make_int2(j, ib);
            n1++;
          }
          if (j == j0) break;
          is--;
          stk_n[is]--;
          j = stk_box[is];
          continue;
        }
        int ns = stk_n[is];
        if (ns == 0) {
          if (j == j0) break;
          is--;
          stk_n[is]--;
          j = stk_box[is];
          continue;
        }
        j = T.kids[8 * j + ns - 1];
        is++;
        if (is >= 64) break;  // deeper than 64 levels below a colleague: cannot happen for < 64-level trees
        stk_box[is] = j;
        stk_n[is] = T.nkids[j];
      }
    }
  }
  if (mode == 0) {
    c1[ib] = n1;
    c3[ib] = n3;
  }
}

// --------------------------------------------------------------------------
// host orchestration
// --------------------------------------------------------------------------
template <class T>
static std::vector<T> to_host(const T* d, size_t n, cudaStream_t st) {
  std::vector<T> h(n);
  if (n) EFMM_CUDA_TRY(cudaMemcpyAsync(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, st));
  EFMM_CUDA_TRY(cudaStreamSynchronize(st));
  return h;
}

static void exclusive_scan(cudaStream_t st, const int* in, int* out, int n, DevBuf<char>& tmp) {
  if (n <= 0) return;
  const size_t bytes = scan_scratch_bytes(n);
  if (bytes > tmp.size()) tmp.resize(bytes);
  exclusive_scan_dev(st, in, out, n, tmp.get());
}

// stable sort of (key, value) pairs whose keys are below 2^bits (sort.cu)
static void sort_pairs(cudaStream_t st, const unsigned long long* kin, unsigned long long* kout, const int* vin,
                       int* vout, int n, const std::vector<int>& shifts, DevBuf<char>& tmp) {
  if (n <= 0) return;
  const size_t bytes = radix_scratch_bytes(n);
  if (bytes > tmp.size()) tmp.resize(bytes);
  radix_sort_pairs(st, kin, kout, vin, vout, n, shifts.data(), (int)shifts.size(), tmp.get());
}

// sort pairs (a, b) of box ids by (a, b) and build CSR over nb boxes
static void pairs_to_csr(cudaStream_t st, DevBuf<int2>& pairs, int np, int nb, DevBuf<int>& start,
                         DevBuf<int>& items, TreeScratch& S);

__global__ void k_pair_keys(int np, const int2* __restrict__ p, unsigned long long* __restrict__ k,
                            int* __restrict__ v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  k[i] = ((unsigned long long)(unsigned)p[i].x << 32) | (unsigned)p[i].y;
  v[i] = p[i].y;
}
__global__ void k_csr_count(int np, const unsigned long long* __restrict__ k, int* __restrict__ cnt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  atomicAdd(&cnt[(int)(k[i] >> 32)], 1);
}

static void pairs_to_csr(cudaStream_t st, DevBuf<int2>& pairs, int np, int nb, DevBuf<int>& start,
                         DevBuf<int>& items, TreeScratch& S) {
  DevBuf<unsigned long long>&k0 = S.k0, &k1 = S.k1;
  DevBuf<int>& v0 = S.v0;
  DevBuf<char>& tmp = S.tmp;
  k0.resize(np);
  k1.resize(np);
  v0.resize(np);
  items.resize(np);
  if (np > 0) {
    k_pair_keys<<<(np + 255) / 256, 256, 0, st>>>(np, pairs.get(), k0.get(), v0.get()); count_launch();
    // keys (a << 32) | b with a, b < nb: only the low digits of each word vary
    int nbits = 1;
    while ((1ll << nbits) < (long long)nb) nbits++;
    std::vector<int> shifts;
    for (int b = 0; b < nbits; b += 8) shifts.push_back(b);
    for (int b = 0; b < nbits; b += 8) shifts.push_back(32 + b);
    sort_pairs(st, k0.get(), k1.get(), v0.get(), items.get(), np, shifts, tmp);
  }
  DevBuf<int>& cnt = S.cnt;
  cnt.resize(nb + 1);
  cnt.zero(st);
  if (np > 0) { k_csr_count<<<(np + 255) / 256, 256, 0, st>>>(np, k1.get(), cnt.get()); count_launch(); }
  start.resize(nb + 1);
  exclusive_scan(st, cnt.get(), start.get(), nb + 1, tmp);
  EFMM_CUDA_TRY(cudaStreamSynchronize(st));
}

__global__ void k_l2_pairs(int nb, const int* __restrict__ off, const int* __restrict__ cnt,
                           const int* __restrict__ items, int2* __restrict__ pairs) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  for (int q = 0; q < cnt[b]; q++) pairs[off[b] + q] = make_int2(b, items[off[b] + q]);
}
__global__ void k_transpose_pairs(int np, const int2* __restrict__ in, int2* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  out[i] = make_int2(in[i].y, in[i].x);
}

// The reference's root (src/d3tstrcr.f:31 d3tstrcr, src/d3tstrcr_mindlin.f:
// 1380): centre and side of the bounding cube of sources and targets; the
// Mindlin variant centres it on z = 0 with side >= 2 max|z|.
static void bounding_root(cudaStream_t st, int n, const double* d_src, int nt, const double* d_tgt, int mindlin,
                          DevBuf<double>& bb, double* c0, double& size) {
  bb.resize(6);
  unsigned long long init[6];
  for (int c = 0; c < 3; c++) {
    init[c] = ~0ull;
    init[3 + c] = 0ull;
  }
  EFMM_CUDA_TRY(cudaMemcpyAsync(bb.get(), init, sizeof(init), cudaMemcpyHostToDevice, st));
  k_bbox<<<148, 256, 0, st>>>(n, d_src, bb.get()); count_launch();
  if (nt > 0) { k_bbox<<<148, 256, 0, st>>>(nt, d_tgt, bb.get()); count_launch(); }
  std::vector<unsigned long long> hb = to_host((unsigned long long*)bb.get(), 6, st);
  double mn[3], mx[3];
  for (int c = 0; c < 3; c++) {
    auto dec = [](unsigned long long b) {
      unsigned long long r = (b & 0x8000000000000000ull) ? (b & 0x7fffffffffffffffull) : ~b;
      double v;
      memcpy(&v, &r, 8);
      return v;
    };
    mn[c] = dec(hb[c]);
    mx[c] = dec(hb[3 + c]);
  }
  size = mx[0] - mn[0];
  const double sy = mx[1] - mn[1], sz = mx[2] - mn[2];
  if (sy > size) size = sy;
  if (sz > size) size = sz;
  for (int c = 0; c < 3; c++) c0[c] = (mn[c] + mx[c]) / 2;
  if (mindlin) {
    const double distz = fabs(mn[2]) > fabs(mx[2]) ? fabs(mn[2]) : fabs(mx[2]);
    c0[2] = 0.0;
    if (2 * distz > size) size = 2 * distz;
  }
}

int build_tree(cudaStream_t st, int n, const double* d_src, int nt, const double* d_tgt, int nbox,
               int mindlin, Tree& tr, const double* forest) {
  if (n < 1) return IER_BADARG;
  TreeScratch& S = tr.scr;
  DevBuf<char>& tmp = S.tmp;
  tr.n = n;
  tr.nt = nt;
  tr.flev = -1;
  double size = 0.0;
  if (forest) {
    if (!(forest[3] > 0.0) || forest[4] < 1.0 || forest[4] > 15.0) return IER_BADARG;
    for (int c = 0; c < 3; c++) tr.c0[c] = forest[c];
    size = forest[3];
    tr.flev = (int)forest[4];
  }
  // ---- root: the given cube of a forest, else the points' bounding cube
  if (!forest) bounding_root(st, n, d_src, nt, d_tgt, mindlin, S.bb, tr.c0, size);
  tr.size = size;

  // ---- boxes (grown per level)
  size_t cap = 1024;
  auto growall = [&](size_t m) {
    tr.level.grow(m, st);
    tr.ijk.grow(3 * m, st);
    tr.parent.grow(m, st);
    tr.kids.grow(8 * m, st);
    tr.nkids.grow(m, st);
    tr.sstart.grow(m, st);
    tr.scount.grow(m, st);
    tr.tstart.grow(m, st);
    tr.tcount.grow(m, st);
  };
  growall(cap);
  {
    int root_i[1] = {0}, root_ijk[3] = {1, 1, 1}, root_par[1] = {-1}, kids[8];
    for (int z = 0; z < 8; z++) kids[z] = -1;
    int zero = 0;
    EFMM_CUDA_TRY(cudaMemcpyAsync(tr.level.get(), root_i, 4, cudaMemcpyHostToDevice, st));
    EFMM_CUDA_TRY(cudaMemcpyAsync(tr.ijk.get(), root_ijk, 12, cudaMemcpyHostToDevice, st));
    EFMM_CUDA_TRY(cudaMemcpyAsync(tr.parent.get(), root_par, 4, cudaMemcpyHostToDevice, st));
    EFMM_CUDA_TRY(cudaMemcpyAsync(tr.kids.get(), kids, 32, cudaMemcpyHostToDevice, st));
    EFMM_CUDA_TRY(cudaMemcpyAsync(tr.nkids.get(), &zero, 4, cudaMemcpyHostToDevice, st));
    EFMM_CUDA_TRY(cudaMemcpyAsync(tr.sstart.get(), &zero, 4, cudaMemcpyHostToDevice, st));
    EFMM_CUDA_TRY(cudaMemcpyAsync(tr.scount.get(), &n, 4, cudaMemcpyHostToDevice, st));
    EFMM_CUDA_TRY(cudaMemcpyAsync(tr.tstart.get(), &zero, 4, cudaMemcpyHostToDevice, st));
    EFMM_CUDA_TRY(cudaMemcpyAsync(tr.tcount.get(), &nt, 4, cudaMemcpyHostToDevice, st));
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
  }
  // ---- points
  tr.iz.resize(n);
  tr.izt.resize(nt);
  {
    std::vector<int> id(std::max(n, nt));
    for (int i = 0; i < (int)id.size(); i++) id[i] = i;
    EFMM_CUDA_TRY(cudaMemcpyAsync(tr.iz.get(), id.data(), 4 * (size_t)n, cudaMemcpyHostToDevice, st));
    if (nt) EFMM_CUDA_TRY(cudaMemcpyAsync(tr.izt.get(), id.data(), 4 * (size_t)nt, cudaMemcpyHostToDevice, st));
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
  }
  DevBuf<int>&pbs = S.pbs, &pbt = S.pbt, &izs2 = S.izs2, &izt2 = S.izt2, &split = S.split, &cs = S.cs,
              &ct = S.ct, &nch = S.nch, &off = S.off;
  DevBuf<unsigned long long>&ks = S.ks, &ks2 = S.ks2, &kt = S.kt, &kt2 = S.kt2;
  pbs.resize(n);
  pbs.zero(st);
  pbt.resize(nt);
  pbt.zero(st);
  izs2.resize(n);
  izt2.resize(nt);
  ks.resize(n);
  ks2.resize(n);
  kt.resize(nt);
  kt2.resize(nt);
  int lo = 0, hi = 1, nlev = 0;
  tr.laddr.clear();
  tr.laddr.push_back({0, 1});
  // The reference allows 198 levels but its integer box indices overflow past
  // ~30; only more than nbox coincident points get that deep, so subdivision
  // stops at MAX_LEVELS (boxes at that level stay leaves).
  const int MAX_LEVELS = 50;
  for (int lev = 0; lev < MAX_LEVELS; lev++) {
    int nl = hi - lo;
    split.resize(nl);
    cs.resize(8 * (size_t)nl);
    ct.resize(8 * (size_t)nl);
    nch.resize(nl);
    off.resize(nl);
    cs.zero(st);
    ct.zero(st);
    k_split<<<(nl + 255) / 256, 256, 0, st>>>(lo, hi, nbox, lev < tr.flev ? 1 : 0, tr.scount.get(),
                                              tr.tcount.get(), split.get()); count_launch();
    double side = size / (double)(1ull << lev);
    k_digits<<<(n + 255) / 256, 256, 0, st>>>(n, d_src, tr.iz.get(), pbs.get(), tr.level.get(), lev, lo,
                                              split.get(), tr.ijk.get(), tr.sstart.get(), tr.c0[0],
                                              tr.c0[1], tr.c0[2], size, side, ks.get(), cs.get()); count_launch();
    if (nt > 0)
      k_digits<<<(nt + 255) / 256, 256, 0, st>>>(nt, d_tgt, tr.izt.get(), pbt.get(), tr.level.get(), lev,
                                                 lo, split.get(), tr.ijk.get(), tr.tstart.get(), tr.c0[0],
                                                 tr.c0[1], tr.c0[2], size, side, kt.get(), ct.get()); count_launch();
    k_nchild<<<(nl + 255) / 256, 256, 0, st>>>(nl, split.get(), cs.get(), ct.get(), nch.get()); count_launch();
    exclusive_scan(st, nch.get(), off.get(), nl, tmp);
    int last[2];
    EFMM_CUDA_TRY(cudaMemcpyAsync(&last[0], nch.get() + nl - 1, 4, cudaMemcpyDeviceToHost, st));
    EFMM_CUDA_TRY(cudaMemcpyAsync(&last[1], off.get() + nl - 1, 4, cudaMemcpyDeviceToHost, st));
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
    int nnew = last[0] + last[1];
    if (nnew == 0) break;
    // stable sort of the points by (box start, digit)
    int bits = 3;
    while ((1ll << (bits - 3)) <= (long long)std::max(n, nt) && bits < 64) bits++;
    {
      std::vector<int> shifts;
      for (int b = 0; b < bits; b += 8) shifts.push_back(b);
      sort_pairs(st, ks.get(), ks2.get(), tr.iz.get(), izs2.get(), n, shifts, tmp);
      tr.iz.swap(izs2);
      if (nt > 0) {
        sort_pairs(st, kt.get(), kt2.get(), tr.izt.get(), izt2.get(), nt, shifts, tmp);
        tr.izt.swap(izt2);
      }
    }
    if ((size_t)(hi + nnew) > tr.level.cap) growall(hi + nnew);
    else growall(hi + nnew);
    k_children<<<(nl + 127) / 128, 128, 0, st>>>(lo, hi, lev, split.get(), cs.get(), ct.get(), off.get(),
                                                 tr.level.get(), tr.ijk.get(), tr.parent.get(), tr.kids.get(),
                                                 tr.nkids.get(), tr.sstart.get(), tr.scount.get(),
                                                 tr.tstart.get(), tr.tcount.get()); count_launch();
    int nh = hi + nnew;
    k_pbox<<<(nnew * 32 + 255) / 256, 256, 0, st>>>(hi, nh, tr.sstart.get(), tr.scount.get(), pbs.get()); count_launch();
    if (nt > 0)
      k_pbox<<<(nnew * 32 + 255) / 256, 256, 0, st>>>(hi, nh, tr.tstart.get(), tr.tcount.get(), pbt.get()); count_launch();
    tr.laddr.push_back({hi, nnew});
    lo = hi;
    hi = nh;
    nlev = lev + 1;
  }
  tr.nboxes = hi;
  tr.nlev = nlev;
  EFMM_CUDA_TRY(cudaStreamSynchronize(st));
  return IER_OK;
}

int build_lists(cudaStream_t st, Tree& tr) {
  TreeScratch& S = tr.scr;
  DevBuf<char>& tmp = S.tmp;
  int nb = tr.nboxes;
  tr.coll.resize(27 * (size_t)nb);
  tr.ncoll.resize(nb);
  tr.ncoll.zero(st);
  DevBuf<int>&l2cnt = S.l2cnt, &l2off = S.l2off;
  l2cnt.resize(nb);
  l2cnt.zero(st);
  l2off.resize(nb + 1);
  TreeDev T = tr.dev();
  // lists 5 and 2, level by level (colleagues of the parent must exist)
  for (int lev = 1; lev <= tr.nlev; lev++) {
    int lo = tr.laddr[lev].first, cnt = tr.laddr[lev].second;
    k_list52<<<(cnt + 127) / 128, 128, 0, st>>>(T, lo, lo + cnt, 0, l2cnt.get(), nullptr, nullptr); count_launch();
  }
  exclusive_scan(st, l2cnt.get(), l2off.get(), nb, tmp);
  int tot2 = 0;
  {
    int a = 0, b = 0;
    EFMM_CUDA_TRY(cudaMemcpyAsync(&a, l2cnt.get() + nb - 1, 4, cudaMemcpyDeviceToHost, st));
    EFMM_CUDA_TRY(cudaMemcpyAsync(&b, l2off.get() + nb - 1, 4, cudaMemcpyDeviceToHost, st));
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
    tot2 = a + b;
  }
  DevBuf<int>& l2items = S.l2items;
  l2items.resize(tot2);
  for (int lev = 1; lev <= tr.nlev; lev++) {
    int lo = tr.laddr[lev].first, cnt = tr.laddr[lev].second;
    k_list52<<<(cnt + 127) / 128, 128, 0, st>>>(T, lo, lo + cnt, 1, nullptr, l2off.get(), l2items.get()); count_launch();
  }
  {
    DevBuf<int2>& pairs = S.pairs;
    pairs.resize(tot2);
    if (nb) { k_l2_pairs<<<(nb + 127) / 128, 128, 0, st>>>(nb, l2off.get(), l2cnt.get(), l2items.get(), pairs.get()); count_launch(); }
    pairs_to_csr(st, pairs, tot2, nb, tr.l2_start, tr.l2_items, S);
  }
  // lists 1 and 3
  DevBuf<int>&c1 = S.c1, &c3 = S.c3, &o1 = S.o1, &o3 = S.o3;
  c1.resize(nb);
  c3.resize(nb);
  o1.resize(nb + 1);
  o3.resize(nb + 1);
  k_list13<<<(nb + 127) / 128, 128, 0, st>>>(T, nb, 0, c1.get(), c3.get(), nullptr, nullptr, nullptr, nullptr); count_launch();
  exclusive_scan(st, c1.get(), o1.get(), nb, tmp);
  exclusive_scan(st, c3.get(), o3.get(), nb, tmp);
  int h[4];
  EFMM_CUDA_TRY(cudaMemcpyAsync(&h[0], c1.get() + nb - 1, 4, cudaMemcpyDeviceToHost, st));
  EFMM_CUDA_TRY(cudaMemcpyAsync(&h[1], o1.get() + nb - 1, 4, cudaMemcpyDeviceToHost, st));
  EFMM_CUDA_TRY(cudaMemcpyAsync(&h[2], c3.get() + nb - 1, 4, cudaMemcpyDeviceToHost, st));
  EFMM_CUDA_TRY(cudaMemcpyAsync(&h[3], o3.get() + nb - 1, 4, cudaMemcpyDeviceToHost, st));
  EFMM_CUDA_TRY(cudaStreamSynchronize(st));
  int tot1 = h[0] + h[1], tot3 = h[2] + h[3];
  DevBuf<int2>&p1 = S.p1, &p3 = S.p3, &p4 = S.p4;
  p1.resize(tot1);
  p3.resize(tot3);
  k_list13<<<(nb + 127) / 128, 128, 0, st>>>(T, nb, 1, nullptr, nullptr, o1.get(), o3.get(), p1.get(), p3.get()); count_launch();
  pairs_to_csr(st, p1, tot1, nb, tr.l1_start, tr.l1_items, S);
  p4.resize(tot3);
  if (tot3) { k_transpose_pairs<<<(tot3 + 255) / 256, 256, 0, st>>>(tot3, p3.get(), p4.get()); count_launch(); }
  pairs_to_csr(st, p3, tot3, nb, tr.l3_start, tr.l3_items, S);
  pairs_to_csr(st, p4, tot3, nb, tr.l4_start, tr.l4_items, S);
  EFMM_CUDA_TRY(cudaStreamSynchronize(st));
  return IER_OK;
}

}  // namespace efmm
