// plan.cu -- host orchestration: geometry -> tree -> work lists -> kernels.
#include <algorithm>
#include <functional>
#include <cstdint>
#include <map>
#include <mutex>
#include <vector>
#include <cstring>
#include <cstdlib>
#include <atomic>
#include <chrono>
#include <cmath>
#include "plan.h"
#include "particles.h"
#include "halfspace.h"

namespace efmm {

static std::atomic<long long> g_launches{0};
long long launches_total() { return g_launches.load(); }

cudaError_t smem_raise_fn(const void* kern, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, int> limit;  // (device, kernel) -> limit set
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  int& cur = limit[std::make_pair(dev, kern)];
  if (bytes <= cur) return cudaSuccess;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}
void count_launch(int k) { g_launches += k; }

double iprec_eps(int iprec) {
  switch (iprec) {
    case -2: return 0.5;
    case -1: return 0.5e-1;
    case 0: return 0.5e-2;
    case 1: return 0.5e-3;
    case 2: return 0.5e-6;
    case 3: return 0.5e-9;
    case 4: return 0.5e-12;
    case 5: return 0.5e-15;
    default: return 0.0;
  }
}

int iprec_nbox(int iprec, int nsrc, int ntarg, bool iter) {
  int base;
  switch (iprec) {
    case -2: base = 8; break;
    case -1: base = 15; break;
    case 0: base = 30; break;
    case 1: base = 60; break;
    case 2: base = 120; break;
    case 3: base = 240; break;
    case 4: base = 480; break;
    case 5: base = 700; break;
    default: return nsrc + ntarg;
  }
  return iter ? 2 * base : base / 3;
}

// ------------------------------------------------------------ small kernels
__global__ void k_gather(int n, int w, const int* __restrict__ perm, const double* __restrict__ in,
                         double* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int j = perm[i];
  size_t r = (size_t)blockIdx.y * w * n;  // right-hand side blockIdx.y
  for (int c = 0; c < w; c++) out[r + (size_t)w * i + c] = in[r + (size_t)w * j + c];
}
// M2L pairs of list 2: pass 0 counts per operator group, pass 1 places
// (src box, dst box, 1/s) at the group's cursor
__global__ void k_m2l_pairs(int nb, int pass, const int* __restrict__ level, const int* __restrict__ ijk,
                            const int* __restrict__ scount, const int* __restrict__ tcount,
                            const int* __restrict__ l2s, const int* __restrict__ l2i, const int* __restrict__ m2lg,
                            double size, int* __restrict__ cnt, int* __restrict__ cursor,
                            TransPair* __restrict__ out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  if (level[b] < 2 || scount[b] + tcount[b] == 0) return;
  const double inv_s = (double)(1ull << level[b]) / size;
  for (int q = l2s[b]; q < l2s[b + 1]; q++) {
    const int sb = l2i[q];
    if (scount[sb] == 0) continue;
    const int di = ijk[3 * b] - ijk[3 * sb], dj = ijk[3 * b + 1] - ijk[3 * sb + 1],
              dk = ijk[3 * b + 2] - ijk[3 * sb + 2];
    if (di < -3 || di > 3 || dj < -3 || dj > 3 || dk < -3 || dk > 3) continue;  // not a list-2 offset
    const int g = m2lg[(di + 3) * 49 + (dj + 3) * 7 + (dk + 3)];
    if (g < 0) continue;
    if (pass == 0) {
      atomicAdd(&cnt[g], 1);
    } else {
      const int pos = atomicAdd(&cursor[g], 1);
      out[pos] = TransPair{sb, b, inv_s};
    }
  }
}

// user (R, n, 3) -> tree order, right-hand side innermost: out[(i*3+d)*R + r]
__global__ void k_gather_rhs(int n, int R, const int* __restrict__ perm, const double* __restrict__ in,
                             double* __restrict__ out) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * R) return;
  int i = (int)(idx / R), r = (int)(idx % R);
  int j = perm[i];
  const double* src = in + 3 * ((size_t)r * n + j);
  for (int d = 0; d < 3; d++) out[((size_t)i * 3 + d) * R + r] = src[d];
}
// tree order -> user order; strain 6 (xx yy zz xy xz yz) -> 3x3
__global__ void k_scatter_out(int n, const int* __restrict__ perm, const double* __restrict__ u,
                              const double* __restrict__ e, double* __restrict__ uo,
                              double* __restrict__ eo) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int j = perm[i];
  size_t r = (size_t)blockIdx.y * n;  // right-hand side blockIdx.y
  if (uo)
    for (int c = 0; c < 3; c++) uo[3 * (r + j) + c] = u[3 * (r + i) + c];
  if (eo) {
    const double* s = e + 6 * (r + i);
    double* o = eo + 9 * (r + j);
    o[0] = s[0]; o[4] = s[1]; o[8] = s[2];
    o[1] = o[3] = s[3];
    o[2] = o[6] = s[4];
    o[5] = o[7] = s[5];
  }
}
__global__ void k_sym6to9(int n, const double* __restrict__ e, double* __restrict__ eo) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* s = e + 6 * (size_t)i;
  double* o = eo + 9 * (size_t)i;
  o[0] = s[0]; o[4] = s[1]; o[8] = s[2];
  o[1] = o[3] = s[3];
  o[2] = o[6] = s[4];
  o[5] = o[7] = s[5];
}

__global__ void k_d2f(size_t n, const double* __restrict__ in, float* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}
// normalised single-precision local expansions -> FP64 factorial basis
__global__ void k_f2d_local(size_t n, int D, const double* __restrict__ w, const float* __restrict__ in,
                            double* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (double)in[i] * w[i % D];
}
// operator g in the normalised basis: rows scaled by (M2M) w or (M2L, L2L) 1/w,
// columns by (M2M, M2L) 1/w or (L2L) w
__global__ void k_ops_normalised(const int* __restrict__ kinds, const long long* __restrict__ off,
                                 const int* __restrict__ dims, const double* __restrict__ w,
                                 const double* __restrict__ mats, float* __restrict__ out) {
  const int g = blockIdx.x, kind = kinds[g], dim = dims[g];
  const double* A = mats + off[g];
  float* B = out + off[g];
  for (long long q = threadIdx.x; q < (long long)dim * dim; q += blockDim.x) {
    int i = (int)(q / dim), j = (int)(q % dim);
    double si = kind == 1 ? w[i] : 1.0 / w[i];
    double sj = kind == 2 ? w[j] : 1.0 / w[j];
    B[q] = (float)(A[q] * si * sj);
  }
}

template <class T>
static std::vector<T> d2h(const DevBuf<T>& b, size_t n, cudaStream_t st) {
  std::vector<T> h(n);
  if (n) EFMM_CUDA_TRY(cudaMemcpyAsync(h.data(), b.get(), n * sizeof(T), cudaMemcpyDeviceToHost, st));
  EFMM_CUDA_TRY(cudaStreamSynchronize(st));
  return h;
}
template <class T>
static void h2d(DevBuf<T>& b, const std::vector<T>& h, cudaStream_t st) {
  b.resize(h.size());
  if (!h.empty()) EFMM_CUDA_TRY(cudaMemcpyAsync(b.get(), h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
}

// --------------------------------------------------------------- op pools
static std::mutex g_ops_mu;
static std::map<std::pair<int, std::pair<int, long long>>, OpPool*> g_ops;  // (device, (p, eps bits))

void Plan::ensure_ops() {
  long long ebits;
  std::memcpy(&ebits, &eps_, 8);
  auto key = std::make_pair(dev_, std::make_pair(p_, ebits));
  std::lock_guard<std::mutex> lk(g_ops_mu);
  auto it = g_ops.find(key);
  if (it != g_ops.end()) {
    ops_ = it->second;
    return;
  }
  OpPool* P = new OpPool();
  P->p = p_;
  P->eps = eps_;
  std::vector<OpDesc> descs;
  long long off = 0;
  for (int q = 0; q < 343; q++) P->m2l_group[q] = -1;
  for (int i = -3; i <= 3; i++)
    for (int j = -3; j <= 3; j++)
      for (int k = -3; k <= 3; k++) {
        int mx = std::max(abs(i), std::max(abs(j), abs(k)));
        if (mx < 2) continue;
        int po = std::min(p_, m2l_order(eps_, i, j, k));
        OpDesc d;
        d.kind = 0;
        d.p = po;
        d.d[0] = i; d.d[1] = j; d.d[2] = k;
        d.off = off;
        int dim = 2 * ncoef(po);
        off += (long long)dim * dim;
        P->m2l_group[(i + 3) * 49 + (j + 3) * 7 + (k + 3)] = (int)descs.size();
        P->dims.push_back(dim);
        descs.push_back(d);
      }
  for (int kind = 1; kind <= 2; kind++)
    for (int dg = 0; dg < 8; dg++) {
      OpDesc d;
      d.kind = kind;
      d.p = p_;
      d.d[0] = ((dg & 1) ? 0.25 : -0.25);
      d.d[1] = (((dg >> 1) & 1) ? 0.25 : -0.25);
      d.d[2] = (((dg >> 2) & 1) ? 0.25 : -0.25);
      d.off = off;
      int dim = 2 * ncoef(p_);
      off += (long long)dim * dim;
      (kind == 1 ? P->m2m_group : P->l2l_group)[dg] = (int)descs.size();
      P->dims.push_back(dim);
      descs.push_back(d);
    }
  P->descs = descs;
  {
    std::vector<int> g(P->m2l_group, P->m2l_group + 343);
    h2d(P->m2lg_dev, g, st_);
  }
  P->mats.resize(off);
  DevBuf<OpDesc> dd;
  dd.resize(descs.size());
  EFMM_CUDA_TRY(cudaMemcpyAsync(dd.get(), descs.data(), descs.size() * sizeof(OpDesc),
                                cudaMemcpyHostToDevice, st_));
  launch_build_ops(st_, (int)descs.size(), dd.get(), P->mats.get(), p_);
  std::vector<long long> offs(descs.size());
  for (size_t i = 0; i < descs.size(); i++) offs[i] = descs[i].off;
  std::vector<int> kinds(descs.size());
  for (size_t i = 0; i < descs.size(); i++) kinds[i] = descs[i].kind;
  P->kinds.resize(kinds.size());
  EFMM_CUDA_TRY(cudaMemcpyAsync(P->kinds.get(), kinds.data(), kinds.size() * 4, cudaMemcpyHostToDevice, st_));
  std::vector<double> wn(2 * (size_t)ncoef(p_));
  for (int n = 0; n <= p_; n++)
    for (int m = 0; m <= n; m++)
      wn[2 * cidx(n, m)] = wn[2 * cidx(n, m) + 1] = std::exp(0.5 * (std::lgamma(n + m + 1.0) + std::lgamma(n - m + 1.0)));
  P->wnorm.resize(wn.size());
  EFMM_CUDA_TRY(cudaMemcpyAsync(P->wnorm.get(), wn.data(), wn.size() * 8, cudaMemcpyHostToDevice, st_));
  P->off.resize(offs.size());
  P->dim.resize(P->dims.size());
  EFMM_CUDA_TRY(cudaMemcpyAsync(P->off.get(), offs.data(), offs.size() * 8, cudaMemcpyHostToDevice, st_));
  EFMM_CUDA_TRY(cudaMemcpyAsync(P->dim.get(), P->dims.data(), P->dims.size() * 4, cudaMemcpyHostToDevice, st_));
  EFMM_CUDA_TRY(cudaStreamSynchronize(st_));
  g_ops[key] = P;
  ops_ = P;
}

// ------------------------------------------------------------------ plan
Plan::Plan(int device, cudaStream_t stream) : dev_(device), st_(stream) {
  const char* tr = getenv("ELFMM3D_TRANSLATIONS");  // "dense": per-offset dense operators
  factored_ = !(tr && strcmp(tr, "dense") == 0);
  const char* pm = getenv("ELFMM3D_P2M");  // "nodes": batched P2M as node-feature products
  p2m_unit_ = !(pm && strcmp(pm, "nodes") == 0);
  for (int i = 0; i < 10; i++) EFMM_CUDA_TRY(cudaEventCreate(&ev_[i]));
}
Plan::~Plan() {
  graph_reset();
  for (int i = 0; i < 10; i++) cudaEventDestroy(ev_[i]);
  for (cudaEvent_t e : pev_) cudaEventDestroy(e);
  for (cudaEvent_t e : nev_)
    if (e) cudaEventDestroy(e);
}

void Plan::product_begin() { npev_ = 0; }

void WaveSet::upload(const std::vector<int>& wl, const std::vector<long long>& o1, const std::vector<long long>& o2,
                     const std::vector<long long>& o3, const std::vector<GemmTask>& t, cudaStream_t st) {
  h2d(leaves, wl, st);
  h2d(off1, o1, st);
  h2d(off2, o2, st);
  h2d(off3, o3.empty() ? std::vector<long long>(1, 0) : o3, st);
  h2d(tasks, t, st);
  htasks = t;
  EFMM_CUDA_TRY(cudaStreamSynchronize(st));  // the host vectors may go away
}

template <class T>
void Plan::product_timed(int ntask, const std::vector<GemmTask>& tasks, long long t0, const GemmTask* dtasks,
                         const T* F, const T* W, T* C, int bn) {
  if (capturing_) {
    gemm_product<T>(st_, ntask, dtasks, F, W, C, bn);
    return;
  }
  if (npev_ + 2 > (int)pev_.size()) {
    cudaEvent_t a, b;
    EFMM_CUDA_TRY(cudaEventCreate(&a));
    EFMM_CUDA_TRY(cudaEventCreate(&b));
    pev_.push_back(a);
    pev_.push_back(b);
  }
  EFMM_CUDA_TRY(cudaEventRecord(pev_[npev_], st_));
  gemm_product<T>(st_, ntask, dtasks, F, W, C, bn);
  EFMM_CUDA_TRY(cudaEventRecord(pev_[npev_ + 1], st_));
  npev_ += 2;
  for (long long q = t0; q < t0 + ntask; q++) {
    const GemmTask& t = tasks[q];
    product_flops_ += 2.0 * std::min(128, t.M - t.row0) * std::min(128, t.N - t.col0) * (double)t.K;
  }
}

// after the pass's final synchronisation
// the near-field product of the last replay from the split store (events
// recorded outside graph capture): out[0] ms, out[1] the bytes its operands
// and results take (split store, split densities, FP64 products)
void Plan::near_stats(double* out) const {
  float ms = 0;
  if (near_timed_ && nev_[0] && cudaEventQuery(nev_[1]) == cudaSuccess) cudaEventElapsedTime(&ms, nev_[0], nev_[1]);
  out[0] = near_timed_ ? ms : 0.0;
  out[1] = near_timed_ ? near_bytes_ : 0.0;
}

void Plan::product_collect() {
  for (int i = 0; i + 1 < npev_; i += 2) {
    float ms = 0;
    cudaEventElapsedTime(&ms, pev_[i], pev_[i + 1]);
    product_ms_ += ms;
  }
  npev_ = 0;
}

int Plan::set_geometry(int n, const double* d_tri, const double* d_nrm, const double* d_src, int nt,
                       const double* d_tgt, int iprec, bool iter, bool mindlin) {
  if (n < 1 || nt < 0) return IER_BADARG;
  if (iprec < -2 || iprec > 6) return IER_BADARG;
  n_ = n;
  nt_ = nt;
  iprec_ = iprec;
  eps_ = iprec_eps(iprec);
  nbox_ = leaf_override_ > 0 ? leaf_override_ : iprec_nbox(iprec, n, nt, iter);
  p_ = eps_ > 0 ? order_for_eps(eps_, 1.5) : 0;
  eps_mixed_ = mixed_floor_ > 0 ? std::max(eps_, mixed_floor_) : eps_;
  p_mixed_ = eps_mixed_ > 0 ? std::min(p_, order_for_eps(eps_mixed_, 1.5)) : p_;
  // Expansion orders above 54 (iprec 5, eps 5e-16) exceed the P2M register
  // tiling; at that tolerance the near-field-only evaluation (one box) is used.
  if (p_ > 54) {
    p_ = 0;
    nbox_ = n + nt;
  }
  // no triangles: particles (points with dipole orientations d_nrm)
  points_ = d_tri == nullptr;
  tri_u_.resize(points_ ? 1 : 9 * (size_t)n);
  src_u_.resize(3 * (size_t)n);
  tgt_u_.resize(3 * (size_t)nt);
  if (!points_)
    EFMM_CUDA_TRY(cudaMemcpyAsync(tri_u_.get(), d_tri, 72 * (size_t)n, cudaMemcpyDeviceToDevice, st_));
  nu_u_.resize(3 * (size_t)n);
  if (points_) {
    if (d_nrm)
      EFMM_CUDA_TRY(cudaMemcpyAsync(nu_u_.get(), d_nrm, 24 * (size_t)n, cudaMemcpyDeviceToDevice, st_));
    else
      EFMM_CUDA_TRY(cudaMemsetAsync(nu_u_.get(), 0, 24 * (size_t)n, st_));
  }
  EFMM_CUDA_TRY(cudaMemcpyAsync(src_u_.get(), d_src, 24 * (size_t)n, cudaMemcpyDeviceToDevice, st_));
  if (nt) EFMM_CUDA_TRY(cudaMemcpyAsync(tgt_u_.get(), d_tgt, 24 * (size_t)nt, cudaMemcpyDeviceToDevice, st_));
  auto now = [&]() {
    EFMM_CUDA_TRY(cudaStreamSynchronize(st_));
    return std::chrono::steady_clock::now();
  };
  auto ms = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
    return (float)std::chrono::duration<double, std::milli>(b - a).count();
  };
  auto t0 = now();
  mindlin_ = mindlin;
  img_sched_ = false;
  p2m_waves_.clear();  // the leaf lists change with the geometry
  l2t_waves_.clear();
  graph_reset();
  if (forest_on_ && mindlin && forest_[2] != 0.0) return IER_BADARG;  // the Mindlin root is centred on z = 0
  int ier = build_tree(st_, n, d_src, nt, d_tgt, nbox_, mindlin ? 1 : 0, tr_, forest_on_ ? forest_ : nullptr);
  if (ier) return ier;
  auto t1 = now();
  ier = build_lists(st_, tr_);
  if (ier) return ier;
  auto t2 = now();
  tri_s_.resize(points_ ? 1 : 9 * (size_t)n);
  nrm_s_.resize(3 * (size_t)n);
  src_s_.resize(3 * (size_t)n);
  tgt_s_.resize(3 * (size_t)nt);
  if (!points_) {
    k_gather<<<(n + 255) / 256, 256, 0, st_>>>(n, 9, tr_.iz.get(), d_tri, tri_s_.get()); count_launch();
  }
  k_gather<<<(n + 255) / 256, 256, 0, st_>>>(n, 3, tr_.iz.get(), points_ ? nu_u_.get() : d_nrm, nrm_s_.get());
  count_launch();
  k_gather<<<(n + 255) / 256, 256, 0, st_>>>(n, 3, tr_.iz.get(), d_src, src_s_.get()); count_launch();
  if (nt) { k_gather<<<(nt + 255) / 256, 256, 0, st_>>>(nt, 3, tr_.izt.get(), d_tgt, tgt_s_.get()); count_launch(); }
  build_worklists();
  auto t3 = now();
  if (far_) ensure_ops();
  auto t4 = now();
  timings.geo_tree = ms(t0, t1);
  timings.geo_lists = ms(t1, t2);
  timings.geo_work = ms(t2, t3);
  timings.geo_ops = ms(t3, t4);
  return IER_OK;
}

void Plan::build_worklists() {
  // ELFMM3D_PROFILE_SETUP=1 prints the host time of each phase to stderr
  static const bool prof = getenv("ELFMM3D_PROFILE_SETUP") != nullptr;
  auto tp = std::chrono::steady_clock::now();
  auto mark = [&](const char* what) {
    if (!prof) return;
    auto t = std::chrono::steady_clock::now();
    fprintf(stderr, "build_worklists %-10s %8.2f ms\n", what, std::chrono::duration<double, std::milli>(t - tp).count());
    tp = t;
  };
  int nb = tr_.nboxes;
  auto level = d2h(tr_.level, nb, st_);
  auto ijk = d2h(tr_.ijk, 3 * (size_t)nb, st_);
  auto parent = d2h(tr_.parent, nb, st_);
  auto nkids = d2h(tr_.nkids, nb, st_);
  auto kids = d2h(tr_.kids, 8 * (size_t)nb, st_);
  auto scount = d2h(tr_.scount, nb, st_);
  auto tcount = d2h(tr_.tcount, nb, st_);
  auto csr = [&](const DevBuf<int>& s, const DevBuf<int>& it, std::vector<int>& hs, std::vector<int>& hi) {
    hs = d2h(s, nb + 1, st_);
    hi = d2h(it, hs[nb], st_);
  };
  std::vector<int> l1s, l1i, l2s, l2i, l3s, l3i, l4s, l4i;
  csr(tr_.l1_start, tr_.l1_items, l1s, l1i);
  csr(tr_.l2_start, tr_.l2_items, l2s, l2i);
  csr(tr_.l3_start, tr_.l3_items, l3s, l3i);
  csr(tr_.l4_start, tr_.l4_items, l4s, l4i);

  mark("d2h");
  // near field: per leaf with evaluation points, source boxes from
  // list1 U self U list3 U list4(ancestors-or-self)  (ITER pairing,
  // src/elfmm3dtria_iter_1.f:1188-1225, read from the target side)
  std::vector<int> nleaves, nstart, nitems;
  nstart.push_back(0);
  for (int b = 0; b < nb; b++) {
    if (nkids[b] != 0) continue;
    if (scount[b] + tcount[b] == 0) continue;
    size_t before = nitems.size();
    auto add = [&](int s) {
      if (scount[s] > 0) nitems.push_back(s);
    };
    for (int q = l1s[b]; q < l1s[b + 1]; q++) add(l1i[q]);
    add(b);
    for (int q = l3s[b]; q < l3s[b + 1]; q++) add(l3i[q]);
    for (int a = b; a >= 0; a = parent[a])
      for (int q = l4s[a]; q < l4s[a + 1]; q++) add(l4i[q]);
    if (nitems.size() == before) continue;
    nleaves.push_back(b);
    nstart.push_back((int)nitems.size());
  }
  near_sc_h_.clear();
  near_tc_h_.clear();
  near_ntri_h_.clear();
  for (size_t i = 0; i < nleaves.size(); i++) {
    int b = nleaves[i], nt = 0;
    for (int q = nstart[i]; q < nstart[i + 1]; q++) nt += scount[nitems[q]];
    near_sc_h_.push_back(scount[b]);
    near_tc_h_.push_back(tcount[b]);
    near_ntri_h_.push_back(nt);
  }
  h2d(near_ntri_, near_ntri_h_, st_);
  store_valid_ = false;
  store_gen_++;
  ntc_key_ = -1;
  chunk_key_ = -1;
  near_pairs_ = 0;
  {
    // count point pairs for the throughput model
    auto sst = d2h(tr_.sstart, nb, st_);
    for (size_t i = 0; i < nleaves.size(); i++) {
      int b = nleaves[i];
      long long ne = scount[b] + tcount[b];
      long long ns = 0;
      for (int q = nstart[i]; q < nstart[i + 1]; q++) ns += scount[nitems[q]];
      near_pairs_ += ne * ns;
    }
    (void)sst;
  }
  nnear_ = (int)nleaves.size();
  h2d(near_leaves_, nleaves, st_);
  h2d(near_start_, nstart, st_);
  h2d(near_items_, nitems, st_);

  mark("near");
  // far field
  far_ = (p_ > 0) && (tr_.nlev >= 2);
  std::vector<int> p2m, l2t;
  for (int b = 0; b < nb; b++) {
    if (nkids[b] != 0 || level[b] < 2) continue;
    if (scount[b] > 0) p2m.push_back(b);
    if (scount[b] + tcount[b] > 0) l2t.push_back(b);
  }
  if (p2m.empty()) far_ = false;
  np2m_ = (int)p2m.size();
  nl2t_ = (int)l2t.size();
  p2m_h_ = p2m;
  p2m_sc_h_.clear();
  for (int b : p2m) p2m_sc_h_.push_back(scount[b]);
  l2t_sc_h_.clear();
  l2t_tc_h_.clear();
  l2t_h_ = l2t;
  for (int b : l2t) {
    l2t_sc_h_.push_back(scount[b]);
    l2t_tc_h_.push_back(tcount[b]);
  }
  lchunk_key_ = -1;
  h2d(p2m_leaves_, p2m, st_);
  h2d(l2t_leaves_, l2t, st_);
  m2m_.clear();
  m2l_.clear();
  l2l_.clear();
  if (!far_) return;
  ensure_ops();
  const int* m2lg = ops_->m2l_group;
  const std::vector<int>& dims = ops_->dims;
  // group the pairs of one level by operator; one segment per group
  auto add_level = [&](std::vector<std::pair<int, TransPair>>& gp, std::vector<TransPair>& pairs,
                       TransSched& S) {
    // stable counting sort by operator group
    int ng = 0;
    for (auto& e : gp) ng = std::max(ng, e.first + 1);
    std::vector<int> cnt(ng + 1, 0);
    for (auto& e : gp) cnt[e.first + 1]++;
    for (int g = 0; g < ng; g++) cnt[g + 1] += cnt[g];
    size_t base = pairs.size();
    pairs.resize(base + gp.size());
    std::vector<int> pos(cnt.begin(), cnt.end() - 1);
    for (auto& e : gp) pairs[base + pos[e.first]++] = e.second;
    int s0 = (int)S.segs.size();
    for (int g = 0; g < ng; g++)
      if (cnt[g + 1] > cnt[g]) S.segs.push_back({g, (int)(base + cnt[g]), cnt[g + 1] - cnt[g]});
    S.lev.push_back({s0, (int)S.segs.size() - s0});
  };
  m2m_.clear();
  m2l_.clear();
  l2l_.clear();
  std::vector<TransPair> m2m_pairs, l2l_pairs, m2l_pairs;
  mark("far-leaves");
  // M2M bottom-up: children at level lev -> parents at lev-1 (parents >= 2)
  for (int lev = tr_.nlev; lev >= 3; lev--) {
    std::vector<std::pair<int, TransPair>> gp;
    int lo = tr_.laddr[lev].first, cnt = tr_.laddr[lev].second;
    for (int b = lo; b < lo + cnt; b++) {
      if (scount[b] == 0) continue;
      int P = parent[b];
      int dg = ((ijk[3 * b] - 1) & 1) + 2 * ((ijk[3 * b + 1] - 1) & 1) + 4 * ((ijk[3 * b + 2] - 1) & 1);
      gp.push_back({ops_->m2m_group[dg], TransPair{b, P, 1.0}});
    }
    add_level(gp, m2m_pairs, m2m_);
  }
  mark("m2m");
  // M2L: list 2 of every box at level >= 2, grouped by operator on the
  // device (count per group, then fill; order within a group is arbitrary)
  {
    DevBuf<int>& cnt = m2l_cnt_;
    cnt.resize(344);
    cnt.zero(st_);
    const int gb = (nb + 255) / 256;
    k_m2l_pairs<<<gb, 256, 0, st_>>>(nb, 0, tr_.level.get(), tr_.ijk.get(), tr_.scount.get(), tr_.tcount.get(),
                                     tr_.l2_start.get(), tr_.l2_items.get(), ops_->m2lg_dev.get(), tr_.size,
                                     cnt.get(), nullptr, nullptr); count_launch();
    std::vector<int> hc = d2h(cnt, 343, st_);
    std::vector<int> start(344, 0);
    for (int g = 0; g < 343; g++) start[g + 1] = start[g] + hc[g];
    const int tot = start[343];
    int s0 = (int)m2l_.segs.size();
    for (int g = 0; g < 343; g++)
      if (hc[g] > 0) m2l_.segs.push_back({g, start[g], hc[g]});
    m2l_.lev.push_back({s0, (int)m2l_.segs.size() - s0});
    h2d(m2l_cursor_, start, st_);
    m2l_.pairs.resize(std::max(tot, 1));
    k_m2l_pairs<<<gb, 256, 0, st_>>>(nb, 1, tr_.level.get(), tr_.ijk.get(), tr_.scount.get(), tr_.tcount.get(),
                                     tr_.l2_start.get(), tr_.l2_items.get(), ops_->m2lg_dev.get(), tr_.size,
                                     nullptr, m2l_cursor_.get(), m2l_.pairs.get()); count_launch();
    m2l_pairs_h_ = tot;
  }
  mark("m2l");
  // L2L top-down: parents at level lev (>= 2) -> children
  for (int lev = 2; lev < tr_.nlev; lev++) {
    std::vector<std::pair<int, TransPair>> gp;
    int lo = tr_.laddr[lev].first, cnt = tr_.laddr[lev].second;
    for (int b = lo; b < lo + cnt; b++) {
      for (int q = 0; q < nkids[b]; q++) {
        int k = kids[8 * b + q];
        if (scount[k] + tcount[k] == 0) continue;
        int dg = ((ijk[3 * k] - 1) & 1) + 2 * ((ijk[3 * k + 1] - 1) & 1) + 4 * ((ijk[3 * k + 2] - 1) & 1);
        gp.push_back({ops_->l2l_group[dg], TransPair{b, k, 1.0}});
      }
    }
    add_level(gp, l2l_pairs, l2l_);
  }
  mark("l2l");
  h2d(m2m_.pairs, m2m_pairs, st_);
  h2d(l2l_.pairs, l2l_pairs, st_);
  mark("upload");
  int D = 2 * ncoef(p_);
  mpole_.resize((size_t)nb * 4 * D);
  local_.resize((size_t)nb * 4 * D);
  EFMM_CUDA_TRY(cudaStreamSynchronize(st_));
}

void Plan::cut_tasks(TransSched& S, int C, const std::vector<int>* dimsp) {
  if (S.C == C && S.pool == ops_) return;
  std::vector<TransTask> tasks;
  S.lev_tasks.clear();
  const std::vector<int>& dims = dimsp ? *dimsp : ops_->dims;
  for (auto& r : S.lev) {
    int t0 = (int)tasks.size();
    for (int q = r.first; q < r.first + r.second; q++) {
      const TransSeg& g = S.segs[q];
      int ncols = g.npair * C, dim = dims[g.group];
      // row tiles innermost: the tasks of one column tile share their source columns
      for (int c0 = 0; c0 < ncols; c0 += 128)
        for (int r0 = 0; r0 < dim; r0 += 128) tasks.push_back({g.group, r0, g.pair0, ncols, c0});
    }
    S.lev_tasks.push_back({t0, (int)tasks.size() - t0});
  }
  h2d(S.tasks, tasks, st_);
  S.C = C;
  S.pool = ops_;
}

void Plan::cut_rot_tasks(TransSched& S, int C, int W) {
  if (S.rC == C && S.rW == W && S.rpool == ops_) return;
  std::vector<TransTask> tasks;
  S.lev_rtasks.clear();
  S.lev_rdim.clear();
  const std::vector<int>& dims = ops_->dims;
  for (auto& r : S.lev) {
    // within a level, one launch per operator size (shared memory per size)
    std::vector<int> segs;
    for (int q = r.first; q < r.first + r.second; q++) segs.push_back(q);
    std::stable_sort(segs.begin(), segs.end(),
                     [&](int a, int b) { return dims[S.segs[a].group] > dims[S.segs[b].group]; });
    size_t i = 0;
    while (i < segs.size()) {
      const int dim = dims[S.segs[segs[i]].group];
      int t0 = (int)tasks.size();
      for (; i < segs.size() && dims[S.segs[segs[i]].group] == dim; i++) {
        const TransSeg& g = S.segs[segs[i]];
        int ncols = g.npair * C;
        for (int c0 = 0; c0 < ncols; c0 += W) tasks.push_back({g.group, 0, g.pair0, ncols, c0});
      }
      S.lev_rtasks.push_back({t0, (int)tasks.size() - t0});
      S.lev_rdim.push_back(dim);
    }
  }
  h2d(S.rtasks, tasks, st_);
  S.rC = C;
  S.rW = W;
  S.rpool = ops_;
}

// factored operators of the pool: host construction once per (device, p, eps)
void Plan::ensure_factored(bool tc) {
  std::lock_guard<std::mutex> lk(g_ops_mu);
  OpPool* P = ops_;
  if (P->rot_ready && (!tc || P->rot_tc_ready)) return;
  std::vector<int> kinds, orders;
  std::vector<double> offs;
  for (const OpDesc& d : P->descs) {
    kinds.push_back(d.kind);
    orders.push_back(d.p);
    offs.insert(offs.end(), {d.d[0], d.d[1], d.d[2]});
  }
  std::vector<RotOp> rops;
  std::vector<double> pool;
  build_factored_ops(p_, kinds, orders, offs, rops, pool);
  std::vector<double> w(2 * (size_t)ncoef(p_));
  for (int n = 0; n <= p_; n++)
    for (int m = 0; m <= n; m++)
      w[2 * cidx(n, m)] = w[2 * cidx(n, m) + 1] =
          std::exp(0.5 * (std::lgamma(n + m + 1.0) + std::lgamma(n - m + 1.0)));
  std::vector<float> poolf;
  normalise_factored_ops(kinds, rops, pool, w, poolf);
  if (tc && !P->rot_tc_ready) {
    std::vector<RotTcOp> tops;
    std::vector<float> tiles;
    build_rot_tc_tiles(rops, poolf, tops, tiles);
    h2d(P->rot_tc_ops, tops, st_);
    h2d(P->rot_tc_tiles, tiles, st_);
    EFMM_CUDA_TRY(cudaStreamSynchronize(st_));
    P->rot_tc_ready = true;
    if (P->rot_ready) return;
  }
  // device layout: blocks column-major
  column_major_factored(rops, pool);
  {
    std::vector<double> tmp(poolf.begin(), poolf.end());
    column_major_factored(rops, tmp);
    for (size_t i = 0; i < tmp.size(); i++) poolf[i] = (float)tmp[i];
  }
  h2d(P->rot_ops, rops, st_);
  h2d(P->rot_d, pool, st_);
  h2d(P->rot_f, poolf, st_);
  EFMM_CUDA_TRY(cudaStreamSynchronize(st_));
  P->rot_ready = true;
}

// parity-split FP32 operators (rotations.cu build_split_ops), once per pool
void Plan::ensure_split() {
  std::lock_guard<std::mutex> lk(g_ops_mu);
  OpPool* P = ops_;
  if (P->rots_ready) return;
  std::vector<int> kinds, orders;
  std::vector<double> offs;
  for (const OpDesc& d : P->descs) {
    kinds.push_back(d.kind);
    orders.push_back(d.p);
    offs.insert(offs.end(), {d.d[0], d.d[1], d.d[2]});
  }
  std::vector<double> w(2 * (size_t)ncoef(p_));
  for (int n = 0; n <= p_; n++)
    for (int m = 0; m <= n; m++)
      w[2 * cidx(n, m)] = w[2 * cidx(n, m) + 1] =
          std::exp(0.5 * (std::lgamma(n + m + 1.0) + std::lgamma(n - m + 1.0)));
  std::vector<RotSOp> sops;
  std::vector<float> spool;
  build_split_ops(kinds, orders, offs, w, sops, spool);
  h2d(P->rots_ops, sops, st_);
  h2d(P->rots_f, spool, st_);
  EFMM_CUDA_TRY(cudaStreamSynchronize(st_));
  P->rots_ready = true;
}

// parity-split U-kernel M2L operators (rotations.cu build_usplit_ops), once
// per pool
void Plan::ensure_usplit() {
  ensure_uops();
  std::lock_guard<std::mutex> lk(g_ops_mu);
  OpPool* P = ops_;
  if (P->us_ready) return;
  std::vector<int> orders;
  std::vector<double> offs;
  for (const OpDesc& d : P->udescs) {
    orders.push_back(d.p);
    offs.insert(offs.end(), {d.d[0], d.d[1], d.d[2]});
  }
  std::vector<double> w(2 * (size_t)ncoef(p_));
  for (int n = 0; n <= p_; n++)
    for (int m = 0; m <= n; m++)
      w[2 * cidx(n, m)] = w[2 * cidx(n, m) + 1] =
          std::exp(0.5 * (std::lgamma(n + m + 1.0) + std::lgamma(n - m + 1.0)));
  std::vector<USOp> uops;
  std::vector<float> upool;
  double cross = 0;
  build_usplit_ops(orders, offs, w, uops, upool, &cross);
  h2d(P->us_ops, uops, st_);
  h2d(P->us_pool, upool, st_);
  EFMM_CUDA_TRY(cudaStreamSynchronize(st_));
  P->us_ready = true;
}

bool Plan::usplit_on() const {
  static const bool on = [] {
    const char* e = getenv("ELFMM3D_USPLIT");
    return !(e && e[0] == '0');
  }();
  return on && p_ <= 63;
}

// The U-kernel M2L (schedule m2lu_) in the parity-split form: per group 64 x
// 128 tiles of (coefficient rows, concatenated columns), both parts at once
void Plan::run_u_split(int C, const float* src, float* dst) {
  ensure_usplit();
  TransSched& S = m2lu_;
  if (S.uC != C || S.upool != ops_) {
    std::vector<TransTask> tasks;
    for (auto& r : S.lev)
      for (int q = r.first; q < r.first + r.second; q++) {
        const TransSeg& g = S.segs[q];
        const int ncols = g.npair * C, nc = ncoef(ops_->udescs[g.group].p);
        for (int c0 = 0; c0 < ncols; c0 += 128)
          for (int r0 = 0; r0 < nc; r0 += 64) tasks.push_back({g.group, r0, g.pair0, ncols, c0});
      }
    h2d(S.utasks, tasks, st_);
    S.untask = (int)tasks.size();
    S.uC = C;
    S.upool = ops_;
  }
  launch_translate_us(st_, S.untask, S.utasks.get(), S.pairs.get(), ops_->us_ops.get(), ops_->us_pool.get(),
                      2 * ncoef(p_), C, src, dst);
}

// The FP32 translations of orders <= 31 run in the parity-split form unless
// ELFMM3D_ROT_SPLIT=0 (then the full-block kernels of rotations.cu).
bool Plan::split_rot() const {
  static const bool on = [] {
    const char* e = getenv("ELFMM3D_ROT_SPLIT");
    return !(e && e[0] == '0');
  }();
  return on && factored_ && p_ <= 31;
}

// The tensor-core form serves the FP32 translations of pools of order <= 31
// (blocks of at most 64 rows); ELFMM3D_ROT_TC=0 keeps them on the CUDA cores.
bool Plan::rot_tc_usable() const {
  static const bool on = [] {
    const char* e = getenv("ELFMM3D_ROT_TC");
    return !(e && e[0] == '0');
  }();
  return on && factored_ && tc_enabled() && p_ <= 31;
}

void Plan::cut_tc_tasks(TransSched& S, int C, bool one_launch) {
  if (S.tcC == C && S.tcpool == ops_) return;
  std::vector<RotTcSeg> segs;
  std::vector<RotTcTask> tasks;
  S.tcb.clear();
  for (auto& r : S.lev) {
    if (S.tcb.empty() || !one_launch) S.tcb.push_back({(int)tasks.size(), 0, 0});
    TransSched::TcBatch& b = S.tcb.back();
    for (int q = r.first; q < r.first + r.second; q++) {
      const TransSeg& g = S.segs[q];
      const int pg = ops_->descs[g.group].p, ncols = g.npair * C;
      const int si = (int)segs.size();
      segs.push_back({g.group, g.pair0, ncols, 0});
      for (int c0 = 0; c0 < ncols; c0 += RTC_COLS) tasks.push_back({si, c0});
      b.pmax = std::max(b.pmax, pg);
    }
    b.ntask = (int)tasks.size() - b.task0;
  }
  h2d(S.tcsegs, segs, st_);
  h2d(S.tctasks, tasks, st_);
  S.tcC = C;
  S.tcpool = ops_;
}

// The FP32 translations of a schedule on the tensor cores (rot_tc.cu): one
// launch per level (M2M, L2L: a level's sources are the previous level's
// results), or one for all levels (M2L).
void Plan::run_translations_tc(TransSched& S, int C, const float* src, float* dst, bool one_launch) {
  ensure_factored(true);
  cut_tc_tasks(S, C, one_launch);
  const int D = 2 * ncoef(p_);
  int* err = tc_err_ptr();
  for (const auto& b : S.tcb)
    launch_rot_tc(st_, b.ntask, S.tctasks.get() + b.task0, S.tcsegs.get(), S.pairs.get(), ops_->rot_tc_ops.get(),
                  ops_->rot_tc_tiles.get(), D, C, b.pmax, src, dst, err);
}

// The engine of each FP32 translation stage for this pass: the tuner's pick
// for the key (stage, order, leaf capacity, columns, kind); a pass being
// captured into a graph takes the decided engine (or the tensor cores while
// undecided) and reports nothing.
void Plan::tune_begin(int kind, int C) {
  trans_tuning_ = !capturing_ && rot_tc_usable();
  for (int s = 0; s < 3; s++) {
    trans_key_[s] = TuneKey{s, ops_->p, nbox_, C, 1, kind};
    if (!rot_tc_usable())
      trans_cand_[s] = 1;
    else
      trans_cand_[s] = capturing_ ? tune_best(trans_key_[s], 0) : tune_pick(trans_key_[s], 2);
  }
}

void Plan::switch_precision(bool mixed) {
  if (capturing_ || last_mixed_ == (int)mixed) return;
  const bool had = last_mixed_ >= 0;
  last_mixed_ = mixed ? 1 : 0;
  if (!had) return;
  graph_reset();
  if (!mixed) {
    store_f_.release();
    store_s_.release();
    store_tc_gen_ = -1;
    mpole_f_.release();
    local_f_.release();
    img_mp_f_.release();
    img_lc_f_.release();
  } else {
    mpole_.release();
    local_.release();
    img_mp_.release();
    img_lc_.release();
  }
}

void Plan::tune_end() {
  if (!trans_tuning_) return;
  const float ms[3] = {timings.m2m, timings.m2l, timings.l2l};
  for (int s = 0; s < 3; s++) tune_report(trans_key_[s], 2, trans_cand_[s], ms[s]);
  trans_tuning_ = false;
}

template <class T>
void Plan::run_translations(TransSched& S, int C, const T* mats, const T* src, T* dst) {
  int D = 2 * ncoef(p_);
  if constexpr (sizeof(T) == 4) {
    const int stage = (&S == &m2l_ || &S == &m2lv_img_) ? 1 : ((&S == &l2l_ || &S == &l2l_img_ || &S == &l2l_img_u_) ? 2 : 0);
    if (rot_tc_usable() && trans_cand_[stage] == 0) {
      run_translations_tc(S, C, reinterpret_cast<const float*>(src), reinterpret_cast<float*>(dst), stage == 1);
      return;
    }
  }
  // factored form when its column tiles fit in shared memory
  // (the split kernel's tiles have rot_split_cols() columns; the split
  // serves every launch when it is on: p <= 31 bounds every group's order)
  const bool split = sizeof(T) == 4 && split_rot();
  const int W = split ? rot_split_cols() : rot_cols_per_cta(D, (int)sizeof(T));
  const size_t smem = sizeof(T) * 2 * (size_t)D * rot_cols_per_cta(D, (int)sizeof(T));
  if (factored_ && smem <= 227 * 1024) {
    ensure_factored();
    cut_rot_tasks(S, C, W);
    const T* pool = nullptr;
    if (sizeof(T) == 8)
      pool = reinterpret_cast<const T*>(ops_->rot_d.get());
    else
      pool = reinterpret_cast<const T*>(ops_->rot_f.get());
    if (split) ensure_split();
    for (size_t i = 0; i < S.lev_rtasks.size(); i++) {
      if (split && rot_split_ok(S.lev_rdim[i])) {
        launch_translate_rot_split(st_, S.lev_rtasks[i].second, S.rtasks.get() + S.lev_rtasks[i].first,
                                   S.pairs.get(), ops_->rots_ops.get(), ops_->rots_f.get(), D, C, S.lev_rdim[i],
                                   reinterpret_cast<const float*>(src), reinterpret_cast<float*>(dst));
        continue;
      }
      launch_translate_rot<T>(st_, S.lev_rtasks[i].second, S.rtasks.get() + S.lev_rtasks[i].first, S.pairs.get(),
                              ops_->rot_ops.get(), pool, D, C, S.lev_rdim[i], src, dst);
    }
    return;
  }
  cut_tasks(S, C);
  for (auto& r : S.lev_tasks)
    launch_translate<T>(st_, r.second, S.tasks.get() + r.first, S.pairs.get(), mats, ops_->off.get(),
                        ops_->dim.get(), D, C, src, dst);
}

// Size and place the stored near field for the layers / outputs in flags
// (bit 0 single layer, 1 double layer, 2 sources, 3 targets, 4 strain): K
// doubles per (point, triangle) pair, per leaf [point][near triangle][K].
int Plan::store_alloc(int flags, double rlam, double rmu) {
  const int nl = (flags & 1) + ((flags >> 1) & 1), dstr = (flags >> 4) & 1;
  const int do_src = (flags >> 2) & 1, do_tgt = (flags >> 3) & 1;
  const int K = nl * 3 * (3 + 6 * dstr);
  std::vector<long long> base(near_ntri_h_.size());
  long long tot = 0;
  for (size_t i = 0; i < near_ntri_h_.size(); i++) {
    base[i] = tot;
    long long nep = (do_src ? near_sc_h_[i] : 0) + (do_tgt ? near_tc_h_[i] : 0);
    tot += nep * near_ntri_h_[i] * K;
  }
  size_t freeb = 0, totb = 0;
  EFMM_CUDA_TRY(cudaMemGetInfo(&freeb, &totb));
  if ((double)tot * 8.0 > 0.9 * (double)freeb + (double)store_.cap * 8.0) return IER_ALLOC;
  store_.resize((size_t)tot);
  h2d(near_base_, base, st_);
  near_base_h_ = base;
  store_K_ = K;
  store_flags_ = flags;
  store_lam_ = rlam;
  store_mu_ = rmu;
  store_valid_ = false;
  store_gen_++;
  ntc_key_ = -1;
  return IER_OK;
}

// The FP32 product-layout copy of the stored near field (converted once per
// store; false: not enough memory, the tensor cores are off, or no store --
// the caller then replays the FP64 store).
bool Plan::near_tc_ready(const NearArgs& na) {
  if (!tc_enabled() || !store_valid_ || store_K_ <= 0) return false;
  const bool split_on = split_variant() != 0;
  if (store_tc_gen_ == store_gen_ && (near_req_ == (int)split_on || capturing_)) return true;
  if (capturing_) return false;
  near_req_ = split_on ? 1 : 0;
  const int KB0 = 3 + 6 * ((store_flags_ >> 4) & 1), NJ0 = store_K_ / KB0;
  const int dsrc = (store_flags_ >> 2) & 1, dtgt = (store_flags_ >> 3) & 1;
  NearArgs sa = na;
  sa.do_src = dsrc;
  sa.do_tgt = dtgt;
  ntc_key_ = -1;
  // the pre-split store where it fits (else, or with efmm_split_variant(0),
  // the FP32 copy)
  if (split_on) {
    const size_t nl = near_ntri_h_.size();
    tbase_h_.resize(nl);
    nkt_h_.resize(nl);
    long long tot = 0;
    for (size_t i = 0; i < nl; i++) {
      const long long M = (long long)KB0 * ((dsrc ? near_sc_h_[i] : 0) + (dtgt ? near_tc_h_[i] : 0));
      const long long KK = (long long)NJ0 * near_ntri_h_[i];
      tbase_h_[i] = tot;
      nkt_h_[i] = (int)((KK + 31) / 32);
      tot += ((M + 127) / 128) * nkt_h_[i] * 8192;
    }
    size_t freeb = 0, totb = 0;
    EFMM_CUDA_TRY(cudaMemGetInfo(&freeb, &totb));
    if ((double)tot * 4.0 <= 0.8 * (double)freeb + 4.0 * (double)(store_s_.cap + store_f_.cap)) {
      store_f_.release();
      h2d(tbase_, tbase_h_, st_);
      store_s_.resize((size_t)tot);
      launch_near_split_store(st_, sa, near_base_.get(), tbase_.get(), near_ntri_.get(), store_K_, KB0,
                              store_.get(), store_s_.get());
      near_split_ = true;
      store_tc_gen_ = store_gen_;
      return true;
    }
  }
  near_split_ = false;
  store_s_.release();
  fbase_h_.resize(near_ntri_h_.size());
  long long tot = 0;
  for (size_t i = 0; i < near_ntri_h_.size(); i++) {
    const long long M = (long long)KB0 * ((dsrc ? near_sc_h_[i] : 0) + (dtgt ? near_tc_h_[i] : 0));
    fbase_h_[i] = tot;
    tot += ((M + 3) & ~3LL) * NJ0 * near_ntri_h_[i];
  }
  size_t freeb = 0, totb = 0;
  EFMM_CUDA_TRY(cudaMemGetInfo(&freeb, &totb));
  if ((double)tot * 4.0 > 0.8 * (double)freeb + 4.0 * (double)store_f_.cap) return false;
  h2d(fbase_, fbase_h_, st_);
  store_f_.resize((size_t)tot);
  launch_near_store_tc(st_, sa, near_base_.get(), fbase_.get(), near_ntri_.get(), store_K_, KB0, store_.get(),
                       store_f_.get());
  store_tc_gen_ = store_gen_;
  return true;
}

// Mixed replay of the stored near field for R <= 128 right-hand sides: per
// leaf the product of its FP32 blocks (KB x points rows, NJ x near triangles
// columns) with its near densities, on the tensor cores with FP64 sums, and
// the self pairs in FP64; the per-leaf tasks are cut once per (R, store
// layout).
void Plan::near_tc(const NearArgs& na, int R, const double* g0, const double* g1, int n, int nt) {
  const int KB = 3 + 6 * ((store_flags_ >> 4) & 1), NJ = store_K_ / KB;
  const int do_src = (store_flags_ >> 2) & 1, do_tgt = (store_flags_ >> 3) & 1;
  if (near_split_) {
    // tasks per (leaf, 64-column tile, 128-row tile); the split densities of
    // a leaf at so (ceil(R / 64) x nkt tiles of 4096 floats, zero outside
    // the densities: cleared whenever the layout is made)
    const long long key = ((long long)R << 8) | store_flags_ | (1LL << 40);
    if (ntc_key_ != key) {
      std::vector<long long> so, co;
      std::vector<BulkTask> tasks;
      long long stot = 0, ctot = 0;
      const int nct = (R + 63) / 64;
      for (size_t i = 0; i < near_ntri_h_.size(); i++) {
        const long long nep = (do_src ? near_sc_h_[i] : 0) + (do_tgt ? near_tc_h_[i] : 0);
        const long long M = KB * nep, nkt = nkt_h_[i];
        so.push_back(stot);
        co.push_back(ctot);
        for (int ct = 0; ct < nct; ct++)
          for (long long mt = 0; mt * 128 < M; mt++)
            tasks.push_back({tbase_h_[i] + mt * nkt * 8192, stot + ct * nkt * 4096, ctot, (int)M, R, (int)nkt,
                             (int)(128 * mt), 64 * ct, (int)M});
        stot += nct * nkt * 4096;
        ctot += R * M;
      }
      h2d(ntc_soff_, so, st_);
      h2d(ntc_coff_, co, st_);
      h2d(nsp_tasks_, tasks, st_);
      ntc_scratch_.resize((size_t)stot);
      ntc_scratch_.zero(st_);
      EFMM_CUDA_TRY(cudaStreamSynchronize(st_));  // the host vectors go away
      ntc_ntask_ = (int)tasks.size();
      ntc_stot_ = stot;
      ntc_ctot_ = ctot;
      ntc_key_ = key;
    }
    ntc_cbuf_.resize((size_t)ntc_ctot_);
    near_timed_ = !capturing_;
    if (near_timed_)
      for (cudaEvent_t& e : nev_)
        if (!e) EFMM_CUDA_TRY(cudaEventCreate(&e));
    near_bytes_ = 4.0 * (double)store_s_.size() + 4.0 * (double)ntc_stot_ + 8.0 * (double)ntc_ctot_;
    launch_near_split(st_, na, R, NJ, KB, g0, g1, ntc_soff_.get(), near_ntri_.get(), ntc_scratch_.get(), ntc_ntask_,
                      nsp_tasks_.get(), store_s_.get(), ntc_coff_.get(), ntc_cbuf_.get(), n, nt, near_base_.get(),
                      store_.get(), tc_err_ptr(), near_timed_ ? nev_ : nullptr);
    return;
  }
  const long long key = ((long long)R << 8) | store_flags_;
  if (ntc_key_ != key) {
    std::vector<long long> so, co;
    std::vector<GemmTask> tasks;
    long long stot = 0, ctot = 0;
    for (size_t i = 0; i < near_ntri_h_.size(); i++) {
      const long long nep = (do_src ? near_sc_h_[i] : 0) + (do_tgt ? near_tc_h_[i] : 0);
      const long long M = KB * nep, K = (long long)NJ * near_ntri_h_[i], Kp = (K + 3) & ~3LL;
      so.push_back(stot);
      co.push_back(ctot);
      for (int c0 = 0; c0 < R; c0 += 128)
        for (long long r0 = 0; r0 < M; r0 += 128)
          tasks.push_back({fbase_h_[i], stot, ctot, (int)M, R, (int)K, (int)((M + 3) & ~3LL), (int)Kp, (int)M,
                           (int)r0, c0});
      stot += R * Kp;
      ctot += R * M;
    }
    h2d(ntc_soff_, so, st_);
    h2d(ntc_coff_, co, st_);
    h2d(ntc_tasks_, tasks, st_);
    EFMM_CUDA_TRY(cudaStreamSynchronize(st_));  // the host vectors go away
    ntc_ntask_ = (int)tasks.size();
    ntc_stot_ = stot;
    ntc_ctot_ = ctot;
    ntc_key_ = key;
  }
  ntc_scratch_.resize((size_t)ntc_stot_);
  ntc_cbuf_.resize((size_t)ntc_ctot_);
  launch_near_tc(st_, na, R, NJ, KB, g0, g1, ntc_soff_.get(), near_ntri_.get(), ntc_scratch_.get(), ntc_ntask_,
                 ntc_tasks_.get(), store_f_.get(), ntc_coff_.get(), ntc_cbuf_.get(), n, nt, near_base_.get(),
                 store_.get());
}

int Plan::evaluate(double rlam, double rmu, const double* d_ssl, const double* d_sdl, double* d_u_src,
                   double* d_e_src, double* d_u_tgt, double* d_e_tgt, int mode, bool do_far) {
  switch_precision(false);
  if (points_ && mode != 0) return IER_BADARG;  // particles: no stored near field
  int n = n_, nt = nt_;
  int dosl = d_ssl != nullptr, dodl = d_sdl != nullptr;
  int do_src = (d_u_src || d_e_src) ? 1 : 0, do_tgt = (nt > 0 && (d_u_tgt || d_e_tgt)) ? 1 : 0;
  int ds_src = d_e_src ? 1 : 0, ds_tgt = d_e_tgt ? 1 : 0;
  // stored operator layout: layers, evaluation point sets, strain rows
  const int flags = dosl | (dodl << 1) | (do_src << 2) | (do_tgt << 3) | ((ds_src || ds_tgt) << 4);
  if (mode == 2 && (!store_valid_ || flags != store_flags_ || rlam != store_lam_ || rmu != store_mu_))
    return IER_HANDLE;
  if (mode == 1) {
    const int ier = store_alloc(flags, rlam, rmu);
    if (ier) return ier;
  }
  long long launch0 = launches_total();
  EFMM_CUDA_TRY(cudaEventRecord(ev_[0], st_));
  ssl_s_.resize(3 * (size_t)n);
  sdl_s_.resize(3 * (size_t)n);
  if (dosl) { k_gather<<<(n + 255) / 256, 256, 0, st_>>>(n, 3, tr_.iz.get(), d_ssl, ssl_s_.get()); count_launch(); }
  if (dodl) { k_gather<<<(n + 255) / 256, 256, 0, st_>>>(n, 3, tr_.iz.get(), d_sdl, sdl_s_.get()); count_launch(); }
  u_s_.resize(3 * (size_t)n);
  e_s_.resize(6 * (size_t)n);
  ut_s_.resize(3 * (size_t)std::max(nt, 1));
  et_s_.resize(6 * (size_t)std::max(nt, 1));
  u_s_.zero(st_);
  e_s_.zero(st_);
  ut_s_.zero(st_);
  et_s_.zero(st_);
  double c1 = (rlam + rmu) / (rlam + 2 * rmu), c2 = rmu / (rlam + 2 * rmu);
  EFMM_CUDA_TRY(cudaEventRecord(ev_[1], st_));
  int D = 2 * ncoef(p_);
  if (far_ && do_far && (do_src || do_tgt)) {
    mpole_.resize((size_t)tr_.nboxes * 4 * D);
    local_.resize((size_t)tr_.nboxes * 4 * D);
    mpole_.zero(st_);
    local_.zero(st_);
    P2MArgs pa;
    pa.leaves = p2m_leaves_.get();
    pa.level = tr_.level.get(); pa.ijk = tr_.ijk.get();
    pa.sstart = tr_.sstart.get(); pa.scount = tr_.scount.get();
    for (int c = 0; c < 3; c++) pa.c0[c] = tr_.c0[c];
    pa.size = tr_.size;
    pa.flev = tr_.flev;
    pa.tri = tri_s_.get(); pa.nrm = nrm_s_.get(); pa.ssl = ssl_s_.get(); pa.sdl = sdl_s_.get();
    pa.dosl = dosl; pa.dodl = dodl; pa.p = p_;
    pa.c1 = c1; pa.c2 = c2; pa.inv2mu = 0.5 / rmu;
    pa.mpole = mpole_.get();
    pa.points = points_ ? 1 : 0;
    pa.pts = src_s_.get();
    launch_p2m(st_, np2m_, pa);
    EFMM_CUDA_TRY(cudaEventRecord(ev_[2], st_));
    run_translations(m2m_, 4, ops_->mats.get(), mpole_.get(), mpole_.get());
    EFMM_CUDA_TRY(cudaEventRecord(ev_[3], st_));
    run_translations(m2l_, 4, ops_->mats.get(), mpole_.get(), local_.get());
    EFMM_CUDA_TRY(cudaEventRecord(ev_[4], st_));
    run_translations(l2l_, 4, ops_->mats.get(), local_.get(), local_.get());
    EFMM_CUDA_TRY(cudaEventRecord(ev_[5], st_));
    L2TArgs la;
    la.leaves = l2t_leaves_.get();
    la.level = tr_.level.get(); la.ijk = tr_.ijk.get();
    la.sstart = tr_.sstart.get(); la.scount = tr_.scount.get();
    la.tstart = tr_.tstart.get(); la.tcount = tr_.tcount.get();
    for (int c = 0; c < 3; c++) la.c0[c] = tr_.c0[c];
    la.size = tr_.size;
    la.flev = tr_.flev;
    la.local = local_.get();
    la.src_pts = src_s_.get(); la.tgt_pts = tgt_s_.get();
    la.p = p_; la.do_src = do_src; la.do_tgt = do_tgt;
    la.dostrain_src = ds_src; la.dostrain_tgt = ds_tgt;
    la.c1 = c1;
    la.u_src = u_s_.get(); la.e_src = e_s_.get(); la.u_tgt = ut_s_.get(); la.e_tgt = et_s_.get();
    launch_l2t(st_, nl2t_, la);
  } else {
    for (int i = 2; i <= 5; i++) EFMM_CUDA_TRY(cudaEventRecord(ev_[i], st_));
  }
  EFMM_CUDA_TRY(cudaEventRecord(ev_[6], st_));
  // near field
  trir_.resize(n);
  if (mode != 2 && !points_)  // the stored operator replaces the triangle records
    launch_tri_prep(st_, n, tri_s_.get(), nullptr, ssl_s_.get(), sdl_s_.get(), dosl, dodl, trir_.get());
  NearArgs na;
  na.nleaf = nnear_;
  na.leaves = near_leaves_.get(); na.nb_start = near_start_.get(); na.nb_items = near_items_.get();
  na.box_src_start = tr_.sstart.get(); na.box_src_count = tr_.scount.get();
  na.box_tgt_start = tr_.tstart.get(); na.box_tgt_count = tr_.tcount.get();
  na.trir = trir_.get();
  na.src_pts = src_s_.get(); na.tgt_pts = tgt_s_.get();
  na.dosl = dosl; na.dodl = dodl; na.dostrain_src = ds_src; na.dostrain_tgt = ds_tgt;
  na.do_src = do_src; na.do_tgt = do_tgt;
  na.rlam = rlam; na.rmu = rmu;
  na.u_src = u_s_.get(); na.e_src = e_s_.get(); na.u_tgt = ut_s_.get(); na.e_tgt = et_s_.get();
  if (points_) {
    na.part_sl = dosl ? ssl_s_.get() : nullptr;
    na.part_dl = dodl ? sdl_s_.get() : nullptr;
    launch_near_points(st_, na, nrm_s_.get(), rlam, rmu);
  } else if (mode == 0) {
    launch_near_leaf(st_, na);
  } else {
    // stored operator rows carry displacement and (if any output wants it) strain
    NearArgs sa = na;
    sa.dostrain_src = sa.dostrain_tgt = (store_flags_ >> 4) & 1;
    if (mode == 1) {
      launch_near_store(st_, sa, near_base_.get(), near_ntri_.get(), store_K_, 1, store_.get());
      store_valid_ = true;
      store_gen_++;
    }
    NearArgs ra = na;  // outputs as requested by this call
    ra.dostrain_src = sa.dostrain_src;
    ra.dostrain_tgt = sa.dostrain_tgt;
    launch_near_replay(st_, ra, near_base_.get(), near_ntri_.get(), store_K_, 1, ssl_s_.get(), sdl_s_.get(),
                       store_.get());
  }
  EFMM_CUDA_TRY(cudaEventRecord(ev_[7], st_));
  if (do_src) {
    k_scatter_out<<<(n + 255) / 256, 256, 0, st_>>>(n, tr_.iz.get(), u_s_.get(), e_s_.get(), d_u_src, d_e_src); count_launch();
  }
  if (do_tgt) {
    k_scatter_out<<<(nt + 255) / 256, 256, 0, st_>>>(nt, tr_.izt.get(), ut_s_.get(), et_s_.get(), d_u_tgt, d_e_tgt); count_launch();
  }
  EFMM_CUDA_TRY(cudaEventRecord(ev_[8], st_));
  EFMM_CUDA_TRY(cudaGetLastError());
  EFMM_CUDA_TRY(cudaEventSynchronize(ev_[8]));
  cudaEventElapsedTime(&timings.total, ev_[0], ev_[8]);
  cudaEventElapsedTime(&timings.prep, ev_[0], ev_[1]);
  cudaEventElapsedTime(&timings.p2m, ev_[1], ev_[2]);
  cudaEventElapsedTime(&timings.m2m, ev_[2], ev_[3]);
  cudaEventElapsedTime(&timings.m2l, ev_[3], ev_[4]);
  cudaEventElapsedTime(&timings.l2l, ev_[4], ev_[5]);
  cudaEventElapsedTime(&timings.l2t, ev_[5], ev_[6]);
  cudaEventElapsedTime(&timings.near, ev_[6], ev_[7]);
  launches_ = (int)(launches_total() - launch0);
  return IER_OK;
}

void Plan::flops_per_column(double* f) const {
  for (int i = 0; i < 5; i++) f[i] = 0;
  if (!far_ || !ops_) return;
  const double D = 2.0 * ncoef(p_);
  const long long nodes = 12LL * n_;
  f[0] = 2.0 * D * 4.0 * (double)nodes;  // rows x (charge + 3 dipole) per node
  const TransSched* S[3] = {&m2m_, &m2l_, &l2l_};
  // flops of the form that runs: factored (two rotations and the shift along
  // z, each sum_{j=1}^{p+1} (2j)^2 multiply-adds) or dense (dim^2)
  const bool fact = factored_ && 2.0 * D * rot_cols_per_cta((int)D, 4) * 4 <= 227.0 * 1024;
  for (int k = 0; k < 3; k++)
    for (const TransSeg& g : S[k]->segs) {
      if (fact) {
        const double q = ops_->descs[g.group].p + 1;
        const double rs = 4.0 * q * (q + 1) * (2 * q + 1) / 6.0;
        f[1 + k] += 2.0 * 3.0 * rs * g.npair;
      } else {
        double dim = ops_->dims[g.group];
        f[1 + k] += 2.0 * dim * dim * g.npair;
      }
    }
  f[4] = 2.0 * D * 9.0 * (double)(n_ + nt_);  // 9 derivative sums per point
}

void Plan::set_mixed_floor(double eps) {
  mixed_floor_ = eps;
  eps_mixed_ = mixed_floor_ > 0 ? std::max(eps_, mixed_floor_) : eps_;
  p_mixed_ = eps_mixed_ > 0 ? std::min(p_, order_for_eps(eps_mixed_, 1.5)) : p_;
  graph_reset();  // a captured pass holds the previous orders
}

// The mixed form's orders for the duration of a mixed call: order p_mixed_
// and the operator pool of (p_mixed_, eps_mixed_) in place of the iprec
// ones (restored on exit); nothing changes when they coincide.
struct MixedOrders {
  Plan* P;
  int p0 = 0;
  double e0 = 0;
  OpPool* o0 = nullptr;
  bool on = false;
  MixedOrders(Plan* P_, bool mixed) : P(P_) {
    if (!mixed || !P->far_ || P->p_mixed_ >= P->p_) return;
    p0 = P->p_;
    e0 = P->eps_;
    o0 = P->ops_;
    on = true;
    P->p_ = P->p_mixed_;
    P->eps_ = P->eps_mixed_;
    P->ensure_ops();
  }
  ~MixedOrders() {
    if (!on) return;
    P->p_ = p0;
    P->eps_ = e0;
    P->ops_ = o0;
  }
};

void Plan::translation_flops(int R, bool mixed, double* f) {
  for (int i = 0; i < 3; i++) f[i] = 0;
  if (!far_) return;
  MixedOrders orders(this, mixed);
  ensure_ops();
  const double D = 2.0 * ncoef(p_);
  const bool fact = factored_ && 2.0 * D * rot_cols_per_cta((int)D, 4) * 4 <= 227.0 * 1024;
  // the parity-split form (FP32): per column two Ry of sum_n (n+1)^2 + n^2,
  // the shift's re and im blocks (none of order 0 im), two Rz of 4 per
  // coefficient of order m > 0 (1 for m = 0) multiply-adds
  const bool split = mixed && split_rot();
  auto s2 = [](double x) { return x * (x + 1) * (2 * x + 1) / 6.0; };
  auto add = [&](const TransSched& S, int k, double cols) {
    for (const TransSeg& g : S.segs) {
      const double q = ops_->descs[g.group].p + 1;
      if (fact && split && q <= 32) {
        const double ma = 2.0 * (s2(q) + s2(q - 1)) + 2.0 * s2(q) - q * q + 2.0 * (4.0 * (q * (q + 1) / 2 - q) + q);
        f[k] += 2.0 * ma * g.npair * cols;
      } else if (fact) {
        f[k] += 2.0 * 3.0 * (4.0 * q * (q + 1) * (2 * q + 1) / 6.0) * g.npair * cols;
      } else {
        const double dim = ops_->dims[g.group];
        f[k] += 2.0 * dim * dim * g.npair * cols;
      }
    }
  };
  if (!mindlin_) {
    add(m2m_, 0, 4.0 * R);
    add(m2l_, 1, 4.0 * R);
    add(l2l_, 2, 4.0 * R);
    return;
  }
  ensure_uops();
  add(m2m_, 0, 6.0 * R);
  add(m2m_u_, 0, 1.0 * R);
  add(m2lv_img_, 1, 6.0 * R);
  for (const TransSeg& g : m2lu_.segs) {
    if (mixed && usplit_on()) {  // re block ncoef^2, im block (ncoef - p - 1)^2, two Rz
      const double pg = ops_->udescs[g.group].p, nc = (pg + 1) * (pg + 2) / 2, ni = nc - pg - 1;
      f[1] += (2.0 * (nc * nc + ni * ni) + 16.0 * nc) * g.npair * R;
    } else {
      const double dim = ops_->udims[g.group];
      f[1] += 2.0 * dim * dim * g.npair * R;
    }
  }
  add(l2l_img_, 2, 6.0 * R);
  add(l2l_img_u_, 2, 1.0 * R);
}

int Plan::evaluate_batch(double rlam, double rmu, int R, const double* d_ssl, const double* d_sdl,
                         double* d_u_src, double* d_e_src, double* d_u_tgt, double* d_e_tgt, int precision,
                         int mode) {
  if (R < 1 || precision < 0 || precision > 1 || mode < 0 || mode > 2) return IER_BADARG;
  if (points_) return IER_BADARG;  // particles: the single-right-hand-side FP64 form only
  switch_precision(precision == 1);
  MixedOrders orders(this, precision == 1);
  // the mixed form's geometry-only features stay resident for passes that
  // repeat on the same geometry (store / replay, graph replays)
  resident_ = precision == 1 && (mode != 0 || graph_pass_);
  const int n = n_, nt = nt_;
  if (mode) {
    const int dosl = d_ssl != nullptr, dodl = d_sdl != nullptr;
    const int do_src = (d_u_src || d_e_src) ? 1 : 0, do_tgt = (nt > 0 && (d_u_tgt || d_e_tgt)) ? 1 : 0;
    const int flags = dosl | (dodl << 1) | (do_src << 2) | (do_tgt << 3) | ((d_e_src || d_e_tgt) ? 16 : 0);
    if (mode == 2 && (!store_valid_ || flags != store_flags_ || rlam != store_lam_ || rmu != store_mu_))
      return IER_HANDLE;
    if (mode == 1) {
      const int ier = store_alloc(flags, rlam, rmu);
      if (ier) return ier;
    }
  }
  const int D = 2 * ncoef(p_);
  const size_t nb = tr_.nboxes;
  // right-hand sides per pass: at most 64 (near-field kernel), and the
  // expansions (2 x boxes x 4 rc x D doubles) within half the free memory
  int Rc = std::min(R, 64);
  if (capturing_) {
    Rc = rc_last_;  // the warm pass before the capture sized the chunks
  } else if (far_) {
    size_t freeb = 0, totb = 0;
    EFMM_CUDA_TRY(cudaMemGetInfo(&freeb, &totb));
    double have = 0.5 * (double)freeb + 8.0 * (double)(mpole_.cap + local_.cap);
    while (Rc > 1 && 16.0 * nb * 4 * Rc * D > have) Rc /= 2;
  }
  rc_last_ = Rc;
  float tot = 0, near = 0, far = 0;
  product_ms_ = product_flops_ = 0;
  for (int r0 = 0; r0 < R; r0 += Rc) {
    const int rc = std::min(Rc, R - r0);
    int ier = batch_pass(rlam, rmu, rc, d_ssl ? d_ssl + 3 * (size_t)n * r0 : nullptr,
                         d_sdl ? d_sdl + 3 * (size_t)n * r0 : nullptr,
                         d_u_src ? d_u_src + 3 * (size_t)n * r0 : nullptr,
                         d_e_src ? d_e_src + 9 * (size_t)n * r0 : nullptr,
                         d_u_tgt ? d_u_tgt + 3 * (size_t)nt * r0 : nullptr,
                         d_e_tgt ? d_e_tgt + 9 * (size_t)nt * r0 : nullptr, precision == 1,
                         mode == 1 && r0 == 0 ? 1 : (mode ? 2 : 0));
    if (ier) return ier;
    tot += timings.total;
    near += timings.near;
    far += timings.p2m + timings.m2m + timings.m2l + timings.l2l + timings.l2t;
  }
  timings.total = tot;
  return IER_OK;
}

// Two-stage P2M over waves of leaves whose node features and weights fit a
// scratch budget (at most 8 GB or a quarter of the free memory).  The waves
// (leaves, offsets, product tasks) are built and uploaded once per column
// count and element type; later passes (and graph captures) only launch.
// Whether features of elems elements of esz bytes may stay resident: at
// most a third of the free memory (what the scratch already holds counts as
// free).
bool Plan::resident_fits(long long elems, size_t esz, size_t cap_bytes) {
  size_t freeb = 0, totb = 0;
  EFMM_CUDA_TRY(cudaMemGetInfo(&freeb, &totb));
  return (double)elems * (double)esz <= ((double)freeb + (double)cap_bytes) / 3.0;
}

template <class T>
void Plan::p2m_twostage(const P2MArgs& pa, int R, T* mpole) {
  const int D = 2 * ncoef(p_), C = 4 * R;
  WaveSet& W = p2m_waves_;
  const long long key = ((long long)p_ << 40) | ((long long)R << 8) | (sizeof(T) << 2) | 0;
  if (W.key != key) {
    size_t freeb = 0, totb = 0;
    EFMM_CUDA_TRY(cudaMemGetInfo(&freeb, &totb));
    const size_t budget =
        std::min<size_t>((size_t)8 << 30, freeb / 4 + p2m_scratch_.cap * sizeof(double)) / sizeof(T);
    W.clear();
    std::vector<int> wl;
    std::vector<long long> fo, wo, no;
    std::vector<GemmTask> tasks;
    size_t i = 0;
    const size_t nl = p2m_h_.size();
    while (i < nl) {
      WaveSet::Wave w{0, (long long)wl.size(), 0, (long long)tasks.size(), 0, 0, 0};
      long long used = 0, nodes = 0;
      while (i < nl) {
        const long long K = 48LL * p2m_sc_h_[i];
        const long long need = K * D + K * C;
        if (w.nwl > 0 && used + need > (long long)budget) break;
        wl.push_back((int)i);
        fo.push_back(used);
        wo.push_back(used + K * D);
        no.push_back(nodes);
        nodes += 12LL * p2m_sc_h_[i];
        const int box = p2m_h_[i];
        for (int c0 = 0; c0 < C; c0 += 128)
          for (int r0 = 0; r0 < D; r0 += 128)
            tasks.push_back({used, used + K * D, (long long)box * C * D, D, C, (int)K, D, (int)K, D, r0, c0});
        used += need;
        w.maxn = std::max(w.maxn, 12 * p2m_sc_h_[i]);
        w.nwl++;
        i++;
      }
      w.ntask = (int)(tasks.size() - w.t0);
      w.used = used;
      w.nodes = nodes;
      W.w.push_back(w);
    }
    W.upload(wl, fo, wo, no, tasks, st_);
    W.key = key;
  }
  size_t maxu = 1;
  long long maxnodes = 1;
  for (const auto& w : W.w) {
    maxu = std::max(maxu, (size_t)w.used);
    maxnodes = std::max(maxnodes, w.nodes);
  }
  p2m_scratch_.resize((maxu * sizeof(T) + sizeof(double) - 1) / sizeof(double));
  wave_nrec_.resize(8 * (size_t)maxnodes);
  T* scratch = reinterpret_cast<T*>(p2m_scratch_.get());
  for (const auto& w : W.w) {
    launch_p2m_twostage<T>(st_, pa, R, w.nwl, W.leaves.get() + w.wl0, W.off1.get() + w.wl0, W.off2.get() + w.wl0,
                           W.off3.get() + w.wl0, wave_nrec_.get(), w.maxn, scratch, scratch, w.ntask,
                           W.tasks.get() + w.t0, mpole, false);
    product_timed<T>(w.ntask, W.htasks, w.t0, W.tasks.get() + w.t0, scratch, scratch, mpole);
  }
}
template void Plan::p2m_twostage<double>(const P2MArgs&, int, double*);
template void Plan::p2m_twostage<float>(const P2MArgs&, int, float*);

// P2M factored through unit-density multipoles over waves of leaves (budget
// as in p2m_twostage): per leaf the unit multipoles H of its triangles
// ([kind][ns tn][D], nk kinds, ns = 3 or 6 density components: those of the
// layers present) and the densities S (R rows of ns tn rounded up to 4),
// then one product task per (leaf, kind, 128-row tile): K = ns tn, N = R
// (64-column tensor-core tiles when R <= 64).  Column layouts: the
// free-space plan writes columns 4 r + kind of 4R per box; the image plan
// columns kind R + r of 6R (kinds 0..5) and the U column at nb 6R D + box R D.
//
// The resident FP32 form from split operands: one wave of all leaves, per
// leaf the unit multipoles as split tiles (nk kinds x ceil(D / 128) row
// tiles x nkt = ceil(ns tn / 32) K tiles of 8192 floats, off1) and the
// densities as split tiles (ceil(R / 64) x nkt tiles of 4096 floats, off2);
// tasks per (leaf, kind, column tile, row tile) into the same expansion
// columns as the FP32 products.  The scratch is cleared when the layout is
// made (the tiles' padding stays zero).  False when it does not fit.
bool Plan::p2m_split_layout(WaveSet& W, int D, int R, int nk, int ns, bool image, long long key) {
  const long long nb = tr_.nboxes, nmt = (D + 127) / 128, nct = (R + 63) / 64;
  long long all = 0;
  for (size_t j = 0; j < p2m_h_.size(); j++) {
    const long long nkt = ((long long)ns * p2m_sc_h_[j] + 31) / 32;
    all += nk * nmt * nkt * 8192 + nct * nkt * 4096;
  }
  if (!resident_fits(all, sizeof(float), p2m_scratch_.cap * sizeof(double))) return false;
  W.clear();
  W.resident = true;
  W.split = true;
  std::vector<int> wl;
  std::vector<long long> ho, so;
  std::vector<BulkTask> tasks;
  WaveSet::Wave w{0, 0, 0, 0, 0, 0, 0};
  long long used = 0;
  double flops = 0;
  for (size_t i = 0; i < p2m_h_.size(); i++) {
    const int tn = p2m_sc_h_[i];
    const long long K = (long long)ns * tn, nkt = (K + 31) / 32;
    wl.push_back((int)i);
    ho.push_back(used);
    so.push_back(used + nk * nmt * nkt * 8192);
    const long long box = p2m_h_[i];
    for (int q = 0; q < nk; q++) {
      long long coff;
      int ldc;
      if (!image) {
        coff = box * 4 * R * D + (long long)q * D;
        ldc = 4 * D;
      } else if (q < 6) {
        coff = box * 6 * R * D + (long long)q * R * D;
        ldc = D;
      } else {
        coff = nb * 6 * R * D + box * R * D;
        ldc = D;
      }
      for (long long ct = 0; ct < nct; ct++)
        for (long long mt = 0; mt < nmt; mt++) {
          tasks.push_back({ho.back() + (q * nmt + mt) * nkt * 8192, so.back() + ct * nkt * 4096, coff, D, R, (int)nkt,
                           (int)(128 * mt), (int)(64 * ct), ldc});
          flops += 2.0 * std::min<long long>(128, D - 128 * mt) * std::min<long long>(64, R - 64 * ct) * (double)K;
        }
    }
    used += nk * nmt * nkt * 8192 + nct * nkt * 4096;
    w.maxn = std::max(w.maxn, tn);
    w.nwl++;
  }
  w.ntask = (int)tasks.size();
  w.used = used;
  if (w.nwl > 0) W.w.push_back(w);
  W.upload(wl, ho, so, {}, {}, st_);
  h2d(W.btasks, tasks, st_);
  W.bulk_flops = flops;
  p2m_scratch_.resize((std::max<long long>(used, 1) * sizeof(float) + sizeof(double) - 1) / sizeof(double));
  p2m_scratch_.zero(st_);
  EFMM_CUDA_TRY(cudaStreamSynchronize(st_));  // the host vectors go away
  W.key = key;
  return true;
}

// k_tc_bulk (FP32 sums) timed with the tensor-core products (product_ms,
// product_flops: the useful flops of the tasks, flops)
void Plan::bulk_timed(int ntask, double flops, const BulkTask* dtasks, const float* A, const float* B, float* C,
                      int bn) {
  if (capturing_) {
    launch_tc_bulk<float>(st_, ntask, dtasks, A, B, C, tc_err_ptr(), bn);
    return;
  }
  if (npev_ + 2 > (int)pev_.size()) {
    cudaEvent_t a, b;
    EFMM_CUDA_TRY(cudaEventCreate(&a));
    EFMM_CUDA_TRY(cudaEventCreate(&b));
    pev_.push_back(a);
    pev_.push_back(b);
  }
  EFMM_CUDA_TRY(cudaEventRecord(pev_[npev_], st_));
  launch_tc_bulk<float>(st_, ntask, dtasks, A, B, C, tc_err_ptr(), bn);
  EFMM_CUDA_TRY(cudaEventRecord(pev_[npev_ + 1], st_));
  npev_ += 2;
  product_flops_ += flops;
}

template <class T>
bool Plan::p2m_factored(const P2MArgs& pa, int R, T* mpole, bool image) {
  const int D = 2 * ncoef(p_), nk = image ? 7 : 4;
  const long long nb = tr_.nboxes;
  if (p2m_unit_smem(p_, sizeof(T) == 4) > (size_t)227 * 1024) return false;
  // density components carried: single layer 0..2, double layer 3..5
  const int sbase = pa.dosl ? 0 : 3, ns = (pa.dosl && pa.dodl) ? 6 : 3;
  WaveSet& W = p2m_waves_;
  const long long key = ((long long)p_ << 40) | ((long long)R << 12) | ((long long)ns << 8) | (sbase << 5) |
                        (sizeof(T) << 2) | (image ? 3 : 1) | ((long long)resident_ << 62);
  // FP32 and resident: the unit multipoles and densities as split tiles and
  // the bulk-copy product, where they fit
  if constexpr (sizeof(T) == 4) {
    if (resident_ && tc_enabled() && split_variant()) {
      const long long skey = key | (1LL << 61);
      if (W.key != skey && !p2m_split_layout(W, D, R, nk, ns, image, skey)) goto dense;
      const bool do_h = !W.feat_valid;
      for (const auto& w : W.w) {
        if (!launch_p2m_unit<T>(st_, pa, R, nk, w.nwl, w.maxn, W.leaves.get(), W.off1.get(), W.off2.get(), sbase,
                                ns, reinterpret_cast<T*>(p2m_scratch_.get()), reinterpret_cast<T*>(p2m_scratch_.get()),
                                do_h, true))
          return false;
        float* sc = reinterpret_cast<float*>(p2m_scratch_.get());
        bulk_timed(w.ntask, W.bulk_flops, W.btasks.get(), sc, sc, reinterpret_cast<float*>(mpole), 64);
      }
      W.feat_valid = true;
      return true;
    }
  }
dense:
  if (W.key != key) {
    size_t freeb = 0, totb = 0;
    EFMM_CUDA_TRY(cudaMemGetInfo(&freeb, &totb));
    size_t budget = std::min<size_t>((size_t)8 << 30, freeb / 4 + p2m_scratch_.cap * sizeof(double)) / sizeof(T);
    bool res = false;
    if (resident_) {
      long long all = 0;
      for (size_t j = 0; j < p2m_h_.size(); j++) {
        const long long K = (long long)ns * p2m_sc_h_[j];
        all += nk * K * D + R * ((K + 3) & ~3LL);
      }
      res = resident_fits(all, sizeof(T), p2m_scratch_.cap * sizeof(double));
      if (res) budget = (size_t)all;
    }
    W.clear();
    W.resident = res;
    std::vector<int> wl;
    std::vector<long long> ho, so;
    std::vector<GemmTask> tasks;
    size_t i = 0;
    const size_t nl = p2m_h_.size();
    while (i < nl) {
      WaveSet::Wave w{0, (long long)wl.size(), 0, (long long)tasks.size(), 0, 0, 0};
      long long used = 0;
      while (i < nl) {
        const int tn = p2m_sc_h_[i];
        const long long K = (long long)ns * tn, Kp = (K + 3) & ~3LL, hk = K * D;
        const long long need = nk * hk + R * Kp;
        if (w.nwl > 0 && used + need > (long long)budget) break;
        wl.push_back((int)i);
        ho.push_back(used);
        so.push_back(used + nk * hk);
        const long long box = p2m_h_[i];
        for (int q = 0; q < nk; q++) {
          long long coff;
          int ldc;
          if (!image) {
            coff = box * 4 * R * D + (long long)q * D;
            ldc = 4 * D;
          } else if (q < 6) {
            coff = box * 6 * R * D + (long long)q * R * D;
            ldc = D;
          } else {
            coff = nb * 6 * R * D + box * R * D;
            ldc = D;
          }
          for (int c0 = 0; c0 < R; c0 += 128)
            for (int r0 = 0; r0 < D; r0 += 128)
              tasks.push_back({used + q * hk, used + nk * hk, coff, D, R, (int)K, D, (int)Kp, ldc, r0, c0});
        }
        used += need;
        w.maxn = std::max(w.maxn, tn);
        w.nwl++;
        i++;
      }
      w.ntask = (int)(tasks.size() - w.t0);
      w.used = used;
      W.w.push_back(w);
    }
    W.upload(wl, ho, so, {}, tasks, st_);
    W.key = key;
  }
  size_t maxu = 1;
  for (const auto& w : W.w) maxu = std::max(maxu, (size_t)w.used);
  p2m_scratch_.resize((maxu * sizeof(T) + sizeof(double) - 1) / sizeof(double));
  T* scratch = reinterpret_cast<T*>(p2m_scratch_.get());
  const int bn = R <= 64 ? 64 : 128;
  const bool do_h = !(W.resident && W.feat_valid);
  for (const auto& w : W.w) {
    if (!launch_p2m_unit<T>(st_, pa, R, nk, w.nwl, w.maxn, W.leaves.get() + w.wl0, W.off1.get() + w.wl0,
                            W.off2.get() + w.wl0, sbase, ns, scratch, scratch, do_h))
      return false;
    product_timed<T>(w.ntask, W.htasks, w.t0, W.tasks.get() + w.t0, scratch, scratch, mpole, bn);
  }
  W.feat_valid = W.resident;
  return true;
}
template bool Plan::p2m_factored<double>(const P2MArgs&, int, double*, bool);
template bool Plan::p2m_factored<float>(const P2MArgs&, int, float*, bool);

// Two-stage L2T over waves of leaves whose functionals and sums fit a
// scratch budget (at most 8 GB or a quarter of the free memory).
// mixed: FP32 normalised locals (local_f_) against normalised functionals,
// the product on the tensor cores
// One resident wave of all L2T leaves from split operands: per leaf (P
// points) the functionals as split tiles (nmt = ceil(9P / 128) row tiles x
// nkt = ceil(D / 32) K tiles of 8192 floats, off1), the products S (C
// columns of l2t_ld(P), off2) and the local expansions as split tiles (nct
// = ceil(C / 128) column tiles x nkt, off3); tasks per (leaf, column tile,
// row tile).  The scratch is cleared when the layout is made (the tiles'
// padding stays zero).
bool Plan::l2t_split_layout(WaveSet& W, int D, int C, const std::vector<int>& Pl, long long key) {
  const long long nkt = (D + 31) / 32, nct = (C + 127) / 128;
  long long all = 0;
  for (int P : Pl)
    if (P > 0) all += ((9LL * P + 127) / 128) * nkt * 8192 + nct * nkt * 8192 + (long long)C * l2t_ld(P);
  if (!resident_fits(all, sizeof(float), l2t_scratch_.cap * sizeof(double))) return false;
  W.clear();
  W.resident = true;
  W.split = true;
  std::vector<int> wl;
  std::vector<long long> go, so, bo;
  std::vector<BulkTask> tasks;
  WaveSet::Wave w{0, 0, 0, 0, 0, 0, 0};
  long long used = 0;
  for (size_t i = 0; i < Pl.size(); i++) {
    const int P = Pl[i];
    if (P == 0) continue;
    const long long nmt = (9LL * P + 127) / 128, LD = l2t_ld(P);
    wl.push_back((int)i);
    go.push_back(used);
    so.push_back(used + nmt * nkt * 8192);
    bo.push_back(used + nmt * nkt * 8192 + C * LD);
    for (long long ct = 0; ct < nct; ct++)
      for (long long mt = 0; mt < nmt; mt++)
        tasks.push_back({go.back() + mt * nkt * 8192, bo.back() + ct * nkt * 8192, so.back(), 9 * P, C, (int)nkt,
                         (int)(128 * mt), (int)(128 * ct), (int)LD});
    used += nmt * nkt * 8192 + C * LD + nct * nkt * 8192;
    w.maxn = std::max(w.maxn, P);
    w.nwl++;
  }
  w.ntask = (int)tasks.size();
  w.used = used;
  if (w.nwl > 0) W.w.push_back(w);
  W.upload(wl, go, so, bo, {}, st_);
  h2d(W.btasks, tasks, st_);
  l2t_scratch_.resize((std::max<long long>(used, 1) * sizeof(float) + sizeof(double) - 1) / sizeof(double));
  l2t_scratch_.zero(st_);
  EFMM_CUDA_TRY(cudaStreamSynchronize(st_));  // the host vectors go away
  W.key = key;
  return true;
}

void Plan::l2t_split_run(const L2TArgs& la, int R, const float* local, bool image) {
  WaveSet& W = l2t_waves_;
  float* sc = reinterpret_cast<float*>(l2t_scratch_.get());
  for (const auto& w : W.w)
    launch_l2t_bulk(st_, la, R, w.nwl, W.leaves.get(), W.off1.get(), W.off2.get(), W.off3.get(), w.maxn, sc, w.ntask,
                    W.btasks.get(), local, (long long)tr_.nboxes, image, !W.feat_valid, tc_err_ptr());
  W.feat_valid = true;
}

void Plan::l2t_twostage(const L2TArgs& la0, int R, int do_src, int do_tgt, bool mixed) {
  const int D = 2 * ncoef(p_), C = 4 * R;
  L2TArgs la = la0;
  la.wnorm = mixed ? ops_->wnorm.get() : nullptr;
  const size_t esz = mixed ? sizeof(float) : sizeof(double);
  WaveSet& W = l2t_waves_;
  const long long key = ((long long)p_ << 40) | ((long long)R << 8) | (esz << 4) | (do_src << 3) | (do_tgt << 2) | 1 |
                        ((long long)resident_ << 62);
  // mixed and resident: split operands streamed by bulk copies, where they fit
  if (mixed && resident_ && tc_enabled() && split_variant()) {
    const long long skey = key | (1LL << 61);
    bool ok = W.key == skey;
    if (!ok) {
      std::vector<int> Pl(l2t_h_.size());
      for (size_t j = 0; j < Pl.size(); j++) Pl[j] = (do_src ? l2t_sc_h_[j] : 0) + (do_tgt ? l2t_tc_h_[j] : 0);
      ok = l2t_split_layout(W, D, C, Pl, skey);
    }
    if (ok) {
      l2t_split_run(la, R, local_f_.get(), false);
      return;
    }
  }
  if (W.key != key) {
    size_t freeb = 0, totb = 0;
    EFMM_CUDA_TRY(cudaMemGetInfo(&freeb, &totb));
    size_t budget = std::min<size_t>((size_t)8 << 30, freeb / 4 + l2t_scratch_.cap * sizeof(double)) / esz;
    bool res = false;
    if (resident_) {
      long long all = 0;
      for (size_t j = 0; j < l2t_h_.size(); j++) {
        const int P = (do_src ? l2t_sc_h_[j] : 0) + (do_tgt ? l2t_tc_h_[j] : 0);
        const long long LD = l2t_ld(P);
        all += (long long)D * LD + (long long)C * LD;
      }
      res = resident_fits(all, esz, l2t_scratch_.cap * sizeof(double));
      if (res) budget = (size_t)all;
    }
    W.clear();
    W.resident = res;
    std::vector<int> wl;
    std::vector<long long> go, so;
    std::vector<GemmTask> tasks;
    size_t i = 0;
    const size_t nl = l2t_h_.size();
    while (i < nl) {
      WaveSet::Wave w{0, (long long)wl.size(), 0, (long long)tasks.size(), 0, 0, 0};
      long long used = 0;
      while (i < nl) {
        const int P = (do_src ? l2t_sc_h_[i] : 0) + (do_tgt ? l2t_tc_h_[i] : 0);
        if (P == 0) {
          i++;
          continue;
        }
        const int LD = (int)l2t_ld(P);
        const long long need = (long long)D * LD + (long long)C * LD;
        if (w.nwl > 0 && used + need > (long long)budget) break;
        wl.push_back((int)i);
        go.push_back(used);
        so.push_back(used + (long long)D * LD);
        const int box = l2t_h_[i];
        for (int c0 = 0; c0 < C; c0 += 128)
          for (int r0 = 0; r0 < 9 * P; r0 += 128)
            tasks.push_back({used, (long long)box * C * D, used + (long long)D * LD, 9 * P, C, D, LD, D, LD, r0, c0});
        used += need;
        w.maxn = std::max(w.maxn, P);
        w.nwl++;
        i++;
      }
      if (w.nwl == 0) break;
      w.ntask = (int)(tasks.size() - w.t0);
      w.used = used;
      W.w.push_back(w);
    }
    W.upload(wl, go, so, {}, tasks, st_);
    W.key = key;
  }
  size_t maxu = 1;
  for (const auto& w : W.w) maxu = std::max(maxu, (size_t)w.used);
  l2t_scratch_.resize((maxu * esz + sizeof(double) - 1) / sizeof(double));
  const bool do_g = !(W.resident && W.feat_valid);
  for (const auto& w : W.w) {
    if (mixed) {
      float* sc = reinterpret_cast<float*>(l2t_scratch_.get());
      launch_l2t_twostage<float>(st_, la, R, w.nwl, W.leaves.get() + w.wl0, W.off1.get() + w.wl0,
                                 W.off2.get() + w.wl0, w.maxn, sc, sc, w.ntask, W.tasks.get() + w.t0,
                                 local_f_.get(), false, do_g);
    } else {
      launch_l2t_twostage<double>(st_, la, R, w.nwl, W.leaves.get() + w.wl0, W.off1.get() + w.wl0,
                                  W.off2.get() + w.wl0, w.maxn, l2t_scratch_.get(), l2t_scratch_.get(), w.ntask,
                                  W.tasks.get() + w.t0, local_.get(), false, do_g);
    }
  }
  W.feat_valid = W.resident;
}

int Plan::batch_pass(double rlam, double rmu, int R, const double* d_ssl, const double* d_sdl,
                     double* d_u_src, double* d_e_src, double* d_u_tgt, double* d_e_tgt, bool mixed, int mode) {
  const int n = n_, nt = nt_;
  const int dosl = d_ssl != nullptr, dodl = d_sdl != nullptr;
  const int do_src = (d_u_src || d_e_src) ? 1 : 0, do_tgt = (nt > 0 && (d_u_tgt || d_e_tgt)) ? 1 : 0;
  const int ds_src = d_e_src ? 1 : 0, ds_tgt = d_e_tgt ? 1 : 0;
  const int D = 2 * ncoef(p_);
  const size_t nb = tr_.nboxes;
  long long launch0 = launches_total();
  product_begin();
  rec(0);
  ssl_s_.resize(3 * (size_t)n * R);
  sdl_s_.resize(3 * (size_t)n * R);
  const int gb = (int)(((long long)n * R + 255) / 256);
  if (dosl) { k_gather_rhs<<<gb, 256, 0, st_>>>(n, R, tr_.iz.get(), d_ssl, ssl_s_.get()); count_launch(); }
  if (dodl) { k_gather_rhs<<<gb, 256, 0, st_>>>(n, R, tr_.iz.get(), d_sdl, sdl_s_.get()); count_launch(); }
  u_s_.resize(3 * (size_t)n * R);
  e_s_.resize(6 * (size_t)n * R);
  ut_s_.resize(3 * (size_t)std::max(nt, 1) * R);
  et_s_.resize(6 * (size_t)std::max(nt, 1) * R);
  u_s_.zero(st_);
  e_s_.zero(st_);
  ut_s_.zero(st_);
  et_s_.zero(st_);
  const double c1 = (rlam + rmu) / (rlam + 2 * rmu), c2 = rmu / (rlam + 2 * rmu);
  rec(1);
  const int C = 4 * R;
  if (far_ && (do_src || do_tgt)) {
    if (mixed) {
      std::lock_guard<std::mutex> lk(g_ops_mu);
      if (ops_->mats_f.size() != ops_->mats.size()) {
        ops_->mats_f.resize(ops_->mats.size());
        k_ops_normalised<<<(int)ops_->dims.size(), 256, 0, st_>>>(ops_->kinds.get(), ops_->off.get(),
                                                                  ops_->dim.get(), ops_->wnorm.get(),
                                                                  ops_->mats.get(), ops_->mats_f.get());
        count_launch();
        EFMM_CUDA_TRY(cudaStreamSynchronize(st_));
      }
      mpole_f_.resize(nb * C * D);
      local_f_.resize(nb * C * D);
      mpole_f_.zero(st_);
      local_f_.zero(st_);
    } else {
      mpole_.resize(nb * C * D);
      local_.resize(nb * C * D);
      mpole_.zero(st_);
      local_.zero(st_);
    }
    P2MArgs pa;
    pa.leaves = p2m_leaves_.get();
    pa.level = tr_.level.get(); pa.ijk = tr_.ijk.get();
    pa.sstart = tr_.sstart.get(); pa.scount = tr_.scount.get();
    for (int c = 0; c < 3; c++) pa.c0[c] = tr_.c0[c];
    pa.size = tr_.size;
    pa.flev = tr_.flev;
    pa.tri = tri_s_.get(); pa.nrm = nrm_s_.get(); pa.ssl = ssl_s_.get(); pa.sdl = sdl_s_.get();
    pa.dosl = dosl; pa.dodl = dodl; pa.p = p_;
    pa.c1 = c1; pa.c2 = c2; pa.inv2mu = 0.5 / rmu;
    pa.mpole = mpole_.get();
    pa.C = C; pa.rstride = 1; pa.tstride = 3 * (long long)R; pa.dstride = R;
    if (mixed) {
      pa.wnorm = ops_->wnorm.get();  // multipoles in the normalised basis
      tune_begin(0, C);
      if (!(p2m_unit_ && p2m_factored<float>(pa, R, mpole_f_.get(), false)))
        p2m_twostage<float>(pa, R, mpole_f_.get());
      rec(2);
      run_translations(m2m_, C, ops_->mats_f.get(), mpole_f_.get(), mpole_f_.get());
      rec(3);
      run_translations(m2l_, C, ops_->mats_f.get(), mpole_f_.get(), local_f_.get());
      rec(4);
      run_translations(l2l_, C, ops_->mats_f.get(), local_f_.get(), local_f_.get());
    } else {
      // product form once the columns fill its tiles
      if (C < 32)
        launch_p2m(st_, np2m_, pa, R);
      else if (!(p2m_unit_ && p2m_factored<double>(pa, R, mpole_.get(), false)))
        p2m_twostage<double>(pa, R, mpole_.get());
      rec(2);
      run_translations(m2m_, C, ops_->mats.get(), mpole_.get(), mpole_.get());
      rec(3);
      run_translations(m2l_, C, ops_->mats.get(), mpole_.get(), local_.get());
      rec(4);
      run_translations(l2l_, C, ops_->mats.get(), local_.get(), local_.get());
    }
    rec(5);
    L2TArgs la;
    la.leaves = l2t_leaves_.get();
    la.level = tr_.level.get(); la.ijk = tr_.ijk.get();
    la.sstart = tr_.sstart.get(); la.scount = tr_.scount.get();
    la.tstart = tr_.tstart.get(); la.tcount = tr_.tcount.get();
    for (int c = 0; c < 3; c++) la.c0[c] = tr_.c0[c];
    la.size = tr_.size;
    la.flev = tr_.flev;
    la.local = local_.get();
    la.src_pts = src_s_.get(); la.tgt_pts = tgt_s_.get();
    la.p = p_; la.do_src = do_src; la.do_tgt = do_tgt;
    la.dostrain_src = ds_src; la.dostrain_tgt = ds_tgt;
    la.c1 = c1;
    la.u_src = u_s_.get(); la.e_src = e_s_.get(); la.u_tgt = ut_s_.get(); la.e_tgt = et_s_.get();
    la.C = C; la.nsrc = n; la.ntgt = nt;
    // two-stage product form once the columns fill its tiles
    bool done = false;
    if (C >= 32) {
      l2t_twostage(la, R, do_src, do_tgt, mixed);
      done = true;
    }
    if (!done && C >= 32) {
      const int key = do_src | (do_tgt << 1);
      if (lchunk_key_ != key) {
        std::vector<int> cl, ce;
        for (size_t i = 0; i < l2t_sc_h_.size(); i++) {
          int nep = (do_src ? l2t_sc_h_[i] : 0) + (do_tgt ? l2t_tc_h_[i] : 0);
          for (int e0 = 0; e0 < nep; e0 += 8) {
            cl.push_back((int)i);
            ce.push_back(e0);
          }
        }
        h2d(lchunk_leaf_, cl, st_);
        h2d(lchunk_e0_, ce, st_);
        nlchunk_ = (int)cl.size();
        lchunk_key_ = key;
      }
      done = mixed ? launch_l2t_gemm<float>(st_, nlchunk_, lchunk_leaf_.get(), lchunk_e0_.get(), la, R,
                                            local_f_.get(), ops_->wnorm.get())
                   : launch_l2t_gemm<double>(st_, nlchunk_, lchunk_leaf_.get(), lchunk_e0_.get(), la, R,
                                             local_.get(), nullptr);
    }
    if (!done) {
      if (mixed) {
        local_.resize(nb * C * D);
        k_f2d_local<<<1184, 256, 0, st_>>>(local_f_.size(), D, ops_->wnorm.get(), local_f_.get(), local_.get());
        count_launch();
      }
      la.local = local_.get();  // after the resize: the buffer may have been (re)allocated just above
      launch_l2t(st_, nl2t_, la, R);
    }
  } else {
    for (int i = 2; i <= 5; i++) rec(i);
  }
  rec(6);
  // near field: frames only (densities enter the batched contraction; the
  // stored operator, when replayed, replaces them)
  trir_.resize(n);
  if (mode != 2) launch_tri_prep(st_, n, tri_s_.get(), nullptr, nullptr, nullptr, 0, 0, trir_.get());
  const int key = do_src | (do_tgt << 1);
  if (chunk_key_ != key) {
    std::vector<int> cl, ce;
    for (size_t i = 0; i < near_sc_h_.size(); i++) {
      int nep = (do_src ? near_sc_h_[i] : 0) + (do_tgt ? near_tc_h_[i] : 0);
      for (int e0 = 0; e0 < nep; e0 += 8) {
        cl.push_back((int)i);
        ce.push_back(e0);
      }
    }
    h2d(chunk_leaf_, cl, st_);
    h2d(chunk_e0_, ce, st_);
    nchunk_ = (int)cl.size();
    chunk_key_ = key;
  }
  NearArgs na;
  na.nleaf = nnear_;
  na.leaves = near_leaves_.get(); na.nb_start = near_start_.get(); na.nb_items = near_items_.get();
  na.box_src_start = tr_.sstart.get(); na.box_src_count = tr_.scount.get();
  na.box_tgt_start = tr_.tstart.get(); na.box_tgt_count = tr_.tcount.get();
  na.trir = trir_.get();
  na.src_pts = src_s_.get(); na.tgt_pts = tgt_s_.get();
  na.dosl = dosl; na.dodl = dodl; na.dostrain_src = ds_src; na.dostrain_tgt = ds_tgt;
  na.do_src = do_src; na.do_tgt = do_tgt;
  na.rlam = rlam; na.rmu = rmu;
  na.u_src = u_s_.get(); na.e_src = e_s_.get(); na.u_tgt = ut_s_.get(); na.e_tgt = et_s_.get();
  if (mode == 1) {
    NearArgs sa = na;  // stored rows: displacement, and strain if any output wants it
    sa.dostrain_src = sa.dostrain_tgt = (store_flags_ >> 4) & 1;
    launch_near_store(st_, sa, near_base_.get(), near_ntri_.get(), store_K_, 1, store_.get());
    store_valid_ = true;
    store_gen_++;
  }
  if (dosl || dodl) {
    if (mixed && mode && near_tc_ready(na))
      near_tc(na, R, dosl ? ssl_s_.get() : sdl_s_.get(), sdl_s_.get(), n, nt);
    else
      launch_near_batch(st_, na, nchunk_, chunk_leaf_.get(), chunk_e0_.get(), R, (ds_src || ds_tgt) ? 1 : 0,
                        ssl_s_.get(), sdl_s_.get(), n, n, nt, mode ? near_base_.get() : nullptr,
                        mode ? near_ntri_.get() : nullptr, mode ? store_.get() : nullptr);
  }
  rec(7);
  if (do_src) {
    k_scatter_out<<<dim3((n + 255) / 256, R), 256, 0, st_>>>(n, tr_.iz.get(), u_s_.get(), e_s_.get(), d_u_src,
                                                              d_e_src); count_launch();
  }
  if (do_tgt) {
    k_scatter_out<<<dim3((nt + 255) / 256, R), 256, 0, st_>>>(nt, tr_.izt.get(), ut_s_.get(), et_s_.get(),
                                                               d_u_tgt, d_e_tgt); count_launch();
  }
  rec(8);
  EFMM_CUDA_TRY(cudaGetLastError());
  if (capturing_) return IER_OK;  // the graph is launched and timed by its caller
  EFMM_CUDA_TRY(cudaEventSynchronize(ev_[8]));
  cudaEventElapsedTime(&timings.total, ev_[0], ev_[8]);
  cudaEventElapsedTime(&timings.prep, ev_[0], ev_[1]);
  cudaEventElapsedTime(&timings.p2m, ev_[1], ev_[2]);
  cudaEventElapsedTime(&timings.m2m, ev_[2], ev_[3]);
  cudaEventElapsedTime(&timings.m2l, ev_[3], ev_[4]);
  cudaEventElapsedTime(&timings.l2l, ev_[4], ev_[5]);
  cudaEventElapsedTime(&timings.l2t, ev_[5], ev_[6]);
  cudaEventElapsedTime(&timings.near, ev_[6], ev_[7]);
  launches_ = (int)(launches_total() - launch0);
  product_collect();
  if (mixed && tc_take_error()) return IER_CUDA;  // a tensor-core product gave up waiting
  if (mixed) tune_end();
  return IER_OK;
}

int Plan::evaluate_direct(double rlam, double rmu, const double* d_ssl, const double* d_sdl,
                          double* d_u_src, double* d_e_src, double* d_u_tgt, double* d_e_tgt, int nsub) {
  int n = n_, nt = nsub > 0 ? 0 : nt_;
  int dosl = d_ssl != nullptr, dodl = d_sdl != nullptr;
  if (points_) {  // particles: the point-pair direct sum, user order
    const int ns = (d_u_src || d_e_src) ? (nsub > 0 ? std::min(nsub, n) : n) : 0;
    const int ntt = (nt > 0 && (d_u_tgt || d_e_tgt)) ? nt : 0;
    u_s_.resize(3 * (size_t)n);
    e_s_.resize(6 * (size_t)n);
    ut_s_.resize(3 * (size_t)std::max(nt, 1));
    et_s_.resize(6 * (size_t)std::max(nt, 1));
    EFMM_CUDA_TRY(cudaEventRecord(ev_[0], st_));
    launch_part_direct(st_, n, ns, src_u_.get(), d_ssl, d_sdl, nu_u_.get(), ntt, tgt_u_.get(), rlam, rmu, u_s_.get(),
                       e_s_.get(), ut_s_.get(), et_s_.get());
    EFMM_CUDA_TRY(cudaEventRecord(ev_[1], st_));
    if (ns && d_u_src) EFMM_CUDA_TRY(cudaMemcpyAsync(d_u_src, u_s_.get(), 24 * (size_t)ns, cudaMemcpyDeviceToDevice, st_));
    if (ns && d_e_src) { k_sym6to9<<<(ns + 255) / 256, 256, 0, st_>>>(ns, e_s_.get(), d_e_src); count_launch(); }
    if (ntt && d_u_tgt) EFMM_CUDA_TRY(cudaMemcpyAsync(d_u_tgt, ut_s_.get(), 24 * (size_t)nt, cudaMemcpyDeviceToDevice, st_));
    if (ntt && d_e_tgt) { k_sym6to9<<<(nt + 255) / 256, 256, 0, st_>>>(nt, et_s_.get(), d_e_tgt); count_launch(); }
    EFMM_CUDA_TRY(cudaGetLastError());
    EFMM_CUDA_TRY(cudaStreamSynchronize(st_));
    cudaEventElapsedTime(&timings.near, ev_[0], ev_[1]);
    timings.total = timings.near;
    return IER_OK;
  }
  trir_.resize(n);
  launch_tri_prep(st_, n, tri_u_.get(), nullptr, d_ssl, d_sdl, dosl, dodl, trir_.get());
  u_s_.resize(3 * (size_t)n);
  e_s_.resize(6 * (size_t)n);
  ut_s_.resize(3 * (size_t)std::max(nt, 1));
  et_s_.resize(6 * (size_t)std::max(nt, 1));
  u_s_.zero(st_);
  e_s_.zero(st_);
  ut_s_.zero(st_);
  et_s_.zero(st_);
  int do_src = (d_u_src || d_e_src) ? (nsub > 0 ? std::min(nsub, n) : n) : 0;
  int do_tgt = (nt > 0 && (d_u_tgt || d_e_tgt)) ? nt : 0;
  const int ns = nsub > 0 ? std::min(nsub, n) : n;
  EFMM_CUDA_TRY(cudaEventRecord(ev_[0], st_));
  launch_direct_all(st_, n, trir_.get(), do_src, src_u_.get(), do_tgt, tgt_u_.get(), dosl, dodl,
                    d_e_src ? 1 : 0, d_e_tgt ? 1 : 0, rlam, rmu, u_s_.get(), e_s_.get(), ut_s_.get(),
                    et_s_.get());
  EFMM_CUDA_TRY(cudaEventRecord(ev_[1], st_));
  if (d_u_src) EFMM_CUDA_TRY(cudaMemcpyAsync(d_u_src, u_s_.get(), 24 * (size_t)ns, cudaMemcpyDeviceToDevice, st_));
  if (d_e_src) { k_sym6to9<<<(ns + 255) / 256, 256, 0, st_>>>(ns, e_s_.get(), d_e_src); count_launch(); }
  if (nt && d_u_tgt) EFMM_CUDA_TRY(cudaMemcpyAsync(d_u_tgt, ut_s_.get(), 24 * (size_t)nt, cudaMemcpyDeviceToDevice, st_));
  if (nt && d_e_tgt) { k_sym6to9<<<(nt + 255) / 256, 256, 0, st_>>>(nt, et_s_.get(), d_e_tgt); count_launch(); }
  EFMM_CUDA_TRY(cudaGetLastError());
  EFMM_CUDA_TRY(cudaStreamSynchronize(st_));
  cudaEventElapsedTime(&timings.near, ev_[0], ev_[1]);
  timings.total = timings.near;
  return IER_OK;
}

// ---------------------------------------------------------- CUDA graphs
// A repeated evaluation on the same geometry, buffers and parameters is
// captured once into a CUDA graph and then replayed with one launch: the
// first call runs the pass normally (allocations, operator and schedule
// caches, wave lists), the second identical pass is captured, and every
// later call with the same key launches the graph.  During the capture no
// host synchronisation, allocation or upload happens (the caches are warm;
// event timing and error checks are skipped and done around the launch).
void Plan::rec(int i) {
  if (!capturing_) EFMM_CUDA_TRY(cudaEventRecord(ev_[i], st_));
}

void Plan::graph_reset() {
  if (gexec_) cudaGraphExecDestroy(gexec_);
  if (graph_) cudaGraphDestroy(graph_);
  gexec_ = nullptr;
  graph_ = nullptr;
  gkey_.clear();
}

int Plan::run_graph(const std::vector<double>& key, const std::function<int()>& pass) {
  if (gexec_ && key == gkey_) {
    EFMM_CUDA_TRY(cudaEventRecord(ev_[0], st_));
    EFMM_CUDA_TRY(cudaGraphLaunch(gexec_, st_));
    EFMM_CUDA_TRY(cudaEventRecord(ev_[8], st_));
    count_launch((int)graph_launches_);
    EFMM_CUDA_TRY(cudaEventSynchronize(ev_[8]));
    cudaEventElapsedTime(&timings.total, ev_[0], ev_[8]);
    launches_ = (int)graph_launches_;
    if (tc_take_error()) return IER_CUDA;
    return IER_OK;
  }
  graph_reset();
  int ier = pass();  // warm pass: caches and buffers in place
  if (ier) return ier;
  const long long l0 = launches_total();
  capturing_ = true;
  EFMM_CUDA_TRY(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
  cudaGraph_t g = nullptr;
  try {
    ier = pass();
  } catch (...) {
    capturing_ = false;
    cudaStreamEndCapture(st_, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  capturing_ = false;
  const cudaError_t e = cudaStreamEndCapture(st_, &g);
  graph_launches_ = launches_total() - l0;
  count_launch(-(int)graph_launches_);  // captured, not launched
  if (ier || e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    return ier ? ier : IER_CUDA;
  }
  graph_ = g;
  EFMM_CUDA_TRY(cudaGraphInstantiate(&gexec_, graph_, 0));
  gkey_ = key;
  return run_graph(key, pass);
}

int Plan::evaluate_batch_graph(double rlam, double rmu, int R, const double* d_ssl, const double* d_sdl,
                               double* d_u_src, double* d_e_src, double* d_u_tgt, double* d_e_tgt, int precision,
                               int mode) {
  // one pass per call (R <= 64): the passes of a chunked call would re-cut
  // their cached work lists inside the capture
  if ((mode != 0 && mode != 2) || R < 1 || R > 64) return IER_BADARG;
  const std::vector<double> key = {1.0, rlam, rmu, (double)R, (double)(uintptr_t)d_ssl, (double)(uintptr_t)d_sdl,
                                   (double)(uintptr_t)d_u_src, (double)(uintptr_t)d_e_src,
                                   (double)(uintptr_t)d_u_tgt, (double)(uintptr_t)d_e_tgt, (double)precision,
                                   (double)mode};
  struct Flag {
    bool& f;
    ~Flag() { f = false; }
  } flag{graph_pass_ = true};
  return run_graph(key, [&]() {
    return evaluate_batch(rlam, rmu, R, d_ssl, d_sdl, d_u_src, d_e_src, d_u_tgt, d_e_tgt, precision, mode);
  });
}

int Plan::evaluate_image_graph(double rlam, double rmu, int R, const double* d_ssl, const double* d_sdl,
                               double* d_u_tgt, double* d_e_tgt, int precision) {
  if (R < 1 || R > 64) return IER_BADARG;  // one pass per call, as above
  const std::vector<double> key = {2.0, rlam, rmu, (double)R, (double)(uintptr_t)d_ssl, (double)(uintptr_t)d_sdl,
                                   (double)(uintptr_t)d_u_tgt, (double)(uintptr_t)d_e_tgt, (double)precision};
  struct Flag {
    bool& f;
    ~Flag() { f = false; }
  } flag{graph_pass_ = true};
  return run_graph(key, [&]() {
    return evaluate_image(rlam, rmu, R, d_ssl, d_sdl, d_u_tgt, d_e_tgt, precision, 2);
  });
}

// ------------------------------------------------------ half-space image
// The image part of the half-space layer potentials (src/elhfmm3dtria_iter.f:
// 544-840 composes it from an anti-image elastic FMM, a Mindlin B/C FMM and
// an image near field).  Here one plan on (sources, reflected targets) runs
// all of it: per right-hand side seven expansion columns, the four
// anti-image passes (free-space passes with c1 = 2 - alpha and the
// double-layer charge constant (2 lam + 3 mu)/(lam + 2 mu)), the 1/r
// potentials Phi_a and Phi_c of the C piece, and the potential W of
// U = R3 log(R + R3) - R for the B piece, whose M2L uses its own dense
// operators (kind 3).  The image sources lie below z = 0 and the reflected
// targets above it, so every M2L pair has a target box at or above its
// source box, where U is regular.

// M2L pairs of the image plan: target boxes holding targets only, sources
// below or level with them; ukind selects the U operators (alpha = box side,
// U grows like r) instead of the Laplace ones (alpha = 1 / box side).
__global__ void k_m2l_pairs_img(int nb, int pass, int ukind, const int* __restrict__ level,
                                const int* __restrict__ ijk, const int* __restrict__ scount,
                                const int* __restrict__ tcount, const int* __restrict__ l2s,
                                const int* __restrict__ l2i, const int* __restrict__ grp, double size,
                                int* __restrict__ cnt, int* __restrict__ cursor, TransPair* __restrict__ out,
                                int* __restrict__ bad) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  if (level[b] < 2 || tcount[b] == 0) return;
  const double s = size / (double)(1ull << level[b]);
  for (int q = l2s[b]; q < l2s[b + 1]; q++) {
    const int sb = l2i[q];
    if (scount[sb] == 0) continue;
    const int di = ijk[3 * b] - ijk[3 * sb], dj = ijk[3 * b + 1] - ijk[3 * sb + 1],
              dk = ijk[3 * b + 2] - ijk[3 * sb + 2];
    if (di < -3 || di > 3 || dj < -3 || dj > 3 || dk < -3 || dk > 3) continue;
    if (dk < 0) {  // a source box above a target box: not a half-space configuration
      if (pass == 0) atomicAdd(bad, 1);
      continue;
    }
    const int g = grp[(di + 3) * 49 + (dj + 3) * 7 + (dk + 3)];
    if (g < 0) continue;
    if (pass == 0) {
      atomicAdd(&cnt[g], 1);
    } else {
      const int pos = atomicAdd(&cursor[g], 1);
      out[pos] = TransPair{sb, b, ukind ? s : 1.0 / s};
    }
  }
}

void Plan::ensure_uops() {
  std::lock_guard<std::mutex> lk(g_ops_mu);
  OpPool* P = ops_;
  if (P->u_ready) return;
  std::vector<OpDesc> descs;
  long long off = 0;
  for (int q = 0; q < 343; q++) P->m2lu_group[q] = -1;
  P->udims.clear();
  for (int i = -3; i <= 3; i++)
    for (int j = -3; j <= 3; j++)
      for (int k = 0; k <= 3; k++) {
        const int mx = std::max(abs(i), std::max(abs(j), abs(k)));
        if (mx < 2) continue;
        OpDesc d;
        d.kind = 3;
        d.p = std::min(p_, m2l_order(eps_, i, j, k));
        d.d[0] = i; d.d[1] = j; d.d[2] = k;
        d.off = off;
        const int dim = 2 * ncoef(d.p);
        off += (long long)dim * dim;
        P->m2lu_group[(i + 3) * 49 + (j + 3) * 7 + (k + 3)] = (int)descs.size();
        P->udims.push_back(dim);
        descs.push_back(d);
      }
  P->umats.resize(off);
  P->udescs = descs;
  DevBuf<OpDesc> dd;
  dd.resize(descs.size());
  EFMM_CUDA_TRY(cudaMemcpyAsync(dd.get(), descs.data(), descs.size() * sizeof(OpDesc), cudaMemcpyHostToDevice,
                                st_));
  launch_build_ops(st_, (int)descs.size(), dd.get(), P->umats.get(), p_);
  std::vector<long long> offs;
  std::vector<int> kinds;
  for (auto& d : descs) {
    offs.push_back(d.off);
    kinds.push_back(3);
  }
  h2d(P->uoff, offs, st_);
  h2d(P->udim, P->udims, st_);
  h2d(P->ukinds, kinds, st_);
  std::vector<int> g(P->m2lu_group, P->m2lu_group + 343);
  h2d(P->m2lug_dev, g, st_);
  EFMM_CUDA_TRY(cudaStreamSynchronize(st_));
  P->u_ready = true;
}

void Plan::ensure_mats_f() {
  std::lock_guard<std::mutex> lk(g_ops_mu);
  if (ops_->mats_f.size() == ops_->mats.size() && (!ops_->u_ready || ops_->umats_f.size() == ops_->umats.size()))
    return;
  if (ops_->mats_f.size() != ops_->mats.size()) {
    ops_->mats_f.resize(ops_->mats.size());
    k_ops_normalised<<<(int)ops_->dims.size(), 256, 0, st_>>>(ops_->kinds.get(), ops_->off.get(), ops_->dim.get(),
                                                              ops_->wnorm.get(), ops_->mats.get(),
                                                              ops_->mats_f.get());
    count_launch();
  }
  if (ops_->u_ready && ops_->umats_f.size() != ops_->umats.size()) {
    ops_->umats_f.resize(ops_->umats.size());
    k_ops_normalised<<<(int)ops_->udims.size(), 256, 0, st_>>>(ops_->ukinds.get(), ops_->uoff.get(),
                                                               ops_->udim.get(), ops_->wnorm.get(),
                                                               ops_->umats.get(), ops_->umats_f.get());
    count_launch();
  }
  EFMM_CUDA_TRY(cudaStreamSynchronize(st_));
}

int Plan::build_image_sched() {
  const int nb = tr_.nboxes;
  const int gb = (nb + 255) / 256;
  DevBuf<int> bad;
  bad.resize(1);
  bad.zero(st_);
  for (int uk = 0; uk < 2; uk++) {
    TransSched& S = uk ? m2lu_ : m2lv_img_;
    const int* grp = uk ? ops_->m2lug_dev.get() : ops_->m2lg_dev.get();
    S.clear();
    DevBuf<int>& cnt = m2l_cnt_;
    cnt.resize(344);
    cnt.zero(st_);
    k_m2l_pairs_img<<<gb, 256, 0, st_>>>(nb, 0, uk, tr_.level.get(), tr_.ijk.get(), tr_.scount.get(),
                                         tr_.tcount.get(), tr_.l2_start.get(), tr_.l2_items.get(), grp, tr_.size,
                                         cnt.get(), nullptr, nullptr, bad.get());
    count_launch();
    std::vector<int> hc = d2h(cnt, 343, st_);
    std::vector<int> start(344, 0);
    for (int g = 0; g < 343; g++) start[g + 1] = start[g] + hc[g];
    const int tot = start[343];
    for (int g = 0; g < 343; g++)
      if (hc[g] > 0) S.segs.push_back({g, start[g], hc[g]});
    S.lev.push_back({0, (int)S.segs.size()});
    h2d(m2l_cursor_, start, st_);
    S.pairs.resize(std::max(tot, 1));
    k_m2l_pairs_img<<<gb, 256, 0, st_>>>(nb, 1, uk, tr_.level.get(), tr_.ijk.get(), tr_.scount.get(),
                                         tr_.tcount.get(), tr_.l2_start.get(), tr_.l2_items.get(), grp, tr_.size,
                                         nullptr, m2l_cursor_.get(), S.pairs.get(), bad.get());
    count_launch();
  }
  std::vector<int> hb = d2h(bad, 1, st_);
  if (hb[0] != 0) return IER_BADARG;
  // L2L into boxes that hold targets only (the boxes below the surface hold
  // the image sources and are never evaluated)
  {
    auto nkids = d2h(tr_.nkids, nb, st_);
    auto kids = d2h(tr_.kids, 8 * (size_t)nb, st_);
    auto tcount = d2h(tr_.tcount, nb, st_);
    auto ijk = d2h(tr_.ijk, 3 * (size_t)nb, st_);
    l2l_img_.clear();
    std::vector<TransPair> pairs;
    for (int lev = 2; lev < tr_.nlev; lev++) {
      std::vector<std::vector<TransPair>> byg(8);
      const int lo = tr_.laddr[lev].first, cnt = tr_.laddr[lev].second;
      for (int b = lo; b < lo + cnt; b++)
        for (int q = 0; q < nkids[b]; q++) {
          const int k = kids[8 * b + q];
          if (tcount[k] == 0) continue;
          const int dg = ((ijk[3 * k] - 1) & 1) + 2 * ((ijk[3 * k + 1] - 1) & 1) + 4 * ((ijk[3 * k + 2] - 1) & 1);
          byg[dg].push_back(TransPair{b, k, 1.0});
        }
      const int s0 = (int)l2l_img_.segs.size();
      for (int dg = 0; dg < 8; dg++) {
        if (byg[dg].empty()) continue;
        l2l_img_.segs.push_back({ops_->l2l_group[dg], (int)pairs.size(), (int)byg[dg].size()});
        pairs.insert(pairs.end(), byg[dg].begin(), byg[dg].end());
      }
      l2l_img_.lev.push_back({s0, (int)l2l_img_.segs.size() - s0});
    }
    if (pairs.empty()) pairs.push_back(TransPair{0, 0, 0.0});
    h2d(l2l_img_.pairs, pairs, st_);
    // the U column (C = R) runs M2M and L2L on its own copies of the
    // schedules, so that each copy keeps the tasks cut for one column count
    l2l_img_u_.clear();
    l2l_img_u_.segs = l2l_img_.segs;
    l2l_img_u_.lev = l2l_img_.lev;
    h2d(l2l_img_u_.pairs, pairs, st_);
    m2m_u_.clear();
    m2m_u_.segs = m2m_.segs;
    m2m_u_.lev = m2m_.lev;
    size_t np = 0;
    for (const TransSeg& g : m2m_.segs) np = std::max(np, (size_t)(g.pair0 + g.npair));
    std::vector<TransPair> mp = np ? d2h(m2m_.pairs, np, st_) : std::vector<TransPair>(1, TransPair{0, 0, 0.0});
    h2d(m2m_u_.pairs, mp, st_);
  }
  img_sched_ = true;
  return IER_OK;
}

template <class T>
void Plan::run_dense(TransSched& S, int C, const T* mats, const T* src, T* dst) {
  const int D = 2 * ncoef(p_);
  cut_tasks(S, C, &ops_->udims);
  for (auto& r : S.lev_tasks)
    launch_translate<T>(st_, r.second, S.tasks.get() + r.first, S.pairs.get(), mats, ops_->uoff.get(),
                        ops_->udim.get(), D, C, src, dst);
}

void Plan::build_chunks(int do_src, int do_tgt) {
  const int key = do_src | (do_tgt << 1);
  if (chunk_key_ == key) return;
  std::vector<int> cl, ce;
  for (size_t i = 0; i < near_sc_h_.size(); i++) {
    int nep = (do_src ? near_sc_h_[i] : 0) + (do_tgt ? near_tc_h_[i] : 0);
    for (int e0 = 0; e0 < nep; e0 += 8) {
      cl.push_back((int)i);
      ce.push_back(e0);
    }
  }
  h2d(chunk_leaf_, cl, st_);
  h2d(chunk_e0_, ce, st_);
  nchunk_ = (int)cl.size();
  chunk_key_ = key;
}

// Two-stage P2M of the image columns over waves of leaves (budget as in
// p2m_twostage, waves cached likewise): 9 feature rows per node, 7R columns
// (6R Laplace, R of U).
template <class T>
void Plan::p2m_img_twostage(const P2MArgs& pa, int R, T* mpole) {
  const int D = 2 * ncoef(p_), Cv = 6 * R, Cu = R;
  const size_t nb = tr_.nboxes;
  WaveSet& W = p2m_waves_;
  const long long key = ((long long)p_ << 40) | ((long long)R << 8) | (sizeof(T) << 2) | 2;
  if (W.key != key) {
    size_t freeb = 0, totb = 0;
    EFMM_CUDA_TRY(cudaMemGetInfo(&freeb, &totb));
    const size_t budget =
        std::min<size_t>((size_t)8 << 30, freeb / 4 + p2m_scratch_.cap * sizeof(double)) / sizeof(T);
    W.clear();
    std::vector<int> wl;
    std::vector<long long> fo, wo, no;
    std::vector<GemmTask> tasks;
    size_t i = 0;
    const size_t nl = p2m_h_.size();
    while (i < nl) {
      WaveSet::Wave w{0, (long long)wl.size(), 0, (long long)tasks.size(), 0, 0, 0};
      long long used = 0, nodes = 0;
      while (i < nl) {
        // features: 4 charge/dipole rows per node, then 5 second-derivative
        // rows per node; the anti-image columns (4R, no quadrupole sources)
        // multiply the first block only
        const long long K = 108LL * p2m_sc_h_[i], K4 = 48LL * p2m_sc_h_[i];
        const long long need = K * D + K * (Cv + Cu);
        if (w.nwl > 0 && used + need > (long long)budget) break;
        wl.push_back((int)i);
        fo.push_back(used);
        wo.push_back(used + K * D);
        no.push_back(nodes);
        nodes += 12LL * p2m_sc_h_[i];
        const long long box = p2m_h_[i], wb = used + K * D;
        const int CA = 4 * R, CP = 2 * R;
        for (int c0 = 0; c0 < CA; c0 += 128)
          for (int r0 = 0; r0 < D; r0 += 128)
            tasks.push_back({used, wb, box * Cv * D, D, CA, (int)K4, D, (int)K, D, r0, c0});
        for (int c0 = 0; c0 < CP; c0 += 128)
          for (int r0 = 0; r0 < D; r0 += 128)
            tasks.push_back({used, wb + (long long)CA * K, box * Cv * D + (long long)CA * D, D, CP, (int)K, D,
                             (int)K, D, r0, c0});
        for (int c0 = 0; c0 < Cu; c0 += 128)
          for (int r0 = 0; r0 < D; r0 += 128)
            tasks.push_back({used, wb + (long long)Cv * K, (long long)(nb * Cv * D) + box * Cu * D, D, Cu, (int)K,
                             D, (int)K, D, r0, c0});
        used += need;
        w.maxn = std::max(w.maxn, 12 * p2m_sc_h_[i]);
        w.nwl++;
        i++;
      }
      w.ntask = (int)(tasks.size() - w.t0);
      w.used = used;
      w.nodes = nodes;
      W.w.push_back(w);
    }
    W.upload(wl, fo, wo, no, tasks, st_);
    W.key = key;
  }
  size_t maxu = 1;
  long long maxnodes = 1;
  for (const auto& w : W.w) {
    maxu = std::max(maxu, (size_t)w.used);
    maxnodes = std::max(maxnodes, w.nodes);
  }
  p2m_scratch_.resize((maxu * sizeof(T) + sizeof(double) - 1) / sizeof(double));
  wave_nrec_.resize(8 * (size_t)maxnodes);
  T* scratch = reinterpret_cast<T*>(p2m_scratch_.get());
  for (const auto& w : W.w) {
    launch_p2m_img_twostage<T>(st_, pa, R, w.nwl, W.leaves.get() + w.wl0, W.off1.get() + w.wl0,
                               W.off2.get() + w.wl0, W.off3.get() + w.wl0, wave_nrec_.get(), w.maxn, scratch,
                               scratch, w.ntask, W.tasks.get() + w.t0, mpole, false);
    product_timed<T>(w.ntask, W.htasks, w.t0, W.tasks.get() + w.t0, scratch, scratch, mpole);
  }
}

// Two-stage L2T of the image columns at the targets (waves cached as in
// l2t_twostage).
void Plan::l2t_img_twostage(const L2TArgs& la0, int R, const double* local, const float* local_f) {
  const int D = 2 * ncoef(p_), Cv = 6 * R, Cu = R, C = Cv + Cu;
  const size_t nb = tr_.nboxes;
  const bool mixed = local_f != nullptr;
  L2TArgs la = la0;
  la.wnorm = mixed ? ops_->wnorm.get() : nullptr;
  const size_t esz = mixed ? sizeof(float) : sizeof(double);
  WaveSet& W = l2t_waves_;
  const long long key = ((long long)p_ << 40) | ((long long)R << 8) | (esz << 4) | 3 | ((long long)resident_ << 62);
  if (mixed && resident_ && tc_enabled() && split_variant()) {
    const long long skey = key | (1LL << 61);
    bool ok = W.key == skey;
    if (!ok) {
      std::vector<int> Pl(l2t_h_.size());
      for (size_t j = 0; j < Pl.size(); j++) Pl[j] = l2t_tc_h_[j];
      ok = l2t_split_layout(W, D, C, Pl, skey);
    }
    if (ok) {
      l2t_split_run(la, R, local_f, true);
      return;
    }
  }
  if (W.key != key) {
    size_t freeb = 0, totb = 0;
    EFMM_CUDA_TRY(cudaMemGetInfo(&freeb, &totb));
    size_t budget = std::min<size_t>((size_t)8 << 30, freeb / 4 + l2t_scratch_.cap * sizeof(double)) / esz;
    bool res = false;
    if (resident_) {
      long long all = 0;
      for (size_t j = 0; j < l2t_h_.size(); j++) {
        const int P = l2t_tc_h_[j];
        const long long LD = l2t_ld(P);
        all += (long long)D * LD + (long long)C * LD;
      }
      res = resident_fits(all, esz, l2t_scratch_.cap * sizeof(double));
      if (res) budget = (size_t)all;
    }
    W.clear();
    W.resident = res;
    std::vector<int> wl;
    std::vector<long long> go, so;
    std::vector<GemmTask> tasks;
    size_t i = 0;
    const size_t nl = l2t_h_.size();
    while (i < nl) {
      WaveSet::Wave w{0, (long long)wl.size(), 0, (long long)tasks.size(), 0, 0, 0};
      long long used = 0;
      while (i < nl) {
        const int P = l2t_tc_h_[i];
        if (P == 0) {
          i++;
          continue;
        }
        const int LD = (int)l2t_ld(P);
        const long long need = (long long)D * LD + (long long)C * LD;
        if (w.nwl > 0 && used + need > (long long)budget) break;
        wl.push_back((int)i);
        go.push_back(used);
        so.push_back(used + (long long)D * LD);
        const long long box = l2t_h_[i];
        for (int c0 = 0; c0 < Cv; c0 += 128)
          for (int r0 = 0; r0 < 9 * P; r0 += 128)
            tasks.push_back({used, box * Cv * D, used + (long long)D * LD, 9 * P, Cv, D, LD, D, LD, r0, c0});
        for (int c0 = 0; c0 < Cu; c0 += 128)
          for (int r0 = 0; r0 < 9 * P; r0 += 128)
            tasks.push_back({used, (long long)(nb * Cv * D) + box * Cu * D,
                             used + (long long)D * LD + (long long)Cv * LD, 9 * P, Cu, D, LD, D, LD, r0, c0});
        used += need;
        w.maxn = std::max(w.maxn, P);
        w.nwl++;
        i++;
      }
      if (w.nwl == 0) break;
      w.ntask = (int)(tasks.size() - w.t0);
      w.used = used;
      W.w.push_back(w);
    }
    W.upload(wl, go, so, {}, tasks, st_);
    W.key = key;
  }
  size_t maxu = 1;
  for (const auto& w : W.w) maxu = std::max(maxu, (size_t)w.used);
  l2t_scratch_.resize((maxu * esz + sizeof(double) - 1) / sizeof(double));
  const bool do_g = !(W.resident && W.feat_valid);
  for (const auto& w : W.w) {
    if (mixed) {
      float* sc = reinterpret_cast<float*>(l2t_scratch_.get());
      launch_l2t_twostage<float>(st_, la, R, w.nwl, W.leaves.get() + w.wl0, W.off1.get() + w.wl0,
                                 W.off2.get() + w.wl0, w.maxn, sc, sc, w.ntask, W.tasks.get() + w.t0, local_f, true,
                                 do_g);
    } else {
      launch_l2t_twostage<double>(st_, la, R, w.nwl, W.leaves.get() + w.wl0, W.off1.get() + w.wl0,
                                  W.off2.get() + w.wl0, w.maxn, l2t_scratch_.get(), l2t_scratch_.get(), w.ntask,
                                  W.tasks.get() + w.t0, local, true, do_g);
    }
  }
  W.feat_valid = W.resident;
}

int Plan::evaluate_image(double rlam, double rmu, int R, const double* d_ssl, const double* d_sdl,
                         double* d_u_tgt, double* d_e_tgt, int precision, int mode) {
  if (R < 1 || precision < 0 || precision > 1 || mode < 0 || mode > 2) return IER_BADARG;
  if (!mindlin_ || rmu <= 0 || rlam + 2 * rmu <= 0) return IER_BADARG;
  if (points_ && (precision != 0 || 7 * R >= 32)) return IER_BADARG;  // particles: FP64, at most 4 right-hand sides
  switch_precision(precision == 1);
  resident_ = precision == 1 && (mode != 0 || graph_pass_);
  const int nt = nt_;
  if (nt == 0 || !(d_u_tgt || d_e_tgt)) return IER_OK;
  if (!(d_ssl || d_sdl)) {
    if (d_u_tgt) EFMM_CUDA_TRY(cudaMemsetAsync(d_u_tgt, 0, 24 * (size_t)nt * R, st_));
    if (d_e_tgt) EFMM_CUDA_TRY(cudaMemsetAsync(d_e_tgt, 0, 72 * (size_t)nt * R, st_));
    EFMM_CUDA_TRY(cudaStreamSynchronize(st_));
    return IER_OK;
  }
  const int flags = (d_ssl ? 1 : 0) | (d_sdl ? 2 : 0) | 8 | (d_e_tgt ? 16 : 0) | 32;
  if (mode == 2 && (!store_valid_ || flags != store_flags_ || rlam != store_lam_ || rmu != store_mu_))
    return IER_HANDLE;
  if (mode != 2) {
    const int ier = store_alloc(flags, rlam, rmu);
    if (ier) return ier;
  }
  MixedOrders orders(this, precision == 1);
  if (far_) {
    ensure_uops();
    if (!img_sched_) {
      const int ier = build_image_sched();
      if (ier) return ier;
    }
    if (precision == 1) ensure_mats_f();
  }
  const int n = n_, D = 2 * ncoef(p_);
  const size_t nb = tr_.nboxes;
  int Rc = std::min(R, 64);
  if (capturing_) {
    Rc = rc_last_;
  } else if (far_) {
    size_t freeb = 0, totb = 0;
    EFMM_CUDA_TRY(cudaMemGetInfo(&freeb, &totb));
    // the pass's two expansion arrays (FP32 in the mixed form), with room to spare
    const double esz = precision == 1 ? 4.0 : 8.0;
    const double have = 0.5 * (double)freeb + (precision == 1 ? 4.0 * (double)(img_mp_f_.cap + img_lc_f_.cap)
                                                              : 8.0 * (double)(img_mp_.cap + img_lc_.cap));
    while (Rc > 1 && 3.0 * esz * nb * 7 * Rc * D > have) Rc /= 2;
  }
  rc_last_ = Rc;
  float tot = 0;
  product_ms_ = product_flops_ = 0;
  for (int r0 = 0; r0 < R; r0 += Rc) {
    const int rc = std::min(Rc, R - r0);
    const int ier = image_pass(rlam, rmu, rc, d_ssl ? d_ssl + 3 * (size_t)n * r0 : nullptr,
                               d_sdl ? d_sdl + 3 * (size_t)n * r0 : nullptr,
                               d_u_tgt ? d_u_tgt + 3 * (size_t)nt * r0 : nullptr,
                               d_e_tgt ? d_e_tgt + 9 * (size_t)nt * r0 : nullptr, precision == 1,
                               mode != 2 && r0 == 0);
    if (ier) return ier;
    tot += timings.total;
  }
  timings.total = tot;
  if (mode == 0) {
    store_valid_ = false;  // the blocks served this call only
    store_gen_++;
  }
  return IER_OK;
}

int Plan::image_pass(double rlam, double rmu, int R, const double* d_ssl, const double* d_sdl, double* d_u_tgt,
                     double* d_e_tgt, bool mixed, bool store_now) {
  const int n = n_, nt = nt_;
  const int dosl = d_ssl != nullptr, dodl = d_sdl != nullptr;
  const int dstr = d_e_tgt ? 1 : 0;
  const int D = 2 * ncoef(p_);
  const size_t nb = tr_.nboxes;
  long long launch0 = launches_total();
  product_begin();
  rec(0);
  ssl_s_.resize(3 * (size_t)n * R);
  sdl_s_.resize(3 * (size_t)n * R);
  const int gb = (int)(((long long)n * R + 255) / 256);
  if (dosl) { k_gather_rhs<<<gb, 256, 0, st_>>>(n, R, tr_.iz.get(), d_ssl, ssl_s_.get()); count_launch(); }
  if (dodl) { k_gather_rhs<<<gb, 256, 0, st_>>>(n, R, tr_.iz.get(), d_sdl, sdl_s_.get()); count_launch(); }
  ut_s_.resize(3 * (size_t)nt * R);
  et_s_.resize(6 * (size_t)nt * R);
  ut_s_.zero(st_);
  et_s_.zero(st_);
  const double al = (rlam + rmu) / (rlam + 2 * rmu);
  rec(1);
  const int Cv = 6 * R, Cu = R;
  if (far_) {
    const size_t tot = nb * (size_t)(Cv + Cu) * D;
    P2MArgs pa;
    pa.leaves = p2m_leaves_.get();
    pa.level = tr_.level.get(); pa.ijk = tr_.ijk.get();
    pa.sstart = tr_.sstart.get(); pa.scount = tr_.scount.get();
    for (int c = 0; c < 3; c++) pa.c0[c] = tr_.c0[c];
    pa.size = tr_.size;
    pa.flev = tr_.flev;
    pa.tri = tri_s_.get(); pa.nrm = nrm_s_.get(); pa.ssl = ssl_s_.get(); pa.sdl = sdl_s_.get();
    pa.dosl = dosl; pa.dodl = dodl; pa.p = p_;
    // anti-image: Kelvin kernel with c1 = 2 - alpha, double-layer charge constant (2 lam + 3 mu)/(lam + 2 mu)
    pa.c1 = 2.0 - al; pa.c2 = (2 * rlam + 3 * rmu) / (rlam + 2 * rmu); pa.inv2mu = 0.5 / rmu;
    pa.alpha = al; pa.lam = rlam; pa.mu = rmu;
    pa.C = Cv + Cu; pa.rstride = 1; pa.tstride = 3 * (long long)R; pa.dstride = R;
    pa.points = points_ ? 1 : 0;
    pa.pts = src_s_.get();
    if (mixed) {
      img_mp_f_.resize(tot);
      img_lc_f_.resize(tot);
      img_mp_f_.zero(st_);
      img_lc_f_.zero(st_);
      float* mp = img_mp_f_.get();
      float* lc = img_lc_f_.get();
      pa.wnorm = ops_->wnorm.get();
      tune_begin(1, Cv + Cu);
      if (7 * R < 32)
        launch_p2m_img<float>(st_, np2m_, pa, R, (long long)(nb * Cv * D), mp);
      else if (!(p2m_unit_ && p2m_factored<float>(pa, R, mp, true)))
        p2m_img_twostage<float>(pa, R, mp);
      rec(2);
      run_translations(m2m_, Cv, ops_->mats_f.get(), mp, mp);
      run_translations(m2m_u_, Cu, ops_->mats_f.get(), mp + nb * Cv * D, mp + nb * Cv * D);
      rec(3);
      run_translations(m2lv_img_, Cv, ops_->mats_f.get(), mp, lc);
      if (usplit_on())
        run_u_split(Cu, mp + nb * Cv * D, lc + nb * Cv * D);
      else
        run_dense(m2lu_, Cu, ops_->umats_f.get(), mp + nb * Cv * D, lc + nb * Cv * D);
      rec(4);
      run_translations(l2l_img_, Cv, ops_->mats_f.get(), lc, lc);
      run_translations(l2l_img_u_, Cu, ops_->mats_f.get(), lc + nb * Cv * D, lc + nb * Cv * D);
    } else {
      img_mp_.resize(tot);
      img_lc_.resize(tot);
      img_mp_.zero(st_);
      img_lc_.zero(st_);
      double* mp = img_mp_.get();
      double* lc = img_lc_.get();
      if (7 * R < 32)
        launch_p2m_img<double>(st_, np2m_, pa, R, (long long)(nb * Cv * D), mp);
      else if (!(p2m_unit_ && p2m_factored<double>(pa, R, mp, true)))
        p2m_img_twostage<double>(pa, R, mp);
      rec(2);
      run_translations(m2m_, Cv, ops_->mats.get(), mp, mp);
      run_translations(m2m_u_, Cu, ops_->mats.get(), mp + nb * Cv * D, mp + nb * Cv * D);
      rec(3);
      run_translations(m2lv_img_, Cv, ops_->mats.get(), mp, lc);
      run_dense(m2lu_, Cu, ops_->umats.get(), mp + nb * Cv * D, lc + nb * Cv * D);
      rec(4);
      run_translations(l2l_img_, Cv, ops_->mats.get(), lc, lc);
      run_translations(l2l_img_u_, Cu, ops_->mats.get(), lc + nb * Cv * D, lc + nb * Cv * D);
    }
    rec(5);
    L2TArgs la;
    la.leaves = l2t_leaves_.get();
    la.level = tr_.level.get(); la.ijk = tr_.ijk.get();
    la.sstart = tr_.sstart.get(); la.scount = tr_.scount.get();
    la.tstart = tr_.tstart.get(); la.tcount = tr_.tcount.get();
    for (int c = 0; c < 3; c++) la.c0[c] = tr_.c0[c];
    la.size = tr_.size;
    la.flev = tr_.flev;
    la.local = mixed ? nullptr : img_lc_.get();
    la.src_pts = src_s_.get(); la.tgt_pts = tgt_s_.get();
    la.p = p_; la.do_src = 0; la.do_tgt = 1;
    la.dostrain_src = 0; la.dostrain_tgt = dstr;
    la.c1 = 2.0 - al; la.alpha = al; la.mu = rmu;
    la.u_src = nullptr; la.e_src = nullptr; la.u_tgt = ut_s_.get(); la.e_tgt = et_s_.get();
    la.C = Cv + Cu; la.nsrc = n; la.ntgt = nt;
    bool done = false;
    if (7 * R < 32) {
      // few right-hand sides: the direct kernel on FP64 locals
      if (mixed) {
        img_lc_.resize(tot);
        k_f2d_local<<<1184, 256, 0, st_>>>(tot, D, ops_->wnorm.get(), img_lc_f_.get(), img_lc_.get());
        count_launch();
      }
      la.local = img_lc_.get();
      done = launch_l2t_img(st_, nl2t_, la, R, (long long)(nb * Cv * D));
    }
    if (!done) l2t_img_twostage(la, R, mixed ? nullptr : img_lc_.get(), mixed ? img_lc_f_.get() : nullptr);
  } else {
    for (int i = 2; i <= 5; i++) rec(i);
  }
  rec(6);
  // near field: refined quadrature of the whole image kernel, stored, then
  // contracted with the right-hand sides
  build_chunks(0, 1);
  if (store_now) {
    HsStoreArgs ha;
    ha.leaves = near_leaves_.get(); ha.nb_start = near_start_.get(); ha.nb_items = near_items_.get();
    ha.box_src_start = tr_.sstart.get(); ha.box_src_count = tr_.scount.get();
    ha.box_tgt_start = tr_.tstart.get(); ha.box_tgt_count = tr_.tcount.get();
    ha.tri = tri_s_.get(); ha.nrm = nrm_s_.get(); ha.tgt = tgt_s_.get();
    ha.base = near_base_.get(); ha.ntri = near_ntri_.get();
    ha.dosl = dosl; ha.dodl = dodl; ha.dstr = dstr; ha.K = store_K_;
    ha.lam = rlam; ha.mu = rmu;
    ha.eps = hs_quad_eps(iprec_);
    ha.ncap = hs_ncap_ptr();
    ha.points = points_ ? 1 : 0;
    ha.pts = src_s_.get();
    launch_hs_store(st_, ha, nchunk_, chunk_leaf_.get(), chunk_e0_.get(), store_.get());
    store_valid_ = true;
    store_gen_++;
  }
  NearArgs na;
  na.nleaf = nnear_;
  na.leaves = near_leaves_.get(); na.nb_start = near_start_.get(); na.nb_items = near_items_.get();
  na.box_src_start = tr_.sstart.get(); na.box_src_count = tr_.scount.get();
  na.box_tgt_start = tr_.tstart.get(); na.box_tgt_count = tr_.tcount.get();
  na.trir = trir_.get();
  na.src_pts = src_s_.get(); na.tgt_pts = tgt_s_.get();
  na.dosl = dosl; na.dodl = dodl; na.dostrain_src = 0; na.dostrain_tgt = dstr;
  na.do_src = 0; na.do_tgt = 1;
  na.rlam = rlam; na.rmu = rmu;
  na.u_src = nullptr; na.e_src = nullptr; na.u_tgt = ut_s_.get(); na.e_tgt = et_s_.get();
  launch_near_batch(st_, na, nchunk_, chunk_leaf_.get(), chunk_e0_.get(), R, dstr, ssl_s_.get(), sdl_s_.get(), n, n,
                    nt, near_base_.get(), near_ntri_.get(), store_.get());
  rec(7);
  k_scatter_out<<<dim3((nt + 255) / 256, R), 256, 0, st_>>>(nt, tr_.izt.get(), ut_s_.get(), et_s_.get(), d_u_tgt,
                                                             d_e_tgt);
  count_launch();
  rec(8);
  EFMM_CUDA_TRY(cudaGetLastError());
  if (capturing_) return IER_OK;  // the graph is launched and timed by its caller
  EFMM_CUDA_TRY(cudaEventSynchronize(ev_[8]));
  cudaEventElapsedTime(&timings.total, ev_[0], ev_[8]);
  cudaEventElapsedTime(&timings.prep, ev_[0], ev_[1]);
  cudaEventElapsedTime(&timings.p2m, ev_[1], ev_[2]);
  cudaEventElapsedTime(&timings.m2m, ev_[2], ev_[3]);
  cudaEventElapsedTime(&timings.m2l, ev_[3], ev_[4]);
  cudaEventElapsedTime(&timings.l2l, ev_[4], ev_[5]);
  cudaEventElapsedTime(&timings.l2t, ev_[5], ev_[6]);
  cudaEventElapsedTime(&timings.near, ev_[6], ev_[7]);
  launches_ = (int)(launches_total() - launch0);
  product_collect();
  if (mixed && tc_take_error()) return IER_CUDA;  // a tensor-core product gave up waiting
  if (mixed) tune_end();
  return IER_OK;
}

}  // namespace efmm
