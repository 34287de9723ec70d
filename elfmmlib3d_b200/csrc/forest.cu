// forest.cu -- many independent half-space problems of uneven sizes in one
// pass (include/elfmm3d_b200.h, efmm_forest_*).
//
// The reference evaluates one fault per call: its drivers form the
// half-space self-evaluation as the free-space call plus the image call
// (examples/elhfmm3dtria_self_iter_dr.f:331-385).  Here all problems share
// two plans.  Problem k is moved in x and y (the free-space kernel depends on
// differences only, the Mindlin image kernel on x and y differences and the
// absolute depths, so a shift in x and y changes no result) to the centre of
// column k of a 2^L x 2^L grid of boxes of level L of one root cube centred
// on z = 0, and both plans build one tree over all problems as a forest
// (tree.cu): the levels above L split unconditionally, lists never join two
// columns, and each problem gets the FMM of the subtree under its column.
// Every stage (near field, image near field, P2M, translations per level,
// L2T) is then one launch over the boxes of all problems, instead of one
// pass (and one tree build with its host synchronisations) per problem.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>
#include "capi_plan.h"
#include "common.cuh"
#include "devbuf.h"
#include "../../include/elfmm3d_b200.h"

using namespace efmm;

struct efmm_forest {
  int device = 0;
  efmm_plan* f = nullptr;    // direct arrival: sources = centroids
  efmm_plan* img = nullptr;  // image part: targets = reflected centroids, Mindlin root
  int nprob = 0, n = 0;
  int leaf_free = 0, leaf_img = 0;  // efmm_forest_set_leaf (0: default)
  double floor = -1;                 // efmm_forest_set_mixed_floor (< 0: the plans' default)
  DevBuf<long long> off;
  DevBuf<double> bb, tri, cen, refl, uf, ui, ei;
  DevBuf<int> flag;
};

namespace {

// Bounding box of each problem's centroids: one CTA per problem.
__global__ void k_seg_bbox(const long long* __restrict__ off, const double* __restrict__ cen,
                           double* __restrict__ bb) {
  __shared__ double red[6][8];
  const int k = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double v[6] = {1e300, 1e300, 1e300, -1e300, -1e300, -1e300};
  for (long long i = off[k] + threadIdx.x; i < off[k + 1]; i += blockDim.x)
    for (int c = 0; c < 3; c++) {
      const double x = cen[3 * i + c];
      v[c] = fmin(v[c], x);
      v[3 + c] = fmax(v[3 + c], x);
    }
  for (int o = 16; o > 0; o >>= 1)
    for (int c = 0; c < 3; c++) {
      v[c] = fmin(v[c], __shfl_xor_sync(0xffffffffu, v[c], o));
      v[3 + c] = fmax(v[3 + c], __shfl_xor_sync(0xffffffffu, v[3 + c], o));
    }
  if (lane == 0)
    for (int c = 0; c < 6; c++) red[c][warp] = v[c];
  __syncthreads();
  if (threadIdx.x < 6) {
    const int c = threadIdx.x;
    double r = red[c][0];
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) r = c < 3 ? fmin(r, red[c][w]) : fmax(r, red[c][w]);
    bb[6 * k + c] = r;
  }
}

// The shifted copies: triangles and centroids moved by (dx, dy) of their
// problem, the reflected centroids (x + dx, y + dy, -z).  *flag = 1 if a
// vertex or a centroid lies above z = 0.  One CTA per problem.
__global__ void k_forest_place(const long long* __restrict__ off, const double* __restrict__ shift,
                               const double* __restrict__ tri, const double* __restrict__ cen,
                               double* __restrict__ tri_s, double* __restrict__ cen_s, double* __restrict__ refl,
                               int* __restrict__ flag) {
  const int k = blockIdx.x;
  const double dx = shift[2 * k], dy = shift[2 * k + 1];
  bool above = false;
  for (long long i = off[k] + threadIdx.x; i < off[k + 1]; i += blockDim.x) {
    for (int v = 0; v < 3; v++) {
      const double* a = tri + 9 * i + 3 * v;
      double* b = tri_s + 9 * i + 3 * v;
      b[0] = a[0] + dx;
      b[1] = a[1] + dy;
      b[2] = a[2];
      above |= a[2] > 0.0;
    }
    const double x = cen[3 * i] + dx, y = cen[3 * i + 1] + dy, z = cen[3 * i + 2];
    above |= z > 0.0;
    cen_s[3 * i] = x;
    cen_s[3 * i + 1] = y;
    cen_s[3 * i + 2] = z;
    refl[3 * i] = x;
    refl[3 * i + 1] = y;
    refl[3 * i + 2] = -z;
  }
  if (above) atomicExch(flag, 1);
}

__global__ void k_forest_add(size_t n, double* __restrict__ a, const double* __restrict__ b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    a[i] += b[i];
}

int guard(efmm_forest* F, const std::function<int()>& body) {
  try {
    cudaSetDevice(F->device);
    return body();
  } catch (const CudaError& e) {
    if (e.code == (int)cudaErrorMemoryAllocation) {
      cudaGetLastError();  // the failed allocation leaves no sticky error
      return IER_ALLOC;
    }
    return IER_CUDA;
  } catch (const std::bad_alloc&) {
    return IER_ALLOC;
  }
}

std::mutex g_forest_mu;
efmm_forest* g_forest = nullptr;
double g_forest_floor = -1;  // efmm_many_host_set_mixed_floor

}  // namespace

// Columns of side s hold the widest problem (x or y extent) with a margin of
// 2^-10 s on each side; the root, 2^L columns wide, holds the deepest point
// (the Mindlin root is centred on z = 0 and reaches depth side / 2).
extern "C" int efmm_forest_layout(int nprob, const double* bb, double* root5, double* shift) {
  if (nprob < 1 || !bb || !root5 || !shift) return IER_BADARG;
  double ext = 0.0, zmax = 0.0;
  for (int k = 0; k < nprob; k++) {
    const double* b = bb + 6 * k;
    for (int c = 0; c < 3; c++)
      if (!(b[c] <= b[3 + c]) || !std::isfinite(b[c]) || !std::isfinite(b[3 + c])) return IER_BADARG;
    if (b[5] > 0.0) return IER_BADARG;
    ext = std::max(ext, std::max(b[3] - b[0], b[4] - b[1]));
    zmax = std::max(zmax, -b[2]);
  }
  int L = 1;
  while ((1LL << (2 * L)) < nprob) L++;
  if (L > 15) return IER_BADARG;
  const double g = (double)(1 << L);
  double s = ext > 0.0 ? ext * (1.0 + 1.0 / 512.0) : 1.0;
  if (g * s < 2.0 * zmax * (1.0 + 1.0 / 512.0)) s = 2.0 * zmax * (1.0 + 1.0 / 512.0) / g;
  const double side = g * s;
  root5[0] = 0.0;
  root5[1] = 0.0;
  root5[2] = 0.0;
  root5[3] = side;
  root5[4] = L;
  for (int k = 0; k < nprob; k++) {
    const double* b = bb + 6 * k;
    const int i = k & ((1 << L) - 1), j = k >> L;
    const double cx = -side / 2 + (i + 0.5) * s, cy = -side / 2 + (j + 0.5) * s;
    shift[2 * k] = cx - 0.5 * (b[0] + b[3]);
    shift[2 * k + 1] = cy - 0.5 * (b[1] + b[4]);
  }
  return IER_OK;
}

extern "C" efmm_forest* efmm_forest_create(int device) {
  efmm_forest* F = new efmm_forest();
  F->device = device;
  F->f = efmm_plan_create(device);
  F->img = efmm_plan_create(device);
  if (!F->f || !F->img) {
    efmm_plan_destroy(F->f);
    efmm_plan_destroy(F->img);
    delete F;
    return nullptr;
  }
  return F;
}

extern "C" void efmm_forest_destroy(efmm_forest* F) {
  if (!F) return;
  cudaSetDevice(F->device);
  efmm_plan_destroy(F->f);
  efmm_plan_destroy(F->img);
  delete F;
}

extern "C" int efmm_forest_set_leaf(efmm_forest* F, int nbox_free, int nbox_image) {
  if (!F) return IER_BADARG;
  F->leaf_free = std::max(nbox_free, 0);
  F->leaf_img = std::max(nbox_image, 0);
  return IER_OK;
}

extern "C" int efmm_forest_set_mixed_floor(efmm_forest* F, double eps) {
  if (!F) return IER_BADARG;
  F->floor = eps;
  for (efmm_plan* p : {F->f, F->img}) {
    const int ier = efmm_plan_set_mixed_floor(p, eps, nullptr);
    if (ier) return ier;
  }
  return IER_OK;
}

extern "C" efmm_plan* efmm_forest_plan(efmm_forest* F, int which) {
  if (!F) return nullptr;
  return which == 0 ? F->f : (which == 1 ? F->img : nullptr);
}

extern "C" int efmm_forest_set_geometry(efmm_forest* F, int nprob, const int* counts, const double* tri,
                                        const double* nrm, const double* cen, int iprec, int iter) {
  if (!F || nprob < 1 || !counts || !tri || !nrm || !cen) return IER_BADARG;
  std::vector<long long> off(nprob + 1, 0);
  for (int k = 0; k < nprob; k++) {
    if (counts[k] < 1) return IER_BADARG;
    off[k + 1] = off[k] + counts[k];
  }
  if (off[nprob] > 0x7fffffffLL) return IER_BADARG;
  const int n = (int)off[nprob];
  return guard(F, [&]() -> int {
    cudaStream_t st = F->f->stream;
    F->n = 0;
    F->nprob = 0;
    F->off.resize(nprob + 1);
    EFMM_CUDA_TRY(cudaMemcpyAsync(F->off.get(), off.data(), 8 * off.size(), cudaMemcpyHostToDevice, st));
    F->bb.resize(6 * (size_t)nprob);
    k_seg_bbox<<<nprob, 256, 0, st>>>(F->off.get(), cen, F->bb.get());
    count_launch();
    std::vector<double> bb(6 * (size_t)nprob), shift(2 * (size_t)nprob);
    EFMM_CUDA_TRY(cudaMemcpyAsync(bb.data(), F->bb.get(), 8 * bb.size(), cudaMemcpyDeviceToHost, st));
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
    double root[5];
    int ier = efmm_forest_layout(nprob, bb.data(), root, shift.data());
    if (ier) return ier;
    DevBuf<double> dshift;
    dshift.resize(shift.size());
    EFMM_CUDA_TRY(cudaMemcpyAsync(dshift.get(), shift.data(), 8 * shift.size(), cudaMemcpyHostToDevice, st));
    F->tri.resize(9 * (size_t)n);
    F->cen.resize(3 * (size_t)n);
    F->refl.resize(3 * (size_t)n);
    F->flag.resize(1);
    F->flag.zero(st);
    k_forest_place<<<nprob, 256, 0, st>>>(F->off.get(), dshift.get(), tri, cen, F->tri.get(), F->cen.get(),
                                          F->refl.get(), F->flag.get());
    count_launch();
    int above = 0;
    EFMM_CUDA_TRY(cudaMemcpyAsync(&above, F->flag.get(), 4, cudaMemcpyDeviceToHost, st));
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
    if (above) return IER_BADARG;
    for (efmm_plan* p : {F->f, F->img}) {
      ier = efmm_plan_set_forest(p, root);
      if (ier) return ier;
    }
    // the image plan's leaves default to half the free-space plan's: its
    // near-field pairs are integrated with the refined image rule, about 2x
    // cheaper in all at half the leaf (hs-uneven-256, iprec 3: 11.0 -> 7.7 s;
    // 60 per leaf 9.6 s, 30 did not fit in memory)
    efmm_plan_set_leaf(F->f, F->leaf_free);
    efmm_plan_set_leaf(F->img, F->leaf_img > 0 ? F->leaf_img : std::max(1, iprec_nbox(iprec, n, 0, iter != 0) / 2));
    ier = efmm_plan_set_geometry(F->f, n, F->tri.get(), nrm, F->cen.get(), 0, nullptr, iprec, iter, 0);
    if (!ier)
      ier = efmm_plan_set_geometry(F->img, n, F->tri.get(), nrm, F->cen.get(), n, F->refl.get(), iprec, iter, 1);
    if (ier) return ier;
    F->n = n;
    F->nprob = nprob;
    return IER_OK;
  });
}

extern "C" int efmm_forest_evaluate(efmm_forest* F, double rlam, double rmu, const double* ssl, const double* sdl,
                                    double* u, double* e, int precision, int mode) {
  if (!F || F->n < 1 || (!ssl && !sdl) || (!u && !e)) return IER_BADARG;
  if (precision < 0 || precision > 1 || mode < 0 || mode > 2) return IER_BADARG;
  return guard(F, [&]() -> int {
    const size_t n3 = 3 * (size_t)F->n, n9 = 9 * (size_t)F->n;
    // the image pass needs a displacement buffer for strain-only calls too
    double* du = u;
    if (!du) {
      F->uf.resize(n3);
      du = F->uf.get();
    }
    F->ui.resize(n3);
    if (e) F->ei.resize(n9);
    double* dei = e ? F->ei.get() : nullptr;
    int ier = mode ? efmm_plan_evaluate_batch_iter(F->f, rlam, rmu, 1, ssl, sdl, du, e, nullptr, nullptr,
                                                   precision, mode)
                   : efmm_plan_evaluate_batch(F->f, rlam, rmu, 1, ssl, sdl, du, e, nullptr, nullptr, precision);
    if (!ier) ier = efmm_plan_evaluate_image(F->img, rlam, rmu, 1, ssl, sdl, F->ui.get(), dei, precision, mode);
    if (ier) return ier;
    cudaStream_t st = F->f->stream;
    EFMM_CUDA_TRY(cudaStreamSynchronize(F->img->stream));
    k_forest_add<<<592, 256, 0, st>>>(n3, du, F->ui.get());
    count_launch();
    if (e) {
      k_forest_add<<<592, 256, 0, st>>>(n9, e, dei);
      count_launch();
    }
    EFMM_CUDA_TRY(cudaGetLastError());
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
    return IER_OK;
  });
}

extern "C" int elhfmm3dtria_many_host(int iprec, double rlam, double rmu, int nprob, const int* counts,
                                      const double* tri, const double* nrm, const double* cen, const double* ssl,
                                      const double* sdl, double* u, double* e, int precision) {
  if (nprob < 1 || !counts || !tri || !nrm || !cen || (!ssl && !sdl) || (!u && !e)) return IER_BADARG;
  long long nl = 0;
  for (int k = 0; k < nprob; k++) {
    if (counts[k] < 1) return IER_BADARG;
    nl += counts[k];
  }
  if (nl > 0x7fffffffLL) return IER_BADARG;
  const size_t n = (size_t)nl;
  std::lock_guard<std::mutex> lk(g_forest_mu);
  if (!g_forest) {
    const char* d = getenv("ELFMM3D_DEVICE");
    if (efmm_device_count() <= (d ? atoi(d) : 0)) return IER_NODEVICE;
    g_forest = efmm_forest_create(d ? atoi(d) : 0);
    if (!g_forest) return IER_NODEVICE;
  }
  efmm_forest* F = g_forest;
  if (g_forest_floor >= 0 && F->floor != g_forest_floor) {
    const int ier = efmm_forest_set_mixed_floor(F, g_forest_floor);
    if (ier) return ier;
  }
  return guard(F, [&]() -> int {
    cudaStream_t st = F->f->stream;
    DevBuf<double> dt, dn, dc, ds, dd, du, de;
    auto up = [&](DevBuf<double>& b, const double* h, size_t m) {
      b.resize(m);
      EFMM_CUDA_TRY(cudaMemcpyAsync(b.get(), h, 8 * m, cudaMemcpyHostToDevice, st));
    };
    up(dt, tri, 9 * n);
    up(dn, nrm, 3 * n);
    up(dc, cen, 3 * n);
    if (ssl) up(ds, ssl, 3 * n);
    if (sdl) up(dd, sdl, 3 * n);
    if (u) du.resize(3 * n);
    if (e) de.resize(9 * n);
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
    int ier = efmm_forest_set_geometry(F, nprob, counts, dt.get(), dn.get(), dc.get(), iprec, 0);
    if (!ier)
      ier = efmm_forest_evaluate(F, rlam, rmu, ssl ? ds.get() : nullptr, sdl ? dd.get() : nullptr,
                                 u ? du.get() : nullptr, e ? de.get() : nullptr, precision, 0);
    if (ier) return ier;
    if (u) EFMM_CUDA_TRY(cudaMemcpyAsync(u, du.get(), 24 * n, cudaMemcpyDeviceToHost, st));
    if (e) EFMM_CUDA_TRY(cudaMemcpyAsync(e, de.get(), 72 * n, cudaMemcpyDeviceToHost, st));
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
    return IER_OK;
  });
}

extern "C" int efmm_many_host_set_mixed_floor(double eps) {
  std::lock_guard<std::mutex> lk(g_forest_mu);
  g_forest_floor = eps > 0 ? eps : 0.0;
  return IER_OK;
}
