// capi.cu -- extern "C" entry points (include/elfmm3d_b200.h).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>
#include "plan.h"
#include "capi_plan.h"
#include "halfspace.h"
#include "solve.h"
#include "harmonics.cuh"
#include "mindlin_gen.cuh"
#include "../../include/elfmm3d_b200.h"

using namespace efmm;


static int env_device() {
  const char* s = getenv("ELFMM3D_DEVICE");
  return s ? atoi(s) : 0;
}

extern "C" int efmm_device_count(void) {
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess) return 0;
  return c;
}

extern "C" efmm_plan* efmm_plan_create(int device) {
  try {
    if (efmm_device_count() <= device) return nullptr;
    EFMM_CUDA_TRY(cudaSetDevice(device));
    efmm_plan* p = new efmm_plan();
    p->device = device;
    EFMM_CUDA_TRY(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
    p->plan.reset(new Plan(device, p->stream));
    for (int i = 0; i < 8; i++) EFMM_CUDA_TRY(cudaEventCreate(&p->user_ev[i]));
    return p;
  } catch (...) {
    return nullptr;
  }
}

extern "C" void efmm_plan_destroy(efmm_plan* p) {
  if (!p) return;
  cudaSetDevice(p->device);
  p->plan.reset();
  for (int i = 0; i < 8; i++) cudaEventDestroy(p->user_ev[i]);
  cudaStreamDestroy(p->stream);
  delete p;
}

#define EFMM_GUARD(body)              \
  try {                               \
    cudaSetDevice(p->device);         \
    body                              \
  } catch (const efmm::CudaError&) {  \
    return IER_CUDA;                  \
  } catch (const std::bad_alloc&) {   \
    return IER_ALLOC;                 \
  }

extern "C" int efmm_plan_set_geometry(efmm_plan* p, int n, const double* tri, const double* nrm,
                                      const double* src, int nt, const double* tgt, int iprec,
                                      int iter, int mindlin) {
  if (!p) return IER_BADARG;
  EFMM_GUARD(return p->plan->set_geometry(n, tri, nrm, src, nt, tgt, iprec, iter != 0, mindlin != 0);)
}

extern "C" int efmm_plan_evaluate(efmm_plan* p, double rlam, double rmu, const double* ssl,
                                  const double* sdl, double* u_src, double* e_src, double* u_tgt,
                                  double* e_tgt) {
  if (!p) return IER_BADARG;
  EFMM_GUARD(return p->plan->evaluate(rlam, rmu, ssl, sdl, u_src, e_src, u_tgt, e_tgt);)
}

extern "C" int efmm_plan_evaluate_iter(efmm_plan* p, double rlam, double rmu, const double* ssl, const double* sdl,
                                       double* u_src, double* e_src, double* u_tgt, double* e_tgt, int mode) {
  if (!p || mode < 1 || mode > 2) return IER_BADARG;
  EFMM_GUARD(return p->plan->evaluate(rlam, rmu, ssl, sdl, u_src, e_src, u_tgt, e_tgt, mode);)
}

extern "C" int efmm_plan_evaluate_direct_subset(efmm_plan* p, double rlam, double rmu, int nsub,
                                                const double* ssl, const double* sdl, double* u_src,
                                                double* e_src) {
  if (!p || nsub < 1) return IER_BADARG;
  EFMM_GUARD(return p->plan->evaluate_direct(rlam, rmu, ssl, sdl, u_src, e_src, nullptr, nullptr, nsub);)
}

extern "C" int efmm_plan_set_leaf(efmm_plan* p, int nbox) {
  if (!p) return IER_BADARG;
  p->plan->set_leaf(nbox);
  return IER_OK;
}

extern "C" int efmm_plan_set_forest(efmm_plan* p, const double* forest) {
  if (!p) return IER_BADARG;
  if (forest && (!(forest[3] > 0.0) || forest[4] < 1.0 || forest[4] > 15.0 || forest[4] != (int)forest[4]))
    return IER_BADARG;
  p->plan->set_forest(forest);
  return IER_OK;
}

extern "C" int efmm_plan_evaluate_batch(efmm_plan* p, double rlam, double rmu, int nrhs, const double* ssl,
                                        const double* sdl, double* u_src, double* e_src, double* u_tgt,
                                        double* e_tgt, int precision) {
  if (!p) return IER_BADARG;
  EFMM_GUARD(return p->plan->evaluate_batch(rlam, rmu, nrhs, ssl, sdl, u_src, e_src, u_tgt, e_tgt, precision);)
}

extern "C" int efmm_plan_evaluate_batch_iter(efmm_plan* p, double rlam, double rmu, int nrhs, const double* ssl,
                                             const double* sdl, double* u_src, double* e_src, double* u_tgt,
                                             double* e_tgt, int precision, int mode) {
  if (!p || mode < 1 || mode > 2) return IER_BADARG;
  EFMM_GUARD(return p->plan->evaluate_batch(rlam, rmu, nrhs, ssl, sdl, u_src, e_src, u_tgt, e_tgt, precision,
                                            mode);)
}

extern "C" int efmm_plan_evaluate_image(efmm_plan* p, double rlam, double rmu, int nrhs, const double* ssl,
                                        const double* sdl, double* u_tgt, double* e_tgt, int precision, int mode) {
  if (!p) return IER_BADARG;
  EFMM_GUARD(return p->plan->evaluate_image(rlam, rmu, nrhs, ssl, sdl, u_tgt, e_tgt, precision, mode);)
}

extern "C" int efmm_plan_evaluate_batch_graph(efmm_plan* p, double rlam, double rmu, int nrhs, const double* ssl,
                                              const double* sdl, double* u_src, double* e_src, double* u_tgt,
                                              double* e_tgt, int precision, int mode) {
  if (!p) return IER_BADARG;
  EFMM_GUARD(return p->plan->evaluate_batch_graph(rlam, rmu, nrhs, ssl, sdl, u_src, e_src, u_tgt, e_tgt, precision,
                                                  mode);)
}

extern "C" int efmm_plan_evaluate_image_graph(efmm_plan* p, double rlam, double rmu, int nrhs, const double* ssl,
                                              const double* sdl, double* u_tgt, double* e_tgt, int precision) {
  if (!p) return IER_BADARG;
  EFMM_GUARD(return p->plan->evaluate_image_graph(rlam, rmu, nrhs, ssl, sdl, u_tgt, e_tgt, precision);)
}

extern "C" long long efmm_plan_stored_bytes(const efmm_plan* p) { return 8 * p->plan->stored_doubles(); }

extern "C" int efmm_plan_solve(efmm_plan* free_plan, efmm_plan* image_plan, int kind, double rlam, double rmu,
                               int nrhs, const double* nrm, const double* rhs, double* x, double tol, int maxit,
                               int precision, int* iters, double* relres, int* ier_cols) {
  efmm_plan* p = free_plan;
  if (!p) return IER_BADARG;
  if (image_plan && image_plan->device != p->device) return IER_BADARG;
  EFMM_GUARD(return solve_layers(p->plan.get(), image_plan ? image_plan->plan.get() : nullptr, kind, rlam, rmu, nrhs,
                                 nrm, rhs, x, tol, maxit, precision, iters, relres, ier_cols);)
}

extern "C" int efmm_plan_set_mixed_floor(efmm_plan* p, double eps, int* order) {
  if (!p) return IER_BADARG;
  EFMM_GUARD(p->plan->set_mixed_floor(eps); if (order) *order = p->plan->mixed_order(); return IER_OK;)
}

extern "C" void efmm_plan_flops(const efmm_plan* p, double* f5) { p->plan->flops_per_column(f5); }

extern "C" int efmm_plan_translation_flops(efmm_plan* p, int nrhs, int precision, double* f3) {
  if (!p || nrhs < 1 || !f3) return IER_BADARG;
  EFMM_GUARD(p->plan->translation_flops(nrhs, precision == 1, f3); return IER_OK;)
}

extern "C" int efmm_plan_evaluate_direct(efmm_plan* p, double rlam, double rmu, const double* ssl,
                                         const double* sdl, double* u_src, double* e_src,
                                         double* u_tgt, double* e_tgt) {
  if (!p) return IER_BADARG;
  EFMM_GUARD(return p->plan->evaluate_direct(rlam, rmu, ssl, sdl, u_src, e_src, u_tgt, e_tgt);)
}

extern "C" long long efmm_kernel_launches(void) { return efmm::launches_total(); }

extern "C" int efmm_plan_record(efmm_plan* p, int slot) {
  if (!p || slot < 0 || slot >= 8) return IER_BADARG;
  EFMM_GUARD(EFMM_CUDA_TRY(cudaEventRecord(p->user_ev[slot], p->stream)); return IER_OK;)
}

extern "C" float efmm_plan_elapsed(efmm_plan* p, int a, int b) {
  if (!p || a < 0 || a >= 8 || b < 0 || b >= 8) return -1.0f;
  cudaSetDevice(p->device);
  float ms = -1.0f;
  if (cudaEventSynchronize(p->user_ev[b]) != cudaSuccess) return -1.0f;
  if (cudaEventElapsedTime(&ms, p->user_ev[a], p->user_ev[b]) != cudaSuccess) return -1.0f;
  return ms;
}

extern "C" void efmm_plan_timings(const efmm_plan* p, float* ms) {
  const Timings& t = p->plan->timings;
  ms[0] = t.total; ms[1] = t.prep; ms[2] = t.p2m; ms[3] = t.m2m;
  ms[4] = t.m2l; ms[5] = t.l2l; ms[6] = t.l2t; ms[7] = t.near;
}

extern "C" void efmm_plan_product_stats(const efmm_plan* p, double* out2) {
  out2[0] = p->plan->product_ms();
  out2[1] = p->plan->product_flops();
}

extern "C" void efmm_plan_near_stats(const efmm_plan* p, double* out2) { p->plan->near_stats(out2); }

extern "C" void efmm_plan_setup_timings(const efmm_plan* p, float* ms) {
  const Timings& t = p->plan->timings;
  ms[0] = t.geo_tree; ms[1] = t.geo_lists; ms[2] = t.geo_work; ms[3] = t.geo_ops;
}

extern "C" void efmm_plan_info(const efmm_plan* p, long long* info) {
  const Plan& P = *p->plan;
  info[0] = P.tree().nboxes;
  info[1] = P.tree().nlev;
  info[2] = P.order();
  info[3] = P.nbox();
  info[4] = P.near_pairs();
  info[5] = P.m2l_pairs();
  info[6] = P.kernel_launches();
  info[7] = P.far_enabled() ? 1 : 0;
}

template <class T>
static std::vector<T> d2h(const DevBuf<T>& b, size_t n, cudaStream_t st) {
  std::vector<T> h(n);
  if (n) EFMM_CUDA_TRY(cudaMemcpyAsync(h.data(), b.get(), n * sizeof(T), cudaMemcpyDeviceToHost, st));
  EFMM_CUDA_TRY(cudaStreamSynchronize(st));
  return h;
}

extern "C" int efmm_plan_tree_export(const efmm_plan* p, int* boxes, int* iz, int* iztarg, int* laddr,
                                     double* cs4, int* lstart, int* litems, long long* lcount5) {
  try {
    cudaSetDevice(p->device);
    const Tree& T = p->plan->tree();
    cudaStream_t st = p->stream;
    int nb = T.nboxes;
    const DevBuf<int>* ls[5][2] = {{&T.l1_start, &T.l1_items}, {&T.l2_start, &T.l2_items},
                                   {&T.l3_start, &T.l3_items}, {&T.l4_start, &T.l4_items},
                                   {nullptr, nullptr}};
    std::vector<int> cstart[5], citems[5];
    auto ncoll = d2h(T.ncoll, nb, st);
    auto coll = d2h(T.coll, 27 * (size_t)nb, st);
    for (int t = 0; t < 4; t++) {
      cstart[t] = d2h(*ls[t][0], nb + 1, st);
      citems[t] = d2h(*ls[t][1], cstart[t][nb], st);
    }
    cstart[4].assign(nb + 1, 0);
    for (int b = 0; b < nb; b++) {
      cstart[4][b + 1] = cstart[4][b] + ncoll[b];
      for (int q = 0; q < ncoll[b]; q++) citems[4].push_back(coll[27 * b + q]);
    }
    for (int t = 0; t < 5; t++) lcount5[t] = cstart[t][nb];
    if (!litems) return IER_OK;
    auto level = d2h(T.level, nb, st);
    auto ijk = d2h(T.ijk, 3 * (size_t)nb, st);
    auto parent = d2h(T.parent, nb, st);
    auto nk = d2h(T.nkids, nb, st);
    auto kids = d2h(T.kids, 8 * (size_t)nb, st);
    auto ss = d2h(T.sstart, nb, st);
    auto sc = d2h(T.scount, nb, st);
    auto ts = d2h(T.tstart, nb, st);
    auto tc = d2h(T.tcount, nb, st);
    for (int b = 0; b < nb; b++) {
      int* B = boxes + 20 * (size_t)b;
      B[0] = level[b];
      B[1] = ijk[3 * b]; B[2] = ijk[3 * b + 1]; B[3] = ijk[3 * b + 2];
      B[4] = parent[b] + 1;
      for (int q = 0; q < 8; q++) B[5 + q] = q < nk[b] ? kids[8 * b + q] + 1 : 0;
      B[13] = ss[b] + 1; B[14] = sc[b];
      B[15] = ts[b] + 1; B[16] = tc[b];
      B[17] = sc[b] > 0 ? (nk[b] > 0 ? 2 : 1) : 0;
      B[18] = tc[b] > 0 ? (nk[b] > 0 ? 2 : 1) : 0;
      B[19] = 0;
    }
    auto hz = d2h(T.iz, T.n, st);
    for (int i = 0; i < T.n; i++) iz[i] = hz[i] + 1;
    auto hzt = d2h(T.izt, T.nt, st);
    for (int i = 0; i < T.nt; i++) iztarg[i] = hzt[i] + 1;
    for (int l = 0; l <= T.nlev; l++) {
      laddr[2 * l] = T.laddr[l].first + 1;
      laddr[2 * l + 1] = T.laddr[l].second;
    }
    cs4[0] = T.c0[0]; cs4[1] = T.c0[1]; cs4[2] = T.c0[2]; cs4[3] = T.size;
    long long off = 0;
    for (int t = 0; t < 5; t++) {
      for (int b = 0; b <= nb; b++) lstart[(size_t)t * (nb + 1) + b] = cstart[t][b];
      for (size_t q = 0; q < citems[t].size(); q++) litems[off + q] = citems[t][q] + 1;
      off += (long long)citems[t].size();
    }
    return IER_OK;
  } catch (...) {
    return IER_CUDA;
  }
}

// ---------------------------------------------------------------------------
// reference-compatible entry points (host arrays)
// ---------------------------------------------------------------------------
namespace {
std::mutex g_mu;
efmm_plan* g_plan = nullptr;

struct HostCall {
  DevBuf<double> tri, nrm, src, tgt, ssl, sdl, u, e, ut, et;
};
HostCall* g_bufs = nullptr;

efmm_plan* shared_plan() {
  if (!g_plan) g_plan = efmm_plan_create(env_device());
  return g_plan;
}

template <class T>
void up(DevBuf<T>& b, const T* h, size_t n, cudaStream_t st) {
  b.resize(n);
  if (n) EFMM_CUDA_TRY(cudaMemcpyAsync(b.get(), h, n * sizeof(T), cudaMemcpyHostToDevice, st));
}
template <class T>
void down(T* h, const DevBuf<T>& b, size_t n, cudaStream_t st) {
  if (n) EFMM_CUDA_TRY(cudaMemcpyAsync(h, b.get(), n * sizeof(T), cudaMemcpyDeviceToHost, st));
}

int host_call(int iprec, double rlam, double rmu, const double* tri, const double* nrm, int n,
              const double* src, int ifsingle, const double* ssl, int ifdouble, const double* sdl,
              int ifptfrc, double* ptfrc, int ifstrain, double* strain, int nt, const double* tgt,
              int ifptfrctarg, double* ptfrctarg, int ifstraintarg, double* straintarg, bool direct,
              bool iter = false) {
  if (n < 1 || nt < 0) return IER_BADARG;
  std::lock_guard<std::mutex> lk(g_mu);
  efmm_plan* p = shared_plan();
  if (!p) return IER_NODEVICE;
  try {
    cudaSetDevice(p->device);
    if (!g_bufs) g_bufs = new HostCall();
    HostCall& B = *g_bufs;
    cudaStream_t st = p->stream;
    up(B.tri, tri, 9 * (size_t)n, st);
    up(B.nrm, nrm, 3 * (size_t)n, st);
    up(B.src, src, 3 * (size_t)n, st);
    up(B.tgt, tgt, 3 * (size_t)nt, st);
    if (ifsingle) up(B.ssl, ssl, 3 * (size_t)n, st);
    if (ifdouble) up(B.sdl, sdl, 3 * (size_t)n, st);
    B.u.resize(3 * (size_t)n);
    B.e.resize(9 * (size_t)n);
    B.ut.resize(3 * (size_t)std::max(nt, 1));
    B.et.resize(9 * (size_t)std::max(nt, 1));
    int ier = p->plan->set_geometry(n, B.tri.get(), B.nrm.get(), B.src.get(), nt, B.tgt.get(),
                                    iprec, iter, false);
    if (ier) return ier;
    bool src_out = ifptfrc || ifstrain, tgt_out = nt > 0 && (ifptfrctarg || ifstraintarg);
    double* du = src_out ? B.u.get() : nullptr;
    double* de = ifstrain ? B.e.get() : nullptr;
    double* dut = tgt_out ? B.ut.get() : nullptr;
    double* det = (nt > 0 && ifstraintarg) ? B.et.get() : nullptr;
    const double* dssl = ifsingle ? B.ssl.get() : nullptr;
    const double* dsdl = ifdouble ? B.sdl.get() : nullptr;
    ier = direct ? p->plan->evaluate_direct(rlam, rmu, dssl, dsdl, du, de, dut, det)
                 : p->plan->evaluate(rlam, rmu, dssl, dsdl, du, de, dut, det);
    if (ier) return ier;
    if (ifptfrc) down(ptfrc, B.u, 3 * (size_t)n, st);
    if (ifstrain) down(strain, B.e, 9 * (size_t)n, st);
    if (nt > 0 && ifptfrctarg) down(ptfrctarg, B.ut, 3 * (size_t)nt, st);
    if (nt > 0 && ifstraintarg) down(straintarg, B.et, 9 * (size_t)nt, st);
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
    return IER_OK;
  } catch (const efmm::CudaError&) {
    return IER_CUDA;
  } catch (const std::bad_alloc&) {
    return IER_ALLOC;
  }
}
}  // namespace

// ---------------------------------------------------------------------------
// Particle FMM (src/elfmm3dpart.f:52-218, el3dpartdirecttarg :506): point
// forces sigma_sl and point displacement discontinuities sigma_dl with
// orientations sigma_dv at the sources; displacement and strain at the
// sources (self-interaction excluded) and at targets.
// ---------------------------------------------------------------------------
namespace {
int part_call(int iprec, double rlam, double rmu, int n, const double* src, int ifsingle, const double* ssl,
              int ifdouble, const double* sdl, const double* sdv, int ifptfrc, double* ptfrc, int ifstrain,
              double* strain, int nt, const double* tgt, int ifptfrctarg, double* ptfrctarg, int ifstraintarg,
              double* straintarg, bool direct) {
  if (n < 1 || nt < 0 || rmu <= 0) return IER_BADARG;
  if (ifdouble && !sdv) return IER_BADARG;
  std::lock_guard<std::mutex> lk(g_mu);
  efmm_plan* p = shared_plan();
  if (!p) return IER_NODEVICE;
  try {
    cudaSetDevice(p->device);
    if (!g_bufs) g_bufs = new HostCall();
    HostCall& B = *g_bufs;
    cudaStream_t st = p->stream;
    up(B.src, src, 3 * (size_t)n, st);
    up(B.tgt, tgt, 3 * (size_t)nt, st);
    if (ifdouble) up(B.nrm, sdv, 3 * (size_t)n, st);
    if (ifsingle) up(B.ssl, ssl, 3 * (size_t)n, st);
    if (ifdouble) up(B.sdl, sdl, 3 * (size_t)n, st);
    B.u.resize(3 * (size_t)n);
    B.e.resize(9 * (size_t)n);
    B.ut.resize(3 * (size_t)std::max(nt, 1));
    B.et.resize(9 * (size_t)std::max(nt, 1));
    int ier = p->plan->set_geometry(n, nullptr, ifdouble ? B.nrm.get() : nullptr, B.src.get(), nt, B.tgt.get(),
                                    iprec, false, false);
    if (ier) return ier;
    const bool src_out = ifptfrc || ifstrain, tgt_out = nt > 0 && (ifptfrctarg || ifstraintarg);
    double* du = src_out ? B.u.get() : nullptr;
    double* de = ifstrain ? B.e.get() : nullptr;
    double* dut = tgt_out ? B.ut.get() : nullptr;
    double* det = (nt > 0 && ifstraintarg) ? B.et.get() : nullptr;
    const double* dssl = ifsingle ? B.ssl.get() : nullptr;
    const double* dsdl = ifdouble ? B.sdl.get() : nullptr;
    ier = direct ? p->plan->evaluate_direct(rlam, rmu, dssl, dsdl, du, de, dut, det)
                 : p->plan->evaluate(rlam, rmu, dssl, dsdl, du, de, dut, det);
    if (ier) return ier;
    if (ifptfrc) down(ptfrc, B.u, 3 * (size_t)n, st);
    if (ifstrain) down(strain, B.e, 9 * (size_t)n, st);
    if (nt > 0 && ifptfrctarg) down(ptfrctarg, B.ut, 3 * (size_t)nt, st);
    if (nt > 0 && ifstraintarg) down(straintarg, B.et, 9 * (size_t)nt, st);
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
    return IER_OK;
  } catch (const efmm::CudaError&) {
    return IER_CUDA;
  } catch (const std::bad_alloc&) {
    return IER_ALLOC;
  }
}
}  // namespace

namespace {
// The half-space particle FMM (src/elhfmm3dpart.f:47-498): the free-space
// particle FMM (the direct arrival) plus the image part through the image
// FMM with one P2M node per source and the image kernels at the points as
// the near field, on the sources (self-interaction of the direct arrival
// excluded; the image of a source acts on it) and on the targets.  Sources
// and targets in z <= 0.  direct: the O(N^2) sums (elh3dpartdirecttarg).
int hs_part_call(int iprec, double rlam, double rmu, int n, const double* src, int ifsingle, const double* ssl,
                 int ifdouble, const double* sdl, const double* sdv, int ifptfrc, double* ptfrc, int ifstrain,
                 double* strain, int nt, const double* tgt, int ifptfrctarg, double* ptfrctarg, int ifstraintarg,
                 double* straintarg, bool direct) {
  if (n < 1 || nt < 0) return IER_BADARG;
  for (int i = 0; i < n; i++)
    if (src[3 * i + 2] > 0.0) return IER_BADARG;
  for (int i = 0; i < nt; i++)
    if (tgt[3 * i + 2] > 0.0) return IER_BADARG;
  int ier = part_call(iprec, rlam, rmu, n, src, ifsingle, ssl, ifdouble, sdl, sdv, ifptfrc, ptfrc, ifstrain, strain,
                      nt, tgt, ifptfrctarg, ptfrctarg, ifstraintarg, straintarg, direct);
  if (ier) return ier;
  const bool on_src = ifptfrc || ifstrain, on_tgt = nt > 0 && (ifptfrctarg || ifstraintarg);
  if (!on_src && !on_tgt) return IER_OK;
  const int ns = on_src ? n : 0, m = ns + (on_tgt ? nt : 0);
  std::vector<double> pts(3 * (size_t)m), ui(3 * (size_t)m), ei(9 * (size_t)m);
  for (int i = 0; i < ns; i++)
    for (int d = 0; d < 3; d++) pts[3 * i + d] = src[3 * i + d];
  for (int i = 0; i < (on_tgt ? nt : 0); i++)
    for (int d = 0; d < 3; d++) pts[3 * (size_t)(ns + i) + d] = tgt[3 * i + d];
  {
    std::lock_guard<std::mutex> lk(g_mu);
    efmm_plan* p = shared_plan();
    if (!p) return IER_NODEVICE;
    try {
      cudaSetDevice(p->device);
      HostCall& B = *g_bufs;  // made by part_call
      cudaStream_t st = p->stream;
      std::vector<double> refl(pts);
      for (int i = 0; i < m; i++) refl[3 * i + 2] = -refl[3 * i + 2];
      up(B.src, src, 3 * (size_t)n, st);
      if (ifdouble) up(B.nrm, sdv, 3 * (size_t)n, st);
      if (ifsingle) up(B.ssl, ssl, 3 * (size_t)n, st);
      if (ifdouble) up(B.sdl, sdl, 3 * (size_t)n, st);
      B.ut.resize(3 * (size_t)m);
      B.et.resize(9 * (size_t)m);
      const double* dssl = ifsingle ? B.ssl.get() : nullptr;
      const double* dsdl = ifdouble ? B.sdl.get() : nullptr;
      if (direct) {
        up(B.tgt, pts.data(), 3 * (size_t)m, st);
        B.u.resize(6 * (size_t)m);
        launch_part_image(st, n, B.src.get(), dssl, dsdl, ifdouble ? B.nrm.get() : nullptr, m, B.tgt.get(), rlam, rmu,
                          B.ut.get(), B.u.get());
        std::vector<double> e6(6 * (size_t)m);
        down(ui.data(), B.ut, 3 * (size_t)m, st);
        down(e6.data(), B.u, 6 * (size_t)m, st);
        EFMM_CUDA_TRY(cudaStreamSynchronize(st));
        for (int i = 0; i < m; i++) {
          const double* q = &e6[6 * (size_t)i];
          double* o = &ei[9 * (size_t)i];
          o[0] = q[0]; o[4] = q[1]; o[8] = q[2];
          o[1] = o[3] = q[3];
          o[2] = o[6] = q[4];
          o[5] = o[7] = q[5];
        }
      } else {
        up(B.tgt, refl.data(), 3 * (size_t)m, st);
        ier = p->plan->set_geometry(n, nullptr, ifdouble ? B.nrm.get() : nullptr, B.src.get(), m, B.tgt.get(), iprec,
                                    false, true);
        if (ier) return ier;
        ier = p->plan->evaluate_image(rlam, rmu, 1, dssl, dsdl, B.ut.get(), B.et.get(), 0, 0);
        if (ier) return ier;
        down(ui.data(), B.ut, 3 * (size_t)m, st);
        down(ei.data(), B.et, 9 * (size_t)m, st);
        EFMM_CUDA_TRY(cudaStreamSynchronize(st));
      }
    } catch (const efmm::CudaError&) {
      return IER_CUDA;
    } catch (const std::bad_alloc&) {
      return IER_ALLOC;
    }
  }
  if (ifptfrc)
    for (size_t k = 0; k < 3 * (size_t)n; k++) ptfrc[k] += ui[k];
  if (ifstrain)
    for (size_t k = 0; k < 9 * (size_t)n; k++) strain[k] += ei[k];
  if (on_tgt && ifptfrctarg)
    for (size_t k = 0; k < 3 * (size_t)nt; k++) ptfrctarg[k] += ui[3 * (size_t)ns + k];
  if (on_tgt && ifstraintarg)
    for (size_t k = 0; k < 9 * (size_t)nt; k++) straintarg[k] += ei[9 * (size_t)ns + k];
  return IER_OK;
}
}  // namespace

extern "C" void elhfmm3dparttarg_(int* ier, const int* iprec, const double* rlam, const double* rmu, const int* nparts,
                                  const double* source, const int* ifsingle, const double* sigma_sl,
                                  const int* ifdouble, const double* sigma_dl, const double* sigma_dv,
                                  const int* ifptfrc, double* ptfrc, const int* ifstrain, double* strain,
                                  const int* ntargs, const double* target, const int* ifptfrctarg, double* ptfrctarg,
                                  const int* ifstraintarg, double* straintarg) {
  *ier = hs_part_call(*iprec, *rlam, *rmu, *nparts, source, *ifsingle, sigma_sl, *ifdouble, sigma_dl, sigma_dv,
                      *ifptfrc, ptfrc, *ifstrain, strain, *ntargs, target, *ifptfrctarg, ptfrctarg, *ifstraintarg,
                      straintarg, false);
}

extern "C" void elhfmm3dpart_(int* ier, const int* iprec, const double* rlam, const double* rmu, const int* nparts,
                              const double* source, const int* ifsingle, const double* sigma_sl, const int* ifdouble,
                              const double* sigma_dl, const double* sigma_dv, const int* ifptfrc, double* ptfrc,
                              const int* ifstrain, double* strain) {
  *ier = hs_part_call(*iprec, *rlam, *rmu, *nparts, source, *ifsingle, sigma_sl, *ifdouble, sigma_dl, sigma_dv,
                      *ifptfrc, ptfrc, *ifstrain, strain, 0, nullptr, 0, nullptr, 0, nullptr, false);
}

extern "C" void elh3dpartdirecttarg_(const double* rlam, const double* rmu, const int* nsource, const double* source,
                                     const int* ifsingle, const double* sigma_sl, const int* ifdouble,
                                     const double* sigma_dl, const double* sigma_dv, const int* ifptfrc,
                                     double* ptfrc, const int* ifstrain, double* strain, const int* ntarget,
                                     const double* target, const int* ifptfrctarg, double* ptfrctarg,
                                     const int* ifstraintarg, double* straintarg) {
  hs_part_call(2, *rlam, *rmu, *nsource, source, *ifsingle, sigma_sl, *ifdouble, sigma_dl, sigma_dv, *ifptfrc, ptfrc,
               *ifstrain, strain, *ntarget, target, *ifptfrctarg, ptfrctarg, *ifstraintarg, straintarg, true);
}

extern "C" void elfmm3dparttarg_(int* ier, const int* iprec, const double* rlam, const double* rmu, const int* nparts,
                                 const double* source, const int* ifsingle, const double* sigma_sl,
                                 const int* ifdouble, const double* sigma_dl, const double* sigma_dv,
                                 const int* ifptfrc, double* ptfrc, const int* ifstrain, double* strain,
                                 const int* ntargs, const double* target, const int* ifptfrctarg, double* ptfrctarg,
                                 const int* ifstraintarg, double* straintarg) {
  *ier = part_call(*iprec, *rlam, *rmu, *nparts, source, *ifsingle, sigma_sl, *ifdouble, sigma_dl, sigma_dv,
                   *ifptfrc, ptfrc, *ifstrain, strain, *ntargs, target, *ifptfrctarg, ptfrctarg, *ifstraintarg,
                   straintarg, false);
}

extern "C" void elfmm3dpart_(int* ier, const int* iprec, const double* rlam, const double* rmu, const int* nparts,
                             const double* source, const int* ifsingle, const double* sigma_sl, const int* ifdouble,
                             const double* sigma_dl, const double* sigma_dv, const int* ifptfrc, double* ptfrc,
                             const int* ifstrain, double* strain) {
  *ier = part_call(*iprec, *rlam, *rmu, *nparts, source, *ifsingle, sigma_sl, *ifdouble, sigma_dl, sigma_dv,
                   *ifptfrc, ptfrc, *ifstrain, strain, 0, nullptr, 0, nullptr, 0, nullptr, false);
}

extern "C" void el3dpartdirecttarg_(const double* rlam, const double* rmu, const int* nsource, const double* source,
                                    const int* ifsingle, const double* sigma_sl, const int* ifdouble,
                                    const double* sigma_dl, const double* sigma_dv, const int* ifptfrc,
                                    double* ptfrc, const int* ifstrain, double* strain, const int* ntarget,
                                    const double* target, const int* ifptfrctarg, double* ptfrctarg,
                                    const int* ifstraintarg, double* straintarg) {
  part_call(2, *rlam, *rmu, *nsource, source, *ifsingle, sigma_sl, *ifdouble, sigma_dl, sigma_dv, *ifptfrc, ptfrc,
            *ifstrain, strain, *ntarget, target, *ifptfrctarg, ptfrctarg, *ifstraintarg, straintarg, true);
}

extern "C" void elfmm3dtriatarg_(int* ier, const int* iprec, const double* rlam, const double* rmu,
                                 const double* triangle, const double* trinorm, const int* nparts,
                                 const double* source, const int* ifsingle, const double* sigma_sl,
                                 const int* ifdouble, const double* sigma_dl, const int* ifptfrc,
                                 double* ptfrc, const int* ifstrain, double* strain,
                                 const int* ntargs, const double* target, const int* ifptfrctarg,
                                 double* ptfrctarg, const int* ifstraintarg, double* straintarg) {
  *ier = host_call(*iprec, *rlam, *rmu, triangle, trinorm, *nparts, source, *ifsingle, sigma_sl,
                   *ifdouble, sigma_dl, *ifptfrc, ptfrc, *ifstrain, strain, *ntargs, target,
                   *ifptfrctarg, ptfrctarg, *ifstraintarg, straintarg, false);
}

extern "C" void elfmm3dtria_(int* ier, const int* iprec, const double* rlam, const double* rmu,
                             const double* triangle, const double* trinorm, const int* nparts,
                             const double* source, const int* ifsingle, const double* sigma_sl,
                             const int* ifdouble, const double* sigma_dl, const int* ifptfrc,
                             double* ptfrc, const int* ifstrain, double* strain) {
  *ier = host_call(*iprec, *rlam, *rmu, triangle, trinorm, *nparts, source, *ifsingle, sigma_sl,
                   *ifdouble, sigma_dl, *ifptfrc, ptfrc, *ifstrain, strain, 0, nullptr, 0, nullptr,
                   0, nullptr, false);
}

extern "C" void el3dtriadirecttarg_(const double* rlam, const double* rmu, const double* triangle,
                                    const double* trinorm, const int* nsource, const double* source,
                                    const int* ifsingle, const double* sigma_sl, const int* ifdouble,
                                    const double* sigma_dl, const int* ifptfrc, double* ptfrc,
                                    const int* ifstrain, double* strain, const int* ntarget,
                                    const double* target, const int* ifptfrctarg, double* ptfrctarg,
                                    const int* ifstraintarg, double* straintarg) {
  int ier = host_call(6, *rlam, *rmu, triangle, trinorm, *nsource, source, *ifsingle, sigma_sl,
                      *ifdouble, sigma_dl, *ifptfrc, ptfrc, *ifstrain, strain, *ntarget, target,
                      *ifptfrctarg, ptfrctarg, *ifstraintarg, straintarg, true);
  if (ier) fprintf(stderr, "el3dtriadirecttarg: error %d\n", ier);
}

// Many right-hand sides from host arrays (no counterpart in the reference):
// the reference-style call of the batched forms, host copies included.
extern "C" int efmm_batch_host(int iprec, double rlam, double rmu, int n, const double* tri, const double* nrm,
                               const double* src, int nt, const double* tgt, int nrhs, const double* ssl,
                               const double* sdl, double* u_src, double* e_src, double* u_tgt, double* e_tgt,
                               int precision) {
  if (n < 1 || nt < 0 || nrhs < 1) return IER_BADARG;
  std::lock_guard<std::mutex> lk(g_mu);
  efmm_plan* p = shared_plan();
  if (!p) return IER_NODEVICE;
  try {
    cudaSetDevice(p->device);
    if (!g_bufs) g_bufs = new HostCall();
    HostCall& B = *g_bufs;
    cudaStream_t st = p->stream;
    const size_t R = nrhs;
    up(B.tri, tri, 9 * (size_t)n, st);
    up(B.nrm, nrm, 3 * (size_t)n, st);
    up(B.src, src, 3 * (size_t)n, st);
    up(B.tgt, tgt, 3 * (size_t)nt, st);
    if (ssl) up(B.ssl, ssl, 3 * (size_t)n * R, st);
    if (sdl) up(B.sdl, sdl, 3 * (size_t)n * R, st);
    B.u.resize(3 * (size_t)n * R);
    B.e.resize(9 * (size_t)n * R);
    B.ut.resize(3 * (size_t)std::max(nt, 1) * R);
    B.et.resize(9 * (size_t)std::max(nt, 1) * R);
    int ier = p->plan->set_geometry(n, B.tri.get(), B.nrm.get(), B.src.get(), nt, B.tgt.get(), iprec, false, false);
    if (ier) return ier;
    ier = p->plan->evaluate_batch(rlam, rmu, nrhs, ssl ? B.ssl.get() : nullptr, sdl ? B.sdl.get() : nullptr,
                                  (u_src || e_src) ? B.u.get() : nullptr, e_src ? B.e.get() : nullptr,
                                  (nt > 0 && (u_tgt || e_tgt)) ? B.ut.get() : nullptr,
                                  (nt > 0 && e_tgt) ? B.et.get() : nullptr, precision);
    if (ier) return ier;
    if (u_src) down(u_src, B.u, 3 * (size_t)n * R, st);
    if (e_src) down(e_src, B.e, 9 * (size_t)n * R, st);
    if (nt > 0 && u_tgt) down(u_tgt, B.ut, 3 * (size_t)nt * R, st);
    if (nt > 0 && e_tgt) down(e_tgt, B.et, 9 * (size_t)nt * R, st);
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
    return IER_OK;
  } catch (const efmm::CudaError&) {
    return IER_CUDA;
  } catch (const std::bad_alloc&) {
    return IER_ALLOC;
  }
}

// ---------------------------------------------------------------------------
// Half-space image part (src/elhfmm3dtria_iter.f:46-51): direct GPU sum.
// ---------------------------------------------------------------------------
namespace {
struct HsBufs {
  DevBuf<double> tri, nrm, ssl, sdl, tgt, u, e6;
  DevBuf<HsTri> work;
};
HsBufs* g_hs = nullptr;

int hs_call(int iprec, double rlam, double rmu, const double* tri, const double* nrm, int n, int ifsingle,
            const double* ssl, int ifdouble, const double* sdl, int nt, const double* tgt, int ifptfrctarg,
            double* ptfrctarg, int ifstraintarg, double* straintarg, int icomp, int* lused) {
  if (lused) *lused = 8;
  if (n < 1 || nt < 0) return IER_BADARG;
  if (iprec < -2 || iprec > 6) return IER_BADARG;
  if (icomp == 0 || icomp == 4 || nt == 0 || !(ifptfrctarg || ifstraintarg)) return IER_OK;
  if (icomp < 0 || icomp > 5) return IER_BADARG;
  // the half-space is z <= 0: sources and targets must lie in it
  for (int i = 0; i < 3 * n; i++)
    if (tri[3 * i + 2] > 0.0) return IER_BADARG;
  for (int i = 0; i < nt; i++)
    if (tgt[3 * i + 2] > 0.0) return IER_BADARG;
  std::lock_guard<std::mutex> lk(g_mu);
  efmm_plan* p = shared_plan();
  if (!p) return IER_NODEVICE;
  try {
    cudaSetDevice(p->device);
    if (!g_hs) g_hs = new HsBufs();
    HsBufs& B = *g_hs;
    cudaStream_t st = p->stream;
    up(B.tri, tri, 9 * (size_t)n, st);
    up(B.nrm, nrm, 3 * (size_t)n, st);
    if (ifsingle) up(B.ssl, ssl, 3 * (size_t)n, st);
    if (ifdouble) up(B.sdl, sdl, 3 * (size_t)n, st);
    up(B.tgt, tgt, 3 * (size_t)nt, st);
    B.work.resize(n);
    B.u.resize(3 * (size_t)nt);
    B.e6.resize(6 * (size_t)nt);
    launch_hs_image(st, n, B.tri.get(), B.nrm.get(), ifsingle ? B.ssl.get() : nullptr,
                    ifdouble ? B.sdl.get() : nullptr, nt, B.tgt.get(), rlam, rmu, hs_quad_eps(iprec), hs_ncap_ptr(),
                    B.work.get(), B.u.get(), B.e6.get());
    std::vector<double> e6(6 * (size_t)nt);
    if (ifptfrctarg) down(ptfrctarg, B.u, 3 * (size_t)nt, st);
    if (ifstraintarg) down(e6.data(), B.e6, 6 * (size_t)nt, st);
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
    if (ifstraintarg)
      for (int i = 0; i < nt; i++) {
        const double* s = &e6[6 * (size_t)i];
        double* o = straintarg + 9 * (size_t)i;
        o[0] = s[0]; o[4] = s[1]; o[8] = s[2];
        o[1] = o[3] = s[3];
        o[2] = o[6] = s[4];
        o[5] = o[7] = s[5];
      }
    return IER_OK;
  } catch (const efmm::CudaError&) {
    return IER_CUDA;
  } catch (const std::bad_alloc&) {
    return IER_ALLOC;
  }
}
}  // namespace

// Sub-triangles of the image quadrature kept at the adaptive depth cap
// without meeting the tolerance since the last call (on the current device).
extern "C" int efmm_hs_capped(void) {
  try {
    return hs_take_ncap();
  } catch (const efmm::CudaError&) {
    return -1;
  }
}

extern "C" int efmm_hs_image_direct(int iprec, double rlam, double rmu, const double* tri, const double* nrm, int n,
                                    const double* ssl, const double* sdl, int nt, const double* tgt, double* u,
                                    double* e) {
  return hs_call(iprec, rlam, rmu, tri, nrm, n, ssl != nullptr, ssl, sdl != nullptr, sdl, nt, tgt, u != nullptr,
                 u, e != nullptr, e, 1, nullptr);
}

// ---------------------------------------------------------------------------
// ITER entry point (src/elfmm3dtria_iter_1.f:160-165).  The reference keeps
// the near-field operator in the caller's wsave array.  Here the operator
// stays in device memory owned by the library, and wsave holds an 8-word
// handle naming it:
//   [0] magic  [1] layout version  [2] store id  [3] nparts  [4] ntargs
//   [5] iprec  [6] geometry checksum  [7] layer/output flags
// At most ITER_SLOTS stores are live; a store call beyond that evicts the
// least recently used one, whose handle then fails validation (ier 512).
// ---------------------------------------------------------------------------
namespace {
constexpr double ITER_MAGIC = 1162626637.0;  // "ELFM"
constexpr double ITER_VERSION = 1.0;
constexpr int ITER_LUSED = 8;
constexpr int ITER_SLOTS = 4;

struct IterSlot {
  efmm_plan* p = nullptr;
  HostCall bufs;
  long long id = 0;
  long long last_use = 0;
  int n = 0, nt = 0, iprec = 0;
  double checksum = 0;
  int flags = 0;
};
std::vector<IterSlot*> g_iter;
long long g_iter_next_id = 1, g_iter_clock = 0;

// 64-bit FNV-1a over the geometry bytes, kept to 53 bits so it is exact in a double
// A 64-bit hash of the geometry arrays (a repeated call must bring the
// geometry its store was made for): the words of each array go round-robin
// into eight independent multiply-xorshift lanes (no serial chain through
// all the bytes: about a word per cycle), which are folded with the array
// lengths at the end.
double geometry_checksum(const double* tri, const double* nrm, const double* src, int n,
                         const double* tgt, int nt) {
  constexpr unsigned long long K = 0x9E3779B97F4A7C15ull;
  unsigned long long h[8];
  for (int l = 0; l < 8; l++) h[l] = 0x243F6A8885A308D3ull + (unsigned long long)l * K;
  auto mix = [&](const double* a, size_t cnt) {
    size_t i = 0;
    for (; i + 8 <= cnt; i += 8)
      for (int l = 0; l < 8; l++) {
        unsigned long long w;
        std::memcpy(&w, a + i + l, sizeof(w));
        h[l] = (h[l] ^ w) * K;
        h[l] ^= h[l] >> 29;
      }
    for (; i < cnt; i++) {
      unsigned long long w;
      std::memcpy(&w, a + i, sizeof(w));
      h[0] = (h[0] ^ w) * K;
      h[0] ^= h[0] >> 29;
    }
  };
  mix(tri, 9 * (size_t)n);
  mix(nrm, 3 * (size_t)n);
  mix(src, 3 * (size_t)n);
  if (nt > 0) mix(tgt, 3 * (size_t)nt);
  unsigned long long x = ((unsigned long long)(unsigned)n << 32) ^ (unsigned)nt;
  for (int l = 0; l < 8; l++) {
    x = (x ^ h[l]) * K;
    x ^= x >> 31;
  }
  return (double)(x >> 11);
}

IterSlot* iter_find(const double* wsave, int lwsave) {
  if (!wsave || lwsave < ITER_LUSED || wsave[0] != ITER_MAGIC || wsave[1] != ITER_VERSION) return nullptr;
  for (IterSlot* s : g_iter)
    if ((double)s->id == wsave[2]) return s;
  return nullptr;
}

IterSlot* iter_acquire(IterSlot* reuse) {
  if (reuse) return reuse;
  if ((int)g_iter.size() < ITER_SLOTS) {
    IterSlot* s = new IterSlot();
    s->p = efmm_plan_create(env_device());
    if (!s->p) {
      delete s;
      return nullptr;
    }
    g_iter.push_back(s);
    return s;
  }
  IterSlot* lru = g_iter[0];
  for (IterSlot* s : g_iter)
    if (s->last_use < lru->last_use) lru = s;
  return lru;
}

int iter_flags(int ifsingle, int ifdouble, int ifptfrc, int ifstrain, int nt, int ifptfrctarg,
               int ifstraintarg) {
  return (ifsingle ? 1 : 0) | (ifdouble ? 2 : 0) | (ifptfrc ? 4 : 0) | (ifstrain ? 8 : 0) |
         ((nt > 0 && ifptfrctarg) ? 16 : 0) | ((nt > 0 && ifstraintarg) ? 32 : 0);
}

int iter_call(int iprec, double rlam, double rmu, const double* tri, const double* nrm, int n,
              const double* src, int ifsingle, const double* ssl, int ifdouble, const double* sdl,
              int ifptfrc, double* ptfrc, int ifstrain, double* strain, int nt, const double* tgt,
              int ifptfrctarg, double* ptfrctarg, int ifstraintarg, double* straintarg, int icomp,
              double* wsave, int lwsave, int* lused) {
  *lused = ITER_LUSED;
  if (n < 1 || nt < 0) return IER_BADARG;
  if (icomp == 0) return IER_OK;  // the reference evaluates nothing for icomp_type 0
  if (icomp < 1 || icomp > 5) return IER_BADARG;
  // a work array too short for the handle: plain evaluation, as the reference
  // does when wsave cannot hold the stored interactions
  bool storing = (icomp == 2 || icomp == 3 || icomp == 5) && lwsave >= ITER_LUSED && wsave;
  if (icomp == 1 || ((icomp == 2 || icomp == 3) && !storing))
    return host_call(iprec, rlam, rmu, tri, nrm, n, src, ifsingle, ssl, ifdouble, sdl, ifptfrc, ptfrc,
                     ifstrain, strain, nt, tgt, ifptfrctarg, ptfrctarg, ifstraintarg, straintarg, false,
                     true);
  if (icomp == 5 && !storing) return IER_BADARG;
  std::lock_guard<std::mutex> lk(g_mu);
  const int flags = iter_flags(ifsingle, ifdouble, ifptfrc, ifstrain, nt, ifptfrctarg, ifstraintarg);
  IterSlot* S = iter_find(wsave, lwsave);
  double cks = geometry_checksum(tri, nrm, src, n, tgt, nt);
  if (icomp == 3) {
    if (!S || S->n != n || S->nt != nt || S->iprec != iprec || S->checksum != cks || S->flags != flags ||
        wsave[3] != n || wsave[4] != nt || wsave[5] != iprec || wsave[6] != cks || wsave[7] != flags)
      return IER_HANDLE;
  } else {
    S = iter_acquire(S);
    if (!S) return IER_NODEVICE;
    S->id = 0;  // invalid until this store completes
  }
  S->last_use = ++g_iter_clock;
  efmm_plan* p = S->p;
  try {
    cudaSetDevice(p->device);
    HostCall& B = S->bufs;
    cudaStream_t st = p->stream;
    if (icomp != 3) {
      up(B.tri, tri, 9 * (size_t)n, st);
      up(B.nrm, nrm, 3 * (size_t)n, st);
      up(B.src, src, 3 * (size_t)n, st);
      up(B.tgt, tgt, 3 * (size_t)nt, st);
      int ier = p->plan->set_geometry(n, B.tri.get(), B.nrm.get(), B.src.get(), nt, B.tgt.get(), iprec,
                                      true, false);
      if (ier) return ier;
      if (icomp == 4) return IER_OK;  // tree only
    }
    if (ifsingle) up(B.ssl, ssl, 3 * (size_t)n, st);
    if (ifdouble) up(B.sdl, sdl, 3 * (size_t)n, st);
    B.u.resize(3 * (size_t)n);
    B.e.resize(9 * (size_t)n);
    B.ut.resize(3 * (size_t)std::max(nt, 1));
    B.et.resize(9 * (size_t)std::max(nt, 1));
    bool src_out = ifptfrc || ifstrain, tgt_out = nt > 0 && (ifptfrctarg || ifstraintarg);
    int ier = p->plan->evaluate(rlam, rmu, ifsingle ? B.ssl.get() : nullptr, ifdouble ? B.sdl.get() : nullptr,
                                src_out ? B.u.get() : nullptr, ifstrain ? B.e.get() : nullptr,
                                tgt_out ? B.ut.get() : nullptr, (nt > 0 && ifstraintarg) ? B.et.get() : nullptr,
                                icomp == 3 ? 2 : 1, icomp != 5);
    if (ier) return ier;
    if (ifptfrc) down(ptfrc, B.u, 3 * (size_t)n, st);
    if (ifstrain) down(strain, B.e, 9 * (size_t)n, st);
    if (nt > 0 && ifptfrctarg) down(ptfrctarg, B.ut, 3 * (size_t)nt, st);
    if (nt > 0 && ifstraintarg) down(straintarg, B.et, 9 * (size_t)nt, st);
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
    if (icomp != 3) {
      S->id = g_iter_next_id++;
      S->n = n;
      S->nt = nt;
      S->iprec = iprec;
      S->checksum = cks;
      S->flags = flags;
      wsave[0] = ITER_MAGIC;
      wsave[1] = ITER_VERSION;
      wsave[2] = (double)S->id;
      wsave[3] = n;
      wsave[4] = nt;
      wsave[5] = iprec;
      wsave[6] = cks;
      wsave[7] = flags;
    }
    return IER_OK;
  } catch (const efmm::CudaError&) {
    return IER_CUDA;
  } catch (const std::bad_alloc&) {
    return IER_ALLOC;
  }
}
}  // namespace

extern "C" void elfmm3dtriatargiter_(int* ier, const int* iprec, const double* rlam, const double* rmu,
                                     const double* triangle, const double* trinorm, const int* nparts,
                                     const double* source, const int* ifsingle, const double* sigma_sl,
                                     const int* ifdouble, const double* sigma_dl, const int* ifptfrc,
                                     double* ptfrc, const int* ifstrain, double* strain,
                                     const int* ntargs, const double* target, const int* ifptfrctarg,
                                     double* ptfrctarg, const int* ifstraintarg, double* straintarg,
                                     const int* icomp_type, double* wsave, const int* lwsave, int* lused) {
  *ier = iter_call(*iprec, *rlam, *rmu, triangle, trinorm, *nparts, source, *ifsingle, sigma_sl, *ifdouble,
                   sigma_dl, *ifptfrc, ptfrc, *ifstrain, strain, *ntargs, target, *ifptfrctarg, ptfrctarg,
                   *ifstraintarg, straintarg, *icomp_type, wsave, *lwsave, lused);
}

extern "C" void elfmm3dtriaiter_(int* ier, const int* iprec, const double* rlam, const double* rmu,
                                 const double* triangle, const double* trinorm, const int* nparts,
                                 const double* source, const int* ifsingle, const double* sigma_sl,
                                 const int* ifdouble, const double* sigma_dl, const int* ifptfrc,
                                 double* ptfrc, const int* ifstrain, double* strain, const int* icomp_type,
                                 double* wsave, const int* lwsave, int* lused) {
  *ier = iter_call(*iprec, *rlam, *rmu, triangle, trinorm, *nparts, source, *ifsingle, sigma_sl, *ifdouble,
                   sigma_dl, *ifptfrc, ptfrc, *ifstrain, strain, 0, nullptr, 0, nullptr, 0, nullptr,
                   *icomp_type, wsave, *lwsave, lused);
}


// ---------------------------------------------------------------------------
// Half-space image part (elhfmm3dtriatargiter, src/elhfmm3dtria_iter.f:46-51)
// through the image FMM (Plan::evaluate_image) on the sources and the
// reflected targets.  icomp_type 1 evaluates, 2 evaluates and stores the
// image near-field blocks behind a wsave handle (as elfmm3dtriatargiter),
// 3 reuses them with new densities on the same geometry, 0 and 4 only return
// lused, 5 behaves as 2.  Sources and targets must lie in z <= 0.
// ---------------------------------------------------------------------------
namespace {
int hs_fmm_call(int iprec, double rlam, double rmu, const double* tri, const double* nrm, int n, const double* src,
                int ifsingle, const double* ssl, int ifdouble, const double* sdl, int nt, const double* tgt,
                int ifptfrctarg, double* ptfrctarg, int ifstraintarg, double* straintarg, int icomp,
                double* wsave, int lwsave, int* lused) {
  if (lused) *lused = ITER_LUSED;
  if (n < 1 || nt < 0) return IER_BADARG;
  if (iprec < -2 || iprec > 6) return IER_BADARG;
  if (icomp < 0 || icomp > 5) return IER_BADARG;
  if (icomp == 0 || icomp == 4 || nt == 0 || !(ifptfrctarg || ifstraintarg)) return IER_OK;
  for (int i = 0; i < 3 * n; i++)
    if (tri[3 * i + 2] > 0.0) return IER_BADARG;
  for (int i = 0; i < nt; i++)
    if (tgt[3 * i + 2] > 0.0) return IER_BADARG;
  const bool storing = (icomp == 2 || icomp == 3 || icomp == 5) && lwsave >= ITER_LUSED && wsave;
  const int mode = !storing ? 0 : (icomp == 3 ? 2 : 1);
  std::lock_guard<std::mutex> lk(g_mu);
  const int flags = iter_flags(ifsingle, ifdouble, 0, 0, nt, ifptfrctarg, ifstraintarg) | 64;
  const double cks = geometry_checksum(tri, nrm, src, n, tgt, nt);
  IterSlot* S = nullptr;
  efmm_plan* p = nullptr;
  HostCall* B = nullptr;
  if (mode == 0) {
    p = shared_plan();
    if (!p) return IER_NODEVICE;
    if (!g_bufs) g_bufs = new HostCall();
    B = g_bufs;
  } else {
    S = iter_find(wsave, lwsave);
    if (mode == 2) {
      if (!S || S->n != n || S->nt != nt || S->iprec != iprec || S->checksum != cks || S->flags != flags ||
          wsave[3] != n || wsave[4] != nt || wsave[5] != iprec || wsave[6] != cks || wsave[7] != flags)
        return IER_HANDLE;
    } else {
      S = iter_acquire(S);
      if (!S) return IER_NODEVICE;
      S->id = 0;  // invalid until this store completes
    }
    S->last_use = ++g_iter_clock;
    p = S->p;
    B = &S->bufs;
  }
  try {
    cudaSetDevice(p->device);
    cudaStream_t st = p->stream;
    if (mode != 2) {
      std::vector<double> refl(3 * (size_t)nt);
      for (int i = 0; i < nt; i++) {
        refl[3 * i] = tgt[3 * i];
        refl[3 * i + 1] = tgt[3 * i + 1];
        refl[3 * i + 2] = -tgt[3 * i + 2];
      }
      up(B->tri, tri, 9 * (size_t)n, st);
      up(B->nrm, nrm, 3 * (size_t)n, st);
      up(B->src, src, 3 * (size_t)n, st);
      up(B->tgt, refl.data(), 3 * (size_t)nt, st);
      const int ier = p->plan->set_geometry(n, B->tri.get(), B->nrm.get(), B->src.get(), nt, B->tgt.get(), iprec,
                                            true, true);
      if (ier) return ier;
    }
    if (ifsingle) up(B->ssl, ssl, 3 * (size_t)n, st);
    if (ifdouble) up(B->sdl, sdl, 3 * (size_t)n, st);
    B->ut.resize(3 * (size_t)nt);
    B->et.resize(9 * (size_t)nt);
    const int ier = p->plan->evaluate_image(rlam, rmu, 1, ifsingle ? B->ssl.get() : nullptr,
                                            ifdouble ? B->sdl.get() : nullptr, B->ut.get(),
                                            ifstraintarg ? B->et.get() : nullptr, 0, mode);
    if (ier) return ier;
    if (ifptfrctarg) down(ptfrctarg, B->ut, 3 * (size_t)nt, st);
    if (ifstraintarg) down(straintarg, B->et, 9 * (size_t)nt, st);
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
    if (mode == 1) {
      S->id = g_iter_next_id++;
      S->n = n;
      S->nt = nt;
      S->iprec = iprec;
      S->checksum = cks;
      S->flags = flags;
      wsave[0] = ITER_MAGIC;
      wsave[1] = ITER_VERSION;
      wsave[2] = (double)S->id;
      wsave[3] = n;
      wsave[4] = nt;
      wsave[5] = iprec;
      wsave[6] = cks;
      wsave[7] = flags;
    }
    return IER_OK;
  } catch (const efmm::CudaError&) {
    return IER_CUDA;
  } catch (const std::bad_alloc&) {
    return IER_ALLOC;
  }
}
}  // namespace

extern "C" void elhfmm3dtriatargiter_(int* ier, const int* iprec, const double* rlam, const double* rmu,
                                      const double* triangle, const double* trinorm, const int* nparts,
                                      const double* source, const int* ifsingle, const double* sigma_sl,
                                      const int* ifdouble, const double* sigma_dl, const int* ntargs,
                                      const double* target, const int* ifptfrctarg, double* ptfrctarg,
                                      const int* ifstraintarg, double* straintarg, const int* icomp_type,
                                      double* wsave, const int* lwsave, int* lused) {
  *ier = hs_fmm_call(*iprec, *rlam, *rmu, triangle, trinorm, *nparts, source, *ifsingle, sigma_sl, *ifdouble,
                     sigma_dl, *ntargs, target, *ifptfrctarg, ptfrctarg, *ifstraintarg, straintarg, *icomp_type,
                     wsave, *lwsave, lused);
}

// ---------------------------------------------------------------------------
// Half-space total field: the direct arrival (free-space evaluation at the
// centroids, on-surface, and at the targets) plus the image part at the same
// points, the sum the reference's drivers form from two calls
// (examples/elhfmm3dtria_self_iter_dr.f:331-385).  The image part of the
// centroids and the targets is one image-FMM pass over both point sets.
// Sources and targets must lie in z <= 0 (ier 16, nothing evaluated).
// ---------------------------------------------------------------------------
namespace {
int hs_total_call(int iprec, double rlam, double rmu, const double* tri, const double* nrm, int n, const double* src,
                  int ifsingle, const double* ssl, int ifdouble, const double* sdl, int ifptfrc, double* ptfrc,
                  int ifstrain, double* strain, int nt, const double* tgt, int ifptfrctarg, double* ptfrctarg,
                  int ifstraintarg, double* straintarg) {
  if (n < 1 || nt < 0) return IER_BADARG;
  if (iprec < -2 || iprec > 6) return IER_BADARG;
  for (int i = 0; i < 3 * n; i++)
    if (tri[3 * i + 2] > 0.0) return IER_BADARG;
  for (int i = 0; i < n; i++)
    if (src[3 * i + 2] > 0.0) return IER_BADARG;
  for (int i = 0; i < nt; i++)
    if (tgt[3 * i + 2] > 0.0) return IER_BADARG;
  const bool on_src = ifptfrc || ifstrain;
  const bool on_tgt = nt > 0 && (ifptfrctarg || ifstraintarg);
  if (!on_src && !on_tgt) return IER_OK;
  int ier = host_call(iprec, rlam, rmu, tri, nrm, n, src, ifsingle, ssl, ifdouble, sdl, ifptfrc, ptfrc, ifstrain,
                      strain, nt, tgt, ifptfrctarg, ptfrctarg, ifstraintarg, straintarg, false);
  if (ier) return ier;
  const int ns = on_src ? n : 0;
  const int m = ns + (on_tgt ? nt : 0);
  std::vector<double> pts(3 * (size_t)m), ui(3 * (size_t)m), ei(9 * (size_t)m);
  if (on_src) std::copy(src, src + 3 * (size_t)n, pts.begin());
  if (on_tgt) std::copy(tgt, tgt + 3 * (size_t)nt, pts.begin() + 3 * (size_t)ns);
  const int want_u = (on_src && ifptfrc) || (on_tgt && ifptfrctarg);
  const int want_e = (on_src && ifstrain) || (on_tgt && ifstraintarg);
  ier = hs_fmm_call(iprec, rlam, rmu, tri, nrm, n, src, ifsingle, ssl, ifdouble, sdl, m, pts.data(), want_u,
                    ui.data(), want_e, ei.data(), 1, nullptr, 0, nullptr);
  if (ier) return ier;
  if (ifptfrc)
    for (size_t k = 0; k < 3 * (size_t)n; k++) ptfrc[k] += ui[k];
  if (ifstrain)
    for (size_t k = 0; k < 9 * (size_t)n; k++) strain[k] += ei[k];
  if (on_tgt && ifptfrctarg)
    for (size_t k = 0; k < 3 * (size_t)nt; k++) ptfrctarg[k] += ui[3 * (size_t)ns + k];
  if (on_tgt && ifstraintarg)
    for (size_t k = 0; k < 9 * (size_t)nt; k++) straintarg[k] += ei[9 * (size_t)ns + k];
  return IER_OK;
}
}  // namespace

extern "C" void elhfmm3dtria_total_(int* ier, const int* iprec, const double* rlam, const double* rmu,
                                    const double* triangle, const double* trinorm, const int* nparts,
                                    const double* source, const int* ifsingle, const double* sigma_sl,
                                    const int* ifdouble, const double* sigma_dl, const int* ifptfrc, double* ptfrc,
                                    const int* ifstrain, double* strain, const int* ntargs, const double* target,
                                    const int* ifptfrctarg, double* ptfrctarg, const int* ifstraintarg,
                                    double* straintarg) {
  *ier = hs_total_call(*iprec, *rlam, *rmu, triangle, trinorm, *nparts, source, *ifsingle, sigma_sl, *ifdouble,
                       sigma_dl, *ifptfrc, ptfrc, *ifstrain, strain, *ntargs, target, *ifptfrctarg, ptfrctarg,
                       *ifstraintarg, straintarg);
}

// ---------------------------------------------------------------------------
// Half-space self-evaluation of many right-hand sides from host arrays (no
// counterpart in the reference: its multi-slip use is a loop of
// elfmm3dtriatargiter + elhfmm3dtriatargiter call pairs, icomp_type 2 then 3,
// examples/elhfmm3dtria_self_iter_dr.f:222-385).  One slot holds the two
// plans (direct arrival on the centroids; image part on the reflected
// centroids, Mindlin root) and their device buffers; icomp_type 2 stores both
// near fields behind an 8-word handle in wsave, 3 replays them with new
// densities, each plan's pass replayed as one CUDA graph (nrhs <= 64).  One
// store is live at a time: a new store invalidates the previous handle.
// ---------------------------------------------------------------------------
namespace {
__global__ void k_add_into(size_t n, double* __restrict__ a, const double* __restrict__ b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    a[i] += b[i];
}

constexpr double HSB_MAGIC = 1162626642.0;  // "ELFR"

struct HsBatchSlot {
  efmm_plan* f = nullptr;
  efmm_plan* img = nullptr;
  DevBuf<double> tri, nrm, src, refl, ssl, sdl, uf, ef, ui, ei;
  long long id = 0;
  int n = 0, R = 0, iprec = 0, precision = 0, flags = 0;
  double checksum = 0;
};
HsBatchSlot* g_hsb = nullptr;
long long g_hsb_next = 1;

int hs_batch_host(int iprec, double rlam, double rmu, int n, const double* tri, const double* nrm,
                  const double* src, int R, const double* ssl, const double* sdl, double* u, double* e,
                  int precision, int icomp, double* wsave, int lwsave) {
  if (n < 1 || R < 1 || (!ssl && !sdl) || (!u && !e)) return IER_BADARG;
  if (iprec < -2 || iprec > 6 || precision < 0 || precision > 1) return IER_BADARG;
  if (icomp < 1 || icomp > 3) return IER_BADARG;
  if (icomp != 1 && (!wsave || lwsave < ITER_LUSED)) return IER_BADARG;
  for (int i = 0; i < 3 * n; i++)
    if (tri[3 * i + 2] > 0.0) return IER_BADARG;
  for (int i = 0; i < n; i++)
    if (src[3 * i + 2] > 0.0) return IER_BADARG;
  std::lock_guard<std::mutex> lk(g_mu);
  const int flags = (ssl ? 1 : 0) | (sdl ? 2 : 0) | (u ? 4 : 0) | (e ? 8 : 0) | (precision << 4);
  const double cks = geometry_checksum(tri, nrm, src, n, nullptr, 0);
  if (icomp == 3) {
    const HsBatchSlot* S = g_hsb;
    if (!S || S->id == 0 || wsave[0] != HSB_MAGIC || wsave[1] != ITER_VERSION || wsave[2] != (double)S->id ||
        S->n != n || S->R != R || S->iprec != iprec || S->checksum != cks || S->flags != flags ||
        wsave[3] != n || wsave[4] != R || wsave[5] != iprec || wsave[6] != cks || wsave[7] != flags)
      return IER_HANDLE;
  }
  if (!g_hsb) {
    HsBatchSlot* S = new HsBatchSlot();
    S->f = efmm_plan_create(env_device());
    S->img = efmm_plan_create(env_device());
    if (!S->f || !S->img) {
      efmm_plan_destroy(S->f);
      efmm_plan_destroy(S->img);
      delete S;
      return IER_NODEVICE;
    }
    g_hsb = S;
  }
  HsBatchSlot& S = *g_hsb;
  if (icomp != 3) S.id = 0;  // invalid until this store completes
  try {
    cudaSetDevice(S.f->device);
    cudaStream_t st = S.f->stream;
    const size_t N3 = 3 * (size_t)n * R, N9 = 9 * (size_t)n * R;
    if (icomp != 3) {
      std::vector<double> refl(src, src + 3 * (size_t)n);
      for (int i = 0; i < n; i++) refl[3 * i + 2] = -refl[3 * i + 2];
      up(S.tri, tri, 9 * (size_t)n, st);
      up(S.nrm, nrm, 3 * (size_t)n, st);
      up(S.src, src, 3 * (size_t)n, st);
      up(S.refl, refl.data(), 3 * (size_t)n, st);
      EFMM_CUDA_TRY(cudaStreamSynchronize(st));
      const bool iter = icomp == 2;
      int ier = S.f->plan->set_geometry(n, S.tri.get(), S.nrm.get(), S.src.get(), 0, nullptr, iprec, iter, false);
      if (ier) return ier;
      ier = S.img->plan->set_geometry(n, S.tri.get(), S.nrm.get(), S.src.get(), n, S.refl.get(), iprec, iter, true);
      if (ier) return ier;
      S.uf.resize(N3);
      S.ef.resize(N9);
      S.ui.resize(N3);
      S.ei.resize(N9);
    }
    if (ssl) up(S.ssl, ssl, N3, st);
    if (sdl) up(S.sdl, sdl, N3, st);
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
    const double* dssl = ssl ? S.ssl.get() : nullptr;
    const double* dsdl = sdl ? S.sdl.get() : nullptr;
    double* duf = S.uf.get();  // the image pass needs the displacement buffer for strain-only calls too
    double* def = e ? S.ef.get() : nullptr;
    double* dui = S.ui.get();
    double* dei = e ? S.ei.get() : nullptr;
    const int mode = icomp == 1 ? 0 : (icomp == 2 ? 1 : 2);
    int ier;
    if (mode == 2 && R <= 64) {
      ier = S.f->plan->evaluate_batch_graph(rlam, rmu, R, dssl, dsdl, duf, def, nullptr, nullptr, precision, 2);
      if (!ier) ier = S.img->plan->evaluate_image_graph(rlam, rmu, R, dssl, dsdl, dui, dei, precision);
    } else {
      ier = S.f->plan->evaluate_batch(rlam, rmu, R, dssl, dsdl, duf, def, nullptr, nullptr, precision, mode);
      if (!ier) ier = S.img->plan->evaluate_image(rlam, rmu, R, dssl, dsdl, dui, dei, precision, mode);
    }
    if (ier) return ier;
    EFMM_CUDA_TRY(cudaStreamSynchronize(S.img->stream));
    if (u) {
      k_add_into<<<592, 256, 0, st>>>(N3, duf, dui);
      count_launch();
      down(u, S.uf, N3, st);
    }
    if (e) {
      k_add_into<<<592, 256, 0, st>>>(N9, def, dei);
      count_launch();
      down(e, S.ef, N9, st);
    }
    EFMM_CUDA_TRY(cudaGetLastError());
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
    if (icomp == 2) {
      S.id = g_hsb_next++;
      S.n = n;
      S.R = R;
      S.iprec = iprec;
      S.precision = precision;
      S.checksum = cks;
      S.flags = flags;
      wsave[0] = HSB_MAGIC;
      wsave[1] = ITER_VERSION;
      wsave[2] = (double)S.id;
      wsave[3] = n;
      wsave[4] = R;
      wsave[5] = iprec;
      wsave[6] = cks;
      wsave[7] = flags;
    }
    return IER_OK;
  } catch (const efmm::CudaError&) {
    return IER_CUDA;
  } catch (const std::bad_alloc&) {
    return IER_ALLOC;
  }
}
}  // namespace

extern "C" int elhfmm3dtria_batch_host(int iprec, double rlam, double rmu, int n, const double* triangle,
                                       const double* trinorm, const double* source, int nrhs,
                                       const double* sigma_sl, const double* sigma_dl, double* ptfrc,
                                       double* strain, int precision, int icomp_type, double* wsave,
                                       int lwsave) {
  return hs_batch_host(iprec, rlam, rmu, n, triangle, trinorm, source, nrhs, sigma_sl, sigma_dl, ptfrc, strain,
                       precision, icomp_type, wsave, lwsave);
}

extern "C" int efmm_iter_release(const double* wsave, int lwsave) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (wsave && lwsave >= ITER_LUSED && wsave[0] == HSB_MAGIC) {  // an elhfmm3dtria_batch_host store
    if (!g_hsb || g_hsb->id == 0 || wsave[2] != (double)g_hsb->id) return IER_HANDLE;
    HsBatchSlot* S = g_hsb;
    g_hsb = nullptr;
    cudaSetDevice(S->f->device);
    efmm_plan* f = S->f;
    efmm_plan* img = S->img;
    delete S;  // frees the slot's device buffers
    efmm_plan_destroy(f);
    efmm_plan_destroy(img);
    return IER_OK;
  }
  IterSlot* S = iter_find(wsave, lwsave);
  if (!S) return IER_HANDLE;
  for (size_t i = 0; i < g_iter.size(); i++)
    if (g_iter[i] == S) g_iter.erase(g_iter.begin() + i);
  cudaSetDevice(S->p->device);
  efmm_plan* p = S->p;
  delete S;  // frees the host-call buffers on the plan's device
  efmm_plan_destroy(p);
  return IER_OK;
}

extern "C" long long efmm_iter_stored_bytes(const double* wsave, int lwsave) {
  std::lock_guard<std::mutex> lk(g_mu);
  IterSlot* S = iter_find(wsave, lwsave);
  if (!S) return -1;
  return 8 * S->p->plan->stored_doubles();
}

// Host evaluation of one (triangle, point) pair of the free-space analytic
// near field: the closed-form integrals and assembly of tri_integrals.cuh
// that the device near field runs, with the densities rotated into the
// triangle frame as the device does.  u[3] and e6[6] (xx yy zz xy xz yz) are
// overwritten.
extern "C" int efmm_pair_eval_host(double rlam, double rmu, const double* tri, const double* ssl, const double* sdl,
                                   const double* x, int self, double* u, double* e6) {
  if (!tri || !x || !u || !e6 || (!ssl && !sdl)) return IER_BADARG;
  TriFrame f;
  tri_frame(tri, f);
  const double* ax[3] = {f.e1, f.e2, f.e3};
  double sl[3] = {0, 0, 0}, dl[3] = {0, 0, 0};
  for (int c = 0; c < 3; c++) {
    if (ssl) sl[c] = ax[c][0] * ssl[0] + ax[c][1] * ssl[1] + ax[c][2] * ssl[2];
    if (sdl) dl[c] = ax[c][0] * sdl[0] + ax[c][1] * sdl[1] + ax[c][2] * sdl[2];
  }
  for (int c = 0; c < 3; c++) u[c] = 0.0;
  for (int c = 0; c < 6; c++) e6[c] = 0.0;
  pair_eval(f, sl, dl, ssl != nullptr, sdl != nullptr, true, x, self != 0, rlam, rmu, u, e6);
  return IER_OK;
}

// Host evaluation of the generated image kernels (mindlin_gen.cuh) that the
// image near field and the direct image sum integrate: the responses at
// target x to the three unit point forces (layer 0) or to the three unit
// displacement jumps with normal nrm (layer 1) at source s, 27 doubles (per
// direction: displacement, strain xx yy zz xy xz yz).
extern "C" int efmm_mindlin_image_kernel(int layer, double lam, double mu, const double* x, const double* s,
                                         const double* nrm, double* out) {
  if (!x || !s || !out || (layer == 1 && !nrm)) return IER_BADARG;
  if (layer == 0)
    mindlin_image_sl_blk(lam, mu, x[0], x[1], x[2], s[0], s[1], s[2], out);
  else if (layer == 1)
    mindlin_image_dl_blk(lam, mu, x[0], x[1], x[2], s[0], s[1], s[2], nrm[0], nrm[1], nrm[2], out);
  else
    return IER_BADARG;
  return IER_OK;
}

// Host check of the M2L of the half-space kernel U = z log(r + z) - r built
// from u_harmonics (the device operators use the same code): nsrc unit-box
// sources around 0 with random charges, targets in the unit box around the
// offset X; the local expansion of order p (multipole moments through the J
// table) against the direct sum of U.  Returns the largest relative error.
extern "C" double efmm_u_m2l_selfcheck(int p, double X0, double X1, double X2, int nsrc, unsigned seed) {
  using namespace efmm;
  if (p < 1 || p > 54 || nsrc < 1) return -1.0;
  unsigned long long st = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto uni = [&]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return ((st >> 11) * (1.0 / 9007199254740992.0)) - 0.5;
  };
  const int nc = ncoef(p);
  std::vector<cplx> Y(nc), M(nc, cplx{0, 0}), L(nc, cplx{0, 0}), J(ncoef(2 * p));
  std::vector<double> q(nsrc), xs(3 * (size_t)nsrc);
  for (int i = 0; i < nsrc; i++) {
    q[i] = 2 * uni();
    for (int d = 0; d < 3; d++) xs[3 * i + d] = uni();
    regular_harmonics(p, xs[3 * i], xs[3 * i + 1], xs[3 * i + 2], Y.data());
    for (int c = 0; c < nc; c++) M[c] = cadd(M[c], cscale(q[i], cconj(Y[c])));
  }
  u_harmonics(2 * p, X0, X1, X2, J.data());
  for (int n = 0; n <= p; n++)
    for (int m = 0; m <= n; m++) {
      cplx acc = {0, 0};
      for (int k = 0; k <= p; k++)
        for (int l = -k; l <= k; l++) acc = cadd(acc, cmul(m2l_coef(J.data(), n, m, k, l), hget(M.data(), k, l)));
      L[cidx(n, m)] = acc;
    }
  double worst = 0.0;
  for (int t = 0; t < 8; t++) {
    const double z[3] = {uni(), uni(), uni()};
    regular_harmonics(p, z[0], z[1], z[2], Y.data());
    double val = 0.0;
    for (int n = 0; n <= p; n++)
      for (int m = -n; m <= n; m++) {
        const cplx a = hget(L.data(), n, m), y = cconj(hget(Y.data(), n, m));
        val += a.re * y.re - a.im * y.im;
      }
    double ref = 0.0;
    for (int i = 0; i < nsrc; i++) {
      const double r[3] = {X0 + z[0] - xs[3 * i], X1 + z[1] - xs[3 * i + 1], X2 + z[2] - xs[3 * i + 2]};
      const double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      ref += q[i] * (r[2] * log(rr + r[2]) - rr);
    }
    worst = std::max(worst, fabs(val - ref) / fabs(ref));
  }
  return worst;
}
