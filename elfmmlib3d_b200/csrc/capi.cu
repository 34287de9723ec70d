// capi.cu -- extern "C" entry points (include/elfmm3d_b200.h).
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>
#include "plan.h"
#include "../../include/elfmm3d_b200.h"

using namespace efmm;

struct efmm_plan {
  int device;
  cudaStream_t stream;
  std::unique_ptr<Plan> plan;
  cudaEvent_t user_ev[8];
};

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
              int ifptfrctarg, double* ptfrctarg, int ifstraintarg, double* straintarg, bool direct) {
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
                                    iprec, false, false);
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
