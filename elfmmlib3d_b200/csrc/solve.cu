// solve.cu -- the iterative solver loop over the layer-potential operator.
//
// The reference's iterative solvers are MATLAB functions over a function
// handle (matlab/gmres_simple.m, matlab/bicgstab_simple.m, listed in
// matlab/Contents.m:32-33); ITER mode exists so that repeated operator
// applications reuse the stored near field.  Here the minimal-residual
// iteration of gmres_simple runs on the device for many right-hand sides at
// once, each column with its own coefficients, over the plans' stored near
// fields (mode 2, each pass replayed as a CUDA graph):
//   x = 0, r = b;  for i = 1, 2, ...:
//     every 10th step r = b - A x;  w = A r;
//     (wp, rp) = (w, r) orthogonalised against the earlier (Ae_j, e_j) by
//     the Ae_j (modified Gram-Schmidt), scaled by 1 / |wp|, orthogonalised
//     and scaled once more: the new (Ae_i, e_i);
//     d = Ae_i . r,  r -= d Ae_i;  stop (ier 8) if |r| did not decrease,
//     else x += d e_i;  converged when |r| < tol |b|.
// Without convergence in maxit steps ier = 4, as the reference.
//
// Operators (kind): 0 the traction t = (lam tr(e) I + 2 mu e) n at the
// centroids of the double layer of the density (the displacement
// discontinuity of a fault: the slip that carries a given traction); 1 the
// displacement at the centroids of the single layer.  With an image plan,
// the half-space operator (direct arrival + image part).
//
// The same iteration runs on host vectors for a dense matrix
// (efmm_gcr_dense_host), the CPU check of the algorithm.
#include <algorithm>
#include <cmath>
#include <vector>
#include "common.cuh"
#include "plan.h"
#include "solve.h"

namespace efmm {

namespace {

// per-column dot products: out[c] += sum_k a[c L + k] b[c L + k] (out zeroed by the caller)
__global__ void k_coldot(int L, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out) {
  const int c = blockIdx.y;
  const double* ac = a + (size_t)c * L;
  const double* bc = b + (size_t)c * L;
  double s = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < L; k += gridDim.x * blockDim.x) s += ac[k] * bc[k];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double ws[32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) atomicAdd(out + c, s);
  }
}

// y[c] += sgn coef[c] x[c] for the columns with mask[c] != 0 (mask may be null)
__global__ void k_colaxpy(int L, double sgn, const double* __restrict__ coef, const int* __restrict__ mask,
                          const double* __restrict__ x, double* __restrict__ y) {
  const int c = blockIdx.y;
  if (mask && !mask[c]) return;
  const double a = sgn * coef[c];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < L; k += gridDim.x * blockDim.x)
    y[(size_t)c * L + k] += a * x[(size_t)c * L + k];
}

// y[c] = x[c] / sqrt(ss[c]) (a zero column stays zero)
__global__ void k_colscale(int L, const double* __restrict__ ss, const double* __restrict__ x, double* __restrict__ y) {
  const int c = blockIdx.y;
  const double s = ss[c] > 0.0 ? 1.0 / sqrt(ss[c]) : 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < L; k += gridDim.x * blockDim.x)
    y[(size_t)c * L + k] = s * x[(size_t)c * L + k];
}

__global__ void k_sub(size_t n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ y) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    y[k] = a[k] - b[k];
}

__global__ void k_add(size_t n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ y) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    y[k] = a[k] + b[k];
}

// traction (lam tr(e) I + 2 mu e) n per column and centroid from the strain
// e (R, n, 3, 3) plus an optional second strain (the image part)
__global__ void k_traction(int R, int n, const double* __restrict__ nrm, const double* __restrict__ e,
                           const double* __restrict__ e2, double lam, double mu, double* __restrict__ t) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)R * n) return;
  const int tri = (int)(i % n);
  double E[9];
  for (int k = 0; k < 9; k++) E[k] = e[9 * i + k] + (e2 ? e2[9 * i + k] : 0.0);
  const double tr = E[0] + E[4] + E[8];
  const double* nv = nrm + 3 * (size_t)tri;
  for (int a = 0; a < 3; a++) {
    double s = lam * tr * nv[a];
    for (int b = 0; b < 3; b++) s += 2.0 * mu * E[3 * a + b] * nv[b];
    t[3 * i + a] = s;
  }
}

constexpr int COL_THREADS = 256;
inline dim3 col_grid(int L, int R) { return dim3((unsigned)std::min(64, (L + COL_THREADS - 1) / COL_THREADS), R); }

// Device vectors: R columns of L doubles each; coefficients on the device.
struct DevBackend {
  int R, L;
  cudaStream_t st;
  std::function<int(const double*, double*)> apply;  // A on R columns (device)
  DevBuf<double> coef, ss;
  DevBuf<int> mask;
  std::vector<double> hbuf;
  void init() {
    coef.resize(R);
    ss.resize(R);
    mask.resize(R);
    hbuf.resize(R);
  }
  double* cp() { return coef.get(); }
  double* sp() { return ss.get(); }
  int* mp() { return mask.get(); }
  void dots(const double* a, const double* b, double* out) {
    EFMM_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double) * R, st));
    k_coldot<<<col_grid(L, R), COL_THREADS, 0, st>>>(L, a, b, out);
    count_launch();
  }
  void axpy(double sgn, const double* c, const int* m, const double* x, double* y) {
    k_colaxpy<<<col_grid(L, R), COL_THREADS, 0, st>>>(L, sgn, c, m, x, y);
    count_launch();
  }
  void scale(const double* s, const double* x, double* y) {
    k_colscale<<<col_grid(L, R), COL_THREADS, 0, st>>>(L, s, x, y);
    count_launch();
  }
  void copy(const double* x, double* y) {
    EFMM_CUDA_TRY(cudaMemcpyAsync(y, x, sizeof(double) * R * (size_t)L, cudaMemcpyDeviceToDevice, st));
  }
  void zero(double* x) { EFMM_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(double) * R * (size_t)L, st)); }
  void sub(const double* a, const double* b, double* y) {
    k_sub<<<592, 256, 0, st>>>((size_t)R * L, a, b, y);
    count_launch();
  }
  std::vector<double> norms(const double* x) {  // |x_c| on the host
    dots(x, x, ss.get());
    EFMM_CUDA_TRY(cudaMemcpyAsync(hbuf.data(), ss.get(), sizeof(double) * R, cudaMemcpyDeviceToHost, st));
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<double> out(R);
    for (int c = 0; c < R; c++) out[c] = std::sqrt(std::max(hbuf[c], 0.0));
    return out;
  }
  void set_mask(const std::vector<int>& m) {
    EFMM_CUDA_TRY(cudaMemcpyAsync(mask.get(), m.data(), sizeof(int) * R, cudaMemcpyHostToDevice, st));
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));  // m is a host temporary
  }
  double* vec_alloc(DevBuf<double>& b) {
    b.resize((size_t)R * L);
    return b.get();
  }
};

// Host vectors (the dense CPU check): the same interface.
struct HostBackend {
  int R, L;
  std::function<int(const double*, double*)> apply;
  std::vector<double> coef, ss;
  std::vector<int> mask;
  void init() {
    coef.assign(R, 0.0);
    ss.assign(R, 0.0);
    mask.assign(R, 0);
  }
  double* cp() { return coef.data(); }
  double* sp() { return ss.data(); }
  int* mp() { return mask.data(); }
  void dots(const double* a, const double* b, double* out) {
    for (int c = 0; c < R; c++) {
      double s = 0.0;
      for (int k = 0; k < L; k++) s += a[(size_t)c * L + k] * b[(size_t)c * L + k];
      out[c] = s;
    }
  }
  void axpy(double sgn, const double* cf, const int* m, const double* x, double* y) {
    for (int c = 0; c < R; c++)
      if (!m || m[c])
        for (int k = 0; k < L; k++) y[(size_t)c * L + k] += sgn * cf[c] * x[(size_t)c * L + k];
  }
  void scale(const double* s, const double* x, double* y) {
    for (int c = 0; c < R; c++) {
      const double f = s[c] > 0.0 ? 1.0 / std::sqrt(s[c]) : 0.0;
      for (int k = 0; k < L; k++) y[(size_t)c * L + k] = f * x[(size_t)c * L + k];
    }
  }
  void copy(const double* x, double* y) { std::copy(x, x + (size_t)R * L, y); }
  void zero(double* x) { std::fill(x, x + (size_t)R * L, 0.0); }
  void sub(const double* a, const double* b, double* y) {
    for (size_t k = 0; k < (size_t)R * L; k++) y[k] = a[k] - b[k];
  }
  std::vector<double> norms(const double* x) {
    dots(x, x, ss.data());
    std::vector<double> out(R);
    for (int c = 0; c < R; c++) out[c] = std::sqrt(std::max(ss[c], 0.0));
    return out;
  }
  void set_mask(const std::vector<int>& m) { mask = m; }
};

// The iteration (matlab/gmres_simple.m), generic over the vector backend:
// b (right-hand sides), x (solution), work vectors r, w, wp, rp, and the
// directions ae[i], e[i] (i < maxit), all R columns of L.  Returns per
// column ier (0 converged, 4 maxit reached, 8 the residual stopped
// decreasing), iterations and |r| / |b|; the function's value is the first
// nonzero status of an operator application (0 if none).
template <class B>
int gcr_run(B& be, const double* b, double* x, double* r, double* w, double* wp, double* rp,
            const std::vector<double*>& ae, const std::vector<double*>& e, double tol, int maxit,
            std::vector<int>& ier, std::vector<int>& its, std::vector<double>& relres) {
  const int R = be.R;
  ier.assign(R, 4);
  its.assign(R, 0);
  relres.assign(R, 1.0);
  be.zero(x);
  be.copy(b, r);
  const std::vector<double> nb = be.norms(b);
  std::vector<double> er0 = nb;
  std::vector<int> active(R);
  int nact = 0;
  for (int c = 0; c < R; c++) {
    active[c] = nb[c] > 0.0;
    if (!active[c]) {
      ier[c] = 0;
      relres[c] = 0.0;
    }
    nact += active[c];
  }
  for (int i = 0; i < maxit && nact > 0; i++) {
    if ((i + 1) % 10 == 0) {  // recompute the residual every 10 steps
      int st = be.apply(x, w);
      if (st) return st;
      be.sub(b, w, r);
    }
    int st = be.apply(r, w);
    if (st) return st;
    be.copy(w, wp);
    be.copy(r, rp);
    for (int j = 0; j < i; j++) {
      be.dots(ae[j], wp, be.cp());
      be.axpy(-1.0, be.cp(), nullptr, ae[j], wp);
      be.axpy(-1.0, be.cp(), nullptr, e[j], rp);
    }
    be.dots(wp, wp, be.sp());
    be.scale(be.sp(), wp, ae[i]);
    be.scale(be.sp(), rp, e[i]);
    // orthogonalise once more
    for (int j = 0; j < i; j++) {
      be.dots(ae[j], ae[i], be.cp());
      be.axpy(-1.0, be.cp(), nullptr, ae[j], ae[i]);
      be.axpy(-1.0, be.cp(), nullptr, e[j], e[i]);
    }
    be.dots(ae[i], ae[i], be.sp());
    be.scale(be.sp(), ae[i], ae[i]);
    be.scale(be.sp(), e[i], e[i]);
    // residual and solution updates of the active columns
    be.set_mask(active);
    be.dots(ae[i], r, be.cp());
    be.axpy(-1.0, be.cp(), be.mp(), ae[i], r);
    const std::vector<double> er1 = be.norms(r);
    std::vector<int> upd(R, 0);
    for (int c = 0; c < R; c++) {
      if (!active[c]) continue;
      its[c] = i + 1;
      if (!(er1[c] < er0[c])) {  // the residual stopped decreasing: stop this column
        ier[c] = 8;
        active[c] = 0;
        nact--;
        continue;
      }
      er0[c] = er1[c];
      relres[c] = er1[c] / nb[c];
      upd[c] = 1;
    }
    be.set_mask(upd);
    be.axpy(1.0, be.cp(), be.mp(), e[i], x);
    for (int c = 0; c < R; c++)
      if (upd[c] && er1[c] < tol * nb[c]) {
        ier[c] = 0;
        active[c] = 0;
        nact--;
      }
  }
  return 0;
}

}  // namespace

int solve_layers(Plan* F, Plan* I, int kind, double rlam, double rmu, int R, const double* d_nrm,
                 const double* d_rhs, double* d_x, double tol, int maxit, int precision, int* iters,
                 double* relres, int* ier_cols) {
  if (!F || (kind != 0 && kind != 1) || R < 1 || maxit < 1 || !(tol > 0) || !d_rhs || !d_x) return IER_BADARG;
  if (kind == 0 && !d_nrm) return IER_BADARG;
  const int n = F->n();
  if (n < 1 || (I && I->n() != n) || (I && I->nt() != n)) return IER_BADARG;
  const size_t L = 3 * (size_t)n;
  DevBackend be;
  be.R = R;
  be.L = (int)L;
  be.st = F->stream();
  be.init();
  DevBuf<double> vb, vx, vr, vw, vwp, vrp, vin, vu, ve, vui, vei;
  std::vector<DevBuf<double>> vae(maxit), ve_(maxit);
  std::vector<double*> ae(maxit), e(maxit);
  for (int i = 0; i < maxit; i++) {
    ae[i] = be.vec_alloc(vae[i]);
    e[i] = be.vec_alloc(ve_[i]);
  }
  double* b = be.vec_alloc(vb);
  double* x = be.vec_alloc(vx);
  double* r = be.vec_alloc(vr);
  double* w = be.vec_alloc(vw);
  double* wp = be.vec_alloc(vwp);
  double* rp = be.vec_alloc(vrp);
  double* in = be.vec_alloc(vin);  // the operator's fixed input buffer (graph replays)
  double* u = be.vec_alloc(vu);
  double* ui = I ? be.vec_alloc(vui) : nullptr;
  double* es = nullptr;
  double* esi = nullptr;
  if (kind == 0) {
    ve.resize(3 * (size_t)R * L);
    es = ve.get();
    if (I) {
      vei.resize(3 * (size_t)R * L);
      esi = vei.get();
    }
  }
  EFMM_CUDA_TRY(cudaMemcpyAsync(b, d_rhs, sizeof(double) * R * L, cudaMemcpyDeviceToDevice, be.st));
  // A on R columns: the plans' stored near fields (the first application
  // stores them when a plan holds none for these layers and outputs)
  bool first = true;
  be.apply = [&](const double* src, double* dst) -> int {
    EFMM_CUDA_TRY(cudaMemcpyAsync(in, src, sizeof(double) * R * L, cudaMemcpyDeviceToDevice, be.st));
    EFMM_CUDA_TRY(cudaStreamSynchronize(be.st));
    const double* ssl = kind == 1 ? in : nullptr;
    const double* sdl = kind == 0 ? in : nullptr;
    const bool graph = !first && R <= 64;
    int ier;
    auto run = [&](int mode) {
      int q;
      if (graph)
        q = F->evaluate_batch_graph(rlam, rmu, R, ssl, sdl, u, es, nullptr, nullptr, precision, mode);
      else
        q = F->evaluate_batch(rlam, rmu, R, ssl, sdl, u, es, nullptr, nullptr, precision, mode);
      if (q || !I) return q;
      if (graph) return I->evaluate_image_graph(rlam, rmu, R, ssl, sdl, ui, esi, precision);
      return I->evaluate_image(rlam, rmu, R, ssl, sdl, ui, esi, precision, mode);
    };
    if (first) {
      const bool stored = F->store_valid() && (!I || I->store_valid());
      ier = stored ? run(2) : IER_HANDLE;
      if (ier == IER_HANDLE) ier = run(1);
      first = false;
    } else {
      ier = run(2);
    }
    if (ier) return ier;
    if (I) EFMM_CUDA_TRY(cudaStreamSynchronize(I->stream()));
    if (kind == 0) {
      const size_t rn = (size_t)R * n;
      k_traction<<<(unsigned)((rn + 255) / 256), 256, 0, be.st>>>(R, n, d_nrm, es, esi, rlam, rmu, dst);
      count_launch();
    } else if (I) {
      k_add<<<592, 256, 0, be.st>>>((size_t)R * L, u, ui, dst);
      count_launch();
    } else {
      be.copy(u, dst);
    }
    EFMM_CUDA_TRY(cudaGetLastError());
    return IER_OK;
  };
  std::vector<int> ier, its;
  std::vector<double> rel;
  const int st = gcr_run(be, b, x, r, w, wp, rp, ae, e, tol, maxit, ier, its, rel);
  if (st) return st;
  EFMM_CUDA_TRY(cudaMemcpyAsync(d_x, x, sizeof(double) * R * L, cudaMemcpyDeviceToDevice, be.st));
  EFMM_CUDA_TRY(cudaStreamSynchronize(be.st));
  for (int c = 0; c < R; c++) {
    if (iters) iters[c] = its[c];
    if (relres) relres[c] = rel[c];
    if (ier_cols) ier_cols[c] = ier[c];
  }
  return IER_OK;
}

}  // namespace efmm

// The iteration on host vectors for a dense matrix A (n x n, row-major):
// R right-hand sides B (R, n) -> X (R, n).  The CPU check of the algorithm.
extern "C" int efmm_gcr_dense_host(int n, int R, const double* A, const double* Bm, double* X, double tol, int maxit,
                                   int* iters, double* relres, int* ier_cols) {
  using namespace efmm;
  if (n < 1 || R < 1 || maxit < 1 || !A || !Bm || !X) return IER_BADARG;
  HostBackend be;
  be.R = R;
  be.L = n;
  be.init();
  be.apply = [&](const double* src, double* dst) -> int {
    for (int c = 0; c < R; c++)
      for (int i = 0; i < n; i++) {
        double s = 0.0;
        for (int k = 0; k < n; k++) s += A[(size_t)i * n + k] * src[(size_t)c * n + k];
        dst[(size_t)c * n + i] = s;
      }
    return 0;
  };
  const size_t sz = (size_t)R * n;
  std::vector<double> x(sz), r(sz), w(sz), wp(sz), rp(sz);
  std::vector<std::vector<double>> vae(maxit, std::vector<double>(sz)), ve(maxit, std::vector<double>(sz));
  std::vector<double*> ae(maxit), e(maxit);
  for (int i = 0; i < maxit; i++) {
    ae[i] = vae[i].data();
    e[i] = ve[i].data();
  }
  std::vector<int> ier, its;
  std::vector<double> rel;
  gcr_run(be, Bm, x.data(), r.data(), w.data(), wp.data(), rp.data(), ae, e, tol, maxit, ier, its, rel);
  std::copy(x.begin(), x.end(), X);
  for (int c = 0; c < R; c++) {
    if (iters) iters[c] = its[c];
    if (relres) relres[c] = rel[c];
    if (ier_cols) ier_cols[c] = ier[c];
  }
  return 0;
}
