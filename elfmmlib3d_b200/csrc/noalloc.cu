// noalloc.cu -- direct sum entry point that allocates no device memory.
//
// Some callers cannot allocate device memory at the point where they need the
// answer: a solver whose memory pool has already reserved the GPU's free
// memory (cudaMalloc would fail there), or a latency-sensitive loop where an
// allocation (and the device synchronisation cudaFree implies) is not
// acceptable.  For them efmm_direct_noalloc evaluates the same O(N^2) analytic
// direct sum as el3dtriadirecttarg_, with the caller providing inputs and
// outputs in device memory and all intermediate data held in fixed-size
// scratch arrays at file scope below.  Those arrays (about 11 MB) stay on a GPU
// for the life of the process once this file's module is loaded there.  Under
// CUDA's lazy module loading (the default since CUDA 12) that happens at the
// first call on the device, which therefore must come before the caller's pool
// reserves the free memory (a call with one triangle is enough).
#include <mutex>
#include "common.cuh"
#include "kernels.h"

namespace efmm {

constexpr int NOALLOC_MAX_TRI = 32768;  // triangles per call
constexpr int NOALLOC_MAX_PTS = 65536;  // evaluation points per call (centroids + targets)

// Scratch shared by every call on a device; it keeps the last call's
// contents.  Every entry a call reads is written earlier in the same call.
static __device__ __align__(256) TriRec g_noalloc_tri[NOALLOC_MAX_TRI];
static __device__ __align__(256) double g_noalloc_u[3 * NOALLOC_MAX_PTS];
static __device__ __align__(256) double g_noalloc_e[6 * NOALLOC_MAX_PTS];

// Device addresses of the scratch arrays, looked up once per device.  In host
// code the array names above stand for host-side shadows, not device
// addresses, so the kernels must be given these looked-up pointers.  They
// belong to the device's primary context: after cudaDeviceReset they are
// stale, and the entry point must not be used again in that process.
struct NoallocPtrs {
  TriRec* tri;
  double* u;
  double* e;
  bool ready;
};
static std::mutex g_noalloc_mu;
static NoallocPtrs g_noalloc_ptrs[64];

static int noalloc_setup(int dev, NoallocPtrs& out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (dev < 0 || dev >= 64) return IER_BADARG;
  NoallocPtrs& p = g_noalloc_ptrs[dev];
  if (!p.ready) {
    // the device is current here (cudaGetDevice returned it)
    if (cudaGetSymbolAddress((void**)&p.tri, g_noalloc_tri) != cudaSuccess) return IER_CUDA;
    if (cudaGetSymbolAddress((void**)&p.u, g_noalloc_u) != cudaSuccess) return IER_CUDA;
    if (cudaGetSymbolAddress((void**)&p.e, g_noalloc_e) != cudaSuccess) return IER_CUDA;
    p.ready = true;
  }
  out = p;
  return IER_OK;
}

// scratch (3 displacement + 6 symmetric strain per point) -> caller outputs
// (3 per point, 3x3 per point); null outputs are skipped
__global__ void k_noalloc_out(int n, const double* __restrict__ u6, const double* __restrict__ e6,
                              double* __restrict__ uo, double* __restrict__ eo) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (uo)
    for (int c = 0; c < 3; c++) uo[3 * (size_t)i + c] = u6[3 * (size_t)i + c];
  if (eo) {
    const double* s = e6 + 6 * (size_t)i;
    double* o = eo + 9 * (size_t)i;
    o[0] = s[0]; o[4] = s[1]; o[8] = s[2];
    o[1] = o[3] = s[3];
    o[2] = o[6] = s[4];
    o[5] = o[7] = s[5];
  }
}

}  // namespace efmm

using namespace efmm;

// See include/elfmm3d_b200.h.  Enqueues on `stream` and returns; the outputs
// are complete when the stream reaches that point.  The first call on a device
// looks up the scratch addresses for that device (make it before any stream
// capture and before a memory pool reserves the free memory).  Calls that
// overlap on the GPU (different streams or host threads, same device) share
// the scratch and race.  A launch error left pending by earlier work of the
// calling thread is not consumed: the call returns IER_CUDA without running.
extern "C" int efmm_direct_noalloc(double rlam, double rmu, int n, const double* tri,
                                   const double* src, const double* ssl, const double* sdl, int nt,
                                   const double* tgt, double* u_src, double* e_src, double* u_tgt,
                                   double* e_tgt, void* stream) {
  if (n < 1 || nt < 0) return IER_BADARG;
  if (n > NOALLOC_MAX_TRI || (long long)n + nt > NOALLOC_MAX_PTS) {
    fprintf(stderr,
            "efmm_direct_noalloc: %d triangles and %d targets exceed the fixed scratch "
            "(at most %d triangles and %d evaluation points per call)\n",
            n, nt, NOALLOC_MAX_TRI, NOALLOC_MAX_PTS);
    return IER_BADARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return IER_NODEVICE;
  if (cudaPeekAtLastError() != cudaSuccess) return IER_CUDA;
  NoallocPtrs S;
  int ier = noalloc_setup(dev, S);
  if (ier) return ier;
  cudaStream_t st = (cudaStream_t)stream;
  int dosl = ssl != nullptr, dodl = sdl != nullptr;
  int do_src = (u_src || e_src) ? n : 0;
  int do_tgt = (nt > 0 && (u_tgt || e_tgt)) ? nt : 0;
  try {
    launch_tri_prep(st, n, tri, nullptr, ssl, sdl, dosl, dodl, S.tri);
    launch_direct_all(st, n, S.tri, do_src, src, do_tgt, tgt, dosl, dodl, e_src ? 1 : 0,
                      e_tgt ? 1 : 0, rlam, rmu, S.u, S.e, S.u + 3 * (size_t)n, S.e + 6 * (size_t)n);
    if (do_src) {
      k_noalloc_out<<<(n + 255) / 256, 256, 0, st>>>(n, S.u, S.e, u_src, e_src); count_launch();
    }
    if (do_tgt) {
      k_noalloc_out<<<(nt + 255) / 256, 256, 0, st>>>(nt, S.u + 3 * (size_t)n, S.e + 6 * (size_t)n,
                                                       u_tgt, e_tgt); count_launch();
    }
  } catch (const efmm::CudaError&) {
    return IER_CUDA;
  }
  if (cudaGetLastError() != cudaSuccess) return IER_CUDA;
  return IER_OK;
}
