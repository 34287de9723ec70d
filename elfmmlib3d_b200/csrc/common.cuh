// common.cuh -- shared definitions for the sm_100a kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "tri_integrals.cuh"
#include "harmonics.cuh"

namespace efmm {

// Error codes returned through ier.  0/4/8/16 follow the reference
// (src/lfmm3dtrilhess.f:163-169, src/elhfmm3dtria_iter.f:126-131); codes >= 256
// are this library's own.
enum : int {
  IER_OK = 0,
  IER_TREE = 4,          // tree construction failed (reference: allocation retries exhausted)
  IER_ALLOC = 8,         // device allocation failure
  IER_BADARG = 16,       // invalid argument (n < 1, unsupported iprec, ...)
  IER_CUDA = 256,        // CUDA runtime error
  IER_HANDLE = 512,      // stored-operator handle missing or geometry mismatch
  IER_NODEVICE = 1024,   // no CUDA device available
};

// Symmetric 12-point rule of degree 6 on the triangle (barycentric orbits),
// weights normalised to sum 1.  Solved to 25 digits from the moment equations
// (the rule the reference's order-6 triasymq table realises, triasymq.f:40-52).
struct Quad12 {
  double b[12][3];
  double w[12];
};
__host__ __device__ inline void quad12(Quad12& q) {
  const double a1 = 0.2492867451709104212916386, w1 = 0.1167862757263793660252896;
  const double a2 = 0.0630890144915022283403316, w2 = 0.05084490637020681692093681;
  const double b3 = 0.05314504984481694735324967, c3 = 0.3103524510337844054166077,
               w3 = 0.08285107561837357519355346;
  const double d3 = 1.0 - b3 - c3;
  double aa[2] = {a1, a2}, ww[2] = {w1, w2};
  int k = 0;
  for (int o = 0; o < 2; o++) {
    double a = aa[o], e = 1.0 - 2.0 * a;
    double t[3][3] = {{a, a, e}, {a, e, a}, {e, a, a}};
    for (int i = 0; i < 3; i++, k++) {
      q.b[k][0] = t[i][0]; q.b[k][1] = t[i][1]; q.b[k][2] = t[i][2];
      q.w[k] = ww[o];
    }
  }
  double t6[6][3] = {{b3, c3, d3}, {b3, d3, c3}, {c3, b3, d3}, {c3, d3, b3}, {d3, b3, c3}, {d3, c3, b3}};
  for (int i = 0; i < 6; i++, k++) {
    q.b[k][0] = t6[i][0]; q.b[k][1] = t6[i][1]; q.b[k][2] = t6[i][2];
    q.w[k] = w3;
  }
}

// Per-triangle record used by the near-field kernels (tree order).
// 24 doubles = 192 bytes, 16-byte aligned for vector loads.
struct __align__(16) TriRec {
  TriFrame f;        // 16 doubles
  double ssl[3];     // single-layer density in the triangle frame
  double sdl[3];     // double-layer density in the triangle frame
  double pad[2];
};
static_assert(sizeof(TriRec) == 192, "TriRec layout");

// Number of this library's kernels launched so far (all devices, all plans).
// Raise a kernel's dynamic shared-memory limit to at least `bytes`, never
// lowering it: plans driven from several host threads launch the same kernels
// with different sizes, and a lower limit set by one thread between another
// thread's setting and its launch would make that launch fail.
cudaError_t smem_raise_fn(const void* kern, int bytes);
template <class F>
inline cudaError_t smem_raise(F* kern, int bytes) {
  return smem_raise_fn(reinterpret_cast<const void*>(kern), bytes);
}
long long launches_total();
void count_launch(int k = 1);

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace efmm

#define EFMM_CUDA_TRY(expr)                                                   \
  do {                                                                        \
    cudaError_t _e = (expr);                                                  \
    if (_e != cudaSuccess) {                                                  \
      fprintf(stderr, "elfmm3d_b200: %s failed: %s (%s:%d)\n", #expr,         \
              cudaGetErrorString(_e), __FILE__, __LINE__);                    \
      throw efmm::CudaError{(int)_e};                                         \
    }                                                                         \
  } while (0)

namespace efmm {
// two-element vector type of a scalar (8- or 16-byte loads)
template <class T>
struct Vec2;
template <>
struct Vec2<double> { using type = double2; };
template <>
struct Vec2<float> { using type = float2; };

struct CudaError {
  int code;
};
}  // namespace efmm
