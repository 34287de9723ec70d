// devbuf.h -- minimal RAII device buffer used by the host orchestration.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <utility>
#include "common.cuh"

namespace efmm {

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;    // elements in use
  size_t cap = 0;  // elements allocated
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept { swap(o); }
  DevBuf& operator=(DevBuf&& o) noexcept {
    swap(o);
    return *this;
  }
  ~DevBuf() { release(); }
  void swap(DevBuf& o) {
    std::swap(p, o.p);
    std::swap(n, o.n);
    std::swap(cap, o.cap);
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = cap = 0;
  }
  // resize without preserving contents
  void resize(size_t m) {
    if (m > cap) {
      release();
      size_t c = m ? m : 1;
      EFMM_CUDA_TRY(cudaMalloc((void**)&p, c * sizeof(T)));
      cap = c;
    }
    n = m;
  }
  // resize preserving the first n elements
  void grow(size_t m, cudaStream_t st) {
    if (m <= cap) {
      n = m;
      return;
    }
    size_t c = m + m / 2 + 16;
    T* q = nullptr;
    EFMM_CUDA_TRY(cudaMalloc((void**)&q, c * sizeof(T)));
    if (p && n) EFMM_CUDA_TRY(cudaMemcpyAsync(q, p, n * sizeof(T), cudaMemcpyDeviceToDevice, st));
    EFMM_CUDA_TRY(cudaStreamSynchronize(st));
    if (p) cudaFree(p);
    p = q;
    cap = c;
    n = m;
  }
  void zero(cudaStream_t st) {
    if (n) EFMM_CUDA_TRY(cudaMemsetAsync(p, 0, n * sizeof(T), st));
  }
  T* get() const { return p; }
  size_t size() const { return n; }
};

}  // namespace efmm
