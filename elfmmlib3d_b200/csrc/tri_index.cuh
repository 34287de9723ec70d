// tri_index.cuh -- multi-index helpers shared by the near-field code.
#pragma once

#ifdef __CUDACC__
#define EFMM_HD __host__ __device__ __forceinline__
#else
#define EFMM_HD inline
#endif

namespace efmm {

// number of multi-indices (a,b,c) with a+b+c <= n
EFMM_HD constexpr int jet_size(int n) { return (n + 1) * (n + 2) * (n + 3) / 6; }

// linear index of the multi-index (a,b,c): grouped by total degree, then a
// descending, then b descending.
EFMM_HD constexpr int jidx(int a, int b, int c) {
  int n = a + b + c;
  int off = n * (n + 1) * (n + 2) / 6;
  int pos = 0;
  for (int ap = n; ap > a; --ap) pos += n - ap + 1;
  pos += (n - a) - b;
  return off + pos;
}

}  // namespace efmm
