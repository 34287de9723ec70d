// sort.h -- device primitives of the tree builder (sort.cu): a stable LSD
// radix sort of (64-bit key, int value) pairs and an exclusive scan of ints,
// both on caller-provided scratch.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

namespace efmm {

// Bytes of scratch exclusive_scan_dev needs for n ints.
size_t scan_scratch_bytes(int n);
// out[i] = in[0] + ... + in[i-1] (out[0] = 0); in and out distinct.
void exclusive_scan_dev(cudaStream_t st, const int* in, int* out, int n, void* scratch);

// Bytes of scratch radix_sort_pairs needs for n pairs.
size_t radix_scratch_bytes(int n);
// Stable sort of n (key, value) pairs by the 8-bit key digits at the given
// bit shifts (least significant first; digits not named must be equal in
// all keys for a full sort); inputs and outputs distinct, outputs written by
// the last pass.
void radix_sort_pairs(cudaStream_t st, const unsigned long long* kin, unsigned long long* kout, const int* vin,
                      int* vout, int n, const int* shifts, int npass, void* scratch);

}  // namespace efmm
