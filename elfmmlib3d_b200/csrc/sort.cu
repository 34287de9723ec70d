// sort.cu -- the tree builder's device primitives: a stable LSD radix sort of
// (64-bit key, int value) pairs and an exclusive scan of ints.
//
// Radix sort, one pass per 8-bit digit (only the digits the caller names):
//   1. k_rs_hist: each CTA counts the digits of its tile of RS_TILE keys into
//      shared memory and writes hist[digit][tile] (digit-major);
//   2. the exclusive scan of hist gives every (digit, tile) its first output
//      position (all smaller digits, then the same digit in earlier tiles);
//   3. k_rs_scatter: each CTA walks its tile again in order, 256 keys at a
//      time; a key's rank among the equal digits before it is its rank in its
//      warp (__match_any_sync, lanes below) plus the counts of the earlier
//      warps and of the earlier rounds, so equal digits keep their input
//      order and the pass is stable.
// The tree's point orders depend on that stability (points of one box keep
// their relative order, as in the reference's partition, src/d3tstrcr.f).
// Scan: CTAs of 1024 ints scan in shared memory and write their sums, the
// sums are scanned the same way (recursively), and a last kernel adds each
// CTA's offset.
#include <algorithm>
#include <numeric>
#include <random>
#include <vector>
#include "common.cuh"
#include "sort.h"

namespace efmm {

namespace {

constexpr int SC_THREADS = 256, SC_PER = 4, SC_TILE = SC_THREADS * SC_PER;
constexpr int RS_THREADS_ = 256, RS_TILE = 4096, RS_WARPS = RS_THREADS_ / 32;

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

int scan_blocks(int n) { return (n + SC_TILE - 1) / SC_TILE; }

// exclusive scan of one tile per CTA; the tile's total into sums[blockIdx.x]
__global__ void __launch_bounds__(SC_THREADS) k_scan_tile(const int* __restrict__ in, int* __restrict__ out, int n,
                                                           int* __restrict__ sums) {
  __shared__ int ws[SC_THREADS / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long base = (long long)blockIdx.x * SC_TILE + (long long)tid * SC_PER;
  int v[SC_PER], t = 0;
#pragma unroll
  for (int j = 0; j < SC_PER; j++) {
    v[j] = base + j < n ? in[base + j] : 0;
    t += v[j];
  }
  // inclusive scan of the thread totals: within the warp, then across warps
  int x = t;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < SC_THREADS / 32 ? ws[lane] : 0;
#pragma unroll
    for (int o = 1; o < SC_THREADS / 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < SC_THREADS / 32) ws[lane] = w;
  }
  __syncthreads();
  int run = x - t + (warp > 0 ? ws[warp - 1] : 0);
#pragma unroll
  for (int j = 0; j < SC_PER; j++) {
    if (base + j < n) out[base + j] = run;
    run += v[j];
  }
  if (tid == SC_THREADS - 1) sums[blockIdx.x] = run;
}

__global__ void k_scan_add(int* __restrict__ out, int n, const int* __restrict__ offs) {
  const long long i = (long long)blockIdx.x * SC_TILE + threadIdx.x;
  const int a = offs[blockIdx.x];
#pragma unroll
  for (int j = 0; j < SC_PER; j++) {
    const long long q = i + (long long)j * SC_THREADS;
    if (q < n) out[q] += a;
  }
}

// ints of scratch the scan of n ints needs: per level the tile sums and
// their scan
size_t scan_scratch_ints(int n) {
  size_t s = 0;
  for (int m = scan_blocks(n); m > 1; m = scan_blocks(m)) s += 2 * (size_t)m + 64;
  return s + 64;
}

void scan_rec(cudaStream_t st, const int* in, int* out, int n, int* scratch) {
  const int nb = scan_blocks(n);
  int* sums = scratch;
  int* soff = scratch + nb;
  k_scan_tile<<<nb, SC_THREADS, 0, st>>>(in, out, n, sums);
  count_launch();
  if (nb > 1) {
    scan_rec(st, sums, soff, nb, scratch + 2 * (size_t)nb + 64);
    k_scan_add<<<nb, SC_THREADS, 0, st>>>(out, n, soff);
    count_launch();
  }
}

__global__ void __launch_bounds__(RS_THREADS_) k_rs_hist(const unsigned long long* __restrict__ keys, int n,
                                                          int shift, int ntile, int* __restrict__ hist) {
  __shared__ int cnt[256];
  const int tid = threadIdx.x;
  cnt[tid] = 0;
  __syncthreads();
  const long long t0 = (long long)blockIdx.x * RS_TILE;
  const long long t1 = t0 + RS_TILE < n ? t0 + RS_TILE : n;
  for (long long i = t0 + tid; i < t1; i += RS_THREADS_) atomicAdd(&cnt[(int)((keys[i] >> shift) & 255)], 1);
  __syncthreads();
  hist[(size_t)tid * ntile + blockIdx.x] = cnt[tid];
}

__global__ void __launch_bounds__(RS_THREADS_) k_rs_scatter(const unsigned long long* __restrict__ kin,
                                                             const int* __restrict__ vin, int n, int shift, int ntile,
                                                             const int* __restrict__ offs,
                                                             unsigned long long* __restrict__ kout,
                                                             int* __restrict__ vout) {
  __shared__ int wcnt[RS_WARPS][256];  // keys of each digit in each warp, this round
  __shared__ int wpre[RS_WARPS][256];  // their first output position
  __shared__ int next[256];            // next output position of each digit
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int w = 0; w < RS_WARPS; w++) wcnt[w][tid] = 0;
  next[tid] = offs[(size_t)tid * ntile + blockIdx.x];
  __syncthreads();
  const long long t0 = (long long)blockIdx.x * RS_TILE;
  const long long t1 = t0 + RS_TILE < n ? t0 + RS_TILE : n;
  const unsigned lt = (1u << lane) - 1u;
  for (long long r0 = t0; r0 < t1; r0 += RS_THREADS_) {
    const long long i = r0 + tid;
    const bool ok = i < t1;
    unsigned long long k = 0;
    int v = 0, d = 256;  // 256: no key (matches no digit)
    if (ok) {
      k = kin[i];
      v = vin[i];
      d = (int)((k >> shift) & 255);
    }
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int rank = __popc(peers & lt);
    if (ok && rank == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    {  // thread tid: digit tid over the warps in order
      int s = next[tid];
#pragma unroll
      for (int w = 0; w < RS_WARPS; w++) {
        wpre[w][tid] = s;
        s += wcnt[w][tid];
        wcnt[w][tid] = 0;
      }
      next[tid] = s;
    }
    __syncthreads();
    if (ok) {
      const int pos = wpre[warp][d] + rank;
      kout[pos] = k;
      vout[pos] = v;
    }
    // wpre is rewritten only after the next round's first barrier
  }
}

}  // namespace

size_t scan_scratch_bytes(int n) { return align256(sizeof(int) * scan_scratch_ints(n)); }

void exclusive_scan_dev(cudaStream_t st, const int* in, int* out, int n, void* scratch) {
  if (n <= 0) return;
  scan_rec(st, in, out, n, static_cast<int*>(scratch));
}

size_t radix_scratch_bytes(int n) {
  const int ntile = (n + RS_TILE - 1) / RS_TILE;
  const size_t nh = 256 * (size_t)ntile;
  return 2 * align256(sizeof(unsigned long long) * (size_t)n) + 2 * align256(sizeof(int) * (size_t)n) +
         2 * align256(sizeof(int) * nh) + scan_scratch_bytes((int)nh);
}

void radix_sort_pairs(cudaStream_t st, const unsigned long long* kin, unsigned long long* kout, const int* vin,
                      int* vout, int n, const int* shifts, int npass, void* scratch) {
  if (n <= 0) return;
  if (npass <= 0) {
    EFMM_CUDA_TRY(cudaMemcpyAsync(kout, kin, sizeof(unsigned long long) * (size_t)n, cudaMemcpyDeviceToDevice, st));
    EFMM_CUDA_TRY(cudaMemcpyAsync(vout, vin, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, st));
    return;
  }
  const int ntile = (n + RS_TILE - 1) / RS_TILE;
  const size_t nh = 256 * (size_t)ntile;
  char* c = static_cast<char*>(scratch);
  unsigned long long* kb[2];
  int* vb[2];
  kb[0] = reinterpret_cast<unsigned long long*>(c);
  c += align256(sizeof(unsigned long long) * (size_t)n);
  kb[1] = reinterpret_cast<unsigned long long*>(c);
  c += align256(sizeof(unsigned long long) * (size_t)n);
  vb[0] = reinterpret_cast<int*>(c);
  c += align256(sizeof(int) * (size_t)n);
  vb[1] = reinterpret_cast<int*>(c);
  c += align256(sizeof(int) * (size_t)n);
  int* hist = reinterpret_cast<int*>(c);
  c += align256(sizeof(int) * nh);
  int* offs = reinterpret_cast<int*>(c);
  c += align256(sizeof(int) * nh);
  void* sscr = c;
  const unsigned long long* ks = kin;
  const int* vs = vin;
  for (int q = 0; q < npass; q++) {
    unsigned long long* kd = q == npass - 1 ? kout : kb[q & 1];
    int* vd = q == npass - 1 ? vout : vb[q & 1];
    k_rs_hist<<<ntile, RS_THREADS_, 0, st>>>(ks, n, shifts[q], ntile, hist);
    count_launch();
    exclusive_scan_dev(st, hist, offs, (int)nh, sscr);
    k_rs_scatter<<<ntile, RS_THREADS_, 0, st>>>(ks, vs, n, shifts[q], ntile, offs, kd, vd);
    count_launch();
    ks = kd;
    vs = vd;
  }
  EFMM_CUDA_TRY(cudaGetLastError());
}

}  // namespace efmm

// Device check of the radix sort and the scan against the host: n pairs with
// keys below 2^bits drawn with many repeats (values = input positions), the
// sort over the digits of [0, bits), compared with a stable host sort (keys
// and values); the scan of n small ints against the host prefix sums.
// Returns 0 and *bad = the number of mismatches (sorted keys, values, scan).
extern "C" int efmm_sort_selfcheck_device(int n, int bits, unsigned seed, long long* bad) {
  using namespace efmm;
  if (n < 0 || n > (1 << 26) || bits < 1 || bits > 64 || !bad) return 16;
  std::mt19937_64 rng(seed);
  const int dup = std::max(1, n / 7);
  std::vector<unsigned long long> pool(dup);
  for (auto& k : pool) k = bits == 64 ? rng() : (rng() & ((1ull << bits) - 1));
  std::vector<unsigned long long> hk(n);
  std::vector<int> hv(n), cnt(n);
  for (int i = 0; i < n; i++) {
    hk[i] = pool[rng() % dup];
    hv[i] = i;
    cnt[i] = (int)(rng() % 5);
  }
  std::vector<int> shifts;
  for (int b = 0; b < bits; b += 8) shifts.push_back(b);
  unsigned long long *dk = nullptr, *dk2 = nullptr;
  int *dv = nullptr, *dv2 = nullptr, *dc = nullptr, *dcs = nullptr;
  void* scr = nullptr;
  const size_t sb = std::max(radix_scratch_bytes(n), scan_scratch_bytes(n));
  auto release = [&]() {
    cudaFree(dk); cudaFree(dk2); cudaFree(dv); cudaFree(dv2); cudaFree(dc); cudaFree(dcs); cudaFree(scr);
  };
  const size_t m = std::max(n, 1);
  if (cudaMalloc(&dk, 8 * m) || cudaMalloc(&dk2, 8 * m) || cudaMalloc(&dv, 4 * m) || cudaMalloc(&dv2, 4 * m) ||
      cudaMalloc(&dc, 4 * m) || cudaMalloc(&dcs, 4 * m) || cudaMalloc(&scr, std::max(sb, (size_t)256))) {
    release();
    return 256;
  }
  cudaMemcpy(dk, hk.data(), 8 * (size_t)n, cudaMemcpyHostToDevice);
  cudaMemcpy(dv, hv.data(), 4 * (size_t)n, cudaMemcpyHostToDevice);
  cudaMemcpy(dc, cnt.data(), 4 * (size_t)n, cudaMemcpyHostToDevice);
  try {
    radix_sort_pairs(0, dk, dk2, dv, dv2, n, shifts.data(), (int)shifts.size(), scr);
    exclusive_scan_dev(0, dc, dcs, n, scr);
  } catch (const CudaError&) {
    release();
    return 256;
  }
  if (cudaDeviceSynchronize() != cudaSuccess) {
    release();
    return 256;
  }
  std::vector<unsigned long long> gk(n);
  std::vector<int> gv(n), gs(n);
  cudaMemcpy(gk.data(), dk2, 8 * (size_t)n, cudaMemcpyDeviceToHost);
  cudaMemcpy(gv.data(), dv2, 4 * (size_t)n, cudaMemcpyDeviceToHost);
  cudaMemcpy(gs.data(), dcs, 4 * (size_t)n, cudaMemcpyDeviceToHost);
  release();
  std::vector<int> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return hk[a] < hk[b]; });
  long long nb = 0;
  int run = 0;
  for (int i = 0; i < n; i++) {
    nb += gk[i] != hk[ord[i]];
    nb += gv[i] != ord[i];
    nb += gs[i] != run;
    run += cnt[i];
  }
  *bad = nb;
  return 0;
}
