// tc_bulk.cu -- FP32 products on the tensor cores from pre-split operands
// streamed by bulk copies.
//
// The products C[col][row] = sum_k A[k][row] B[col][k] of the mixed form run
// on the tensor cores as the 3-term TF32 split A B ~ Ahi Bhi + Ahi Blo +
// Alo Bhi (x = hi + lo, hi = x rounded to TF32).  Where an operand is
// geometry-only (the stored near field, the L2T functionals), it is split
// once and kept as tiles in the tensor cores' shared-memory layout; the
// other operand (densities, local expansions) is split into the same kind of
// tiles on every call by a cheap pass over it.  A tile of A holds 128 rows x
// 32 k, a tile of B BN columns x 32 k, each its TF32 head followed by its
// tail, both in the canonical no-swizzle K-major layout (element (row, k) at
// float (k % 4) + 4 (row % 8) + 32 (k / 4) + 256 (row / 8)); positions past
// the matrix hold zeros.  A K tile of the product is then two contiguous bulk
// copies from global into shared memory and twelve MMAs: no thread touches
// the operands on the way, where k_gemm_tc_ring splits every tile in shared
// memory on every call.  The head and the tail are full FP32 words, so a
// split operand takes 8 bytes per element.
//
// k_tc_bulk<BN, TC>: one CTA (320 threads) per task (a 128-row x BN-column
// output tile).  Warp 0 issues the copies into a ring of stages (4 of 48 KB
// for BN = 64, 3 of 64 KB for BN = 128); one thread of warp 1 issues the
// MMAs, each K tile into its own TMEM accumulator of BN columns (512 / BN of
// them); warps 2..9 drain every K tile's accumulator into registers of type
// TC (warp w: TMEM lanes 32 (w % 4)..+31, columns BN/2 ((w - 2) / 4)..), so
// the K-tile sums are added in FP32 or FP64 as in k_gemm_tc_ring (a long
// TMEM accumulation would drift by its truncation).  mbarriers: full[s]
// (stage s landed), empty[s] (the MMAs reading stage s completed), accf[a]
// (accumulator a complete), acce[a] (accumulator a drained).  Every wait is
// bounded and watches a shared abort flag; a CTA that gives up sets *err,
// waits (bounded) for its copies and MMAs in flight, frees its TMEM and
// stores nothing.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "common.cuh"
#include "kernels.h"
#include "tc_common.cuh"

namespace efmm {

namespace {

template <int BN>
struct BulkCfg {
  static constexpr int A_HALF = 16384;                  // bytes: 128 x 32 FP32
  static constexpr int B_HALF = BN * 32 * 4;            // bytes: BN x 32 FP32
  static constexpr int STAGE = 2 * A_HALF + 2 * B_HALF;
  static constexpr int STAGES = BN == 64 ? 4 : 3;
  static constexpr int ACC = 512 / BN;                  // TMEM accumulators
  static constexpr int NCOL = BN / 2;                   // columns per drain warp
  static constexpr int SMEM = STAGES * STAGE + 1024 + 256;  // stages, alignment, barriers
};
constexpr int BULK_THREADS = 320, BULK_DRAIN_WARPS = 8;
constexpr uint32_t BULK_LBO = 128, BULK_SBO = 1024;

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive1(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// bounded wait for phase `parity` that gives up at once when another role has
// aborted; a wait that runs out raises the abort flag itself
__device__ __forceinline__ bool wait_or_abort(uint32_t bar, uint32_t parity, volatile int* ab) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (*ab) return false;
    if (clock64() - t0 > TC_WAIT_CYCLES) {
      *ab = 1;
      return false;
    }
  }
  return true;
}

}  // namespace

template <int BN, class TC>
__global__ void __launch_bounds__(BULK_THREADS, 1)
k_tc_bulk(const BulkTask* __restrict__ tasks, const float* __restrict__ A, const float* __restrict__ B,
          TC* __restrict__ Cm, int* __restrict__ err) {
  using Cfg = BulkCfg<BN>;
  constexpr int NS = Cfg::STAGES, NACC = Cfg::ACC, NCOL = Cfg::NCOL;
  constexpr uint32_t IDESC = tc_idesc_mn(128, BN);
  extern __shared__ __align__(1024) unsigned char bk_raw[];
  const uint32_t raw = smem_u32(bk_raw);
  unsigned char* sm = bk_raw + ((1024 - (raw & 1023)) & 1023);
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + NS * Cfg::STAGE);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * NS + 2 * NACC);
  volatile int* abortf = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const uint32_t bar0 = smem_u32(bars);
  const uint32_t full0 = bar0, empty0 = bar0 + 8 * NS, accf0 = bar0 + 16 * NS, acce0 = accf0 + 8 * NACC;
  const BulkTask t = tasks[blockIdx.x];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 32) {
    for (int s = 0; s < NS; s++) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int a = 0; a < NACC; a++) {
      mbar_init(accf0 + 8 * a, 1);
      mbar_init(acce0 + 8 * a, BULK_DRAIN_WARPS);
    }
    *abortf = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const int nkt = t.nkt;

  if (warp == 0) {
    // producer: K tile kt into stage kt % NS once the MMAs of tile kt - NS
    // have read it
    if (lane == 0) {
      int issued = -1;
      for (int kt = 0; kt < nkt; kt++) {
        const int s = kt % NS;
        if (kt >= NS && !wait_or_abort(empty0 + 8 * s, ((kt / NS) - 1) & 1, abortf)) break;
        const uint32_t d = smem_u32(sm + s * Cfg::STAGE);
        mbar_expect_tx(full0 + 8 * s, Cfg::STAGE);
        bulk_g2s(d, A + t.a_off + (size_t)kt * (2 * Cfg::A_HALF / 4), 2 * Cfg::A_HALF, full0 + 8 * s);
        bulk_g2s(d + 2 * Cfg::A_HALF, B + t.b_off + (size_t)kt * (2 * Cfg::B_HALF / 4), 2 * Cfg::B_HALF,
                 full0 + 8 * s);
        issued = kt;
      }
      // no copy outlives the CTA: the last copies into every stage have landed
      for (int kt = issued - NS + 1 > 0 ? issued - NS + 1 : 0; kt <= issued; kt++)
        mbar_wait(full0 + 8 * (kt % NS), (kt / NS) & 1);
    }
  } else if (warp == 1) {
    // MMA issuer: tile kt into accumulator kt % NACC once it is drained
    if (lane == 0) {
      int issued = -1;
      for (int kt = 0; kt < nkt; kt++) {
        const int s = kt % NS, a = kt % NACC;
        if (!wait_or_abort(full0 + 8 * s, (kt / NS) & 1, abortf)) break;
        if (kt >= NACC && !wait_or_abort(acce0 + 8 * a, ((kt / NACC) - 1) & 1, abortf)) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t base = smem_u32(sm + s * Cfg::STAGE);
        const uint64_t dah = umma_desc(base, BULK_LBO, BULK_SBO),
                       dal = umma_desc(base + Cfg::A_HALF, BULK_LBO, BULK_SBO);
        const uint64_t dbh = umma_desc(base + 2 * Cfg::A_HALF, BULK_LBO, BULK_SBO),
                       dbl = umma_desc(base + 2 * Cfg::A_HALF + Cfg::B_HALF, BULK_LBO, BULK_SBO);
        const uint32_t dacc = tmem + (uint32_t)(a * BN);
#pragma unroll
        for (int i = 0; i < 4; i++) {
          // K step i: 2 i core matrices of 128 bytes further in the 16-byte address field
          const uint64_t o = (uint64_t)((2 * i * BULK_LBO) >> 4);
          mma_tf32(dacc, dal + o, dbh + o, IDESC, i > 0 ? 1u : 0u);
          mma_tf32(dacc, dah + o, dbl + o, IDESC, 1u);
          mma_tf32(dacc, dah + o, dbh + o, IDESC, 1u);
        }
        mma_commit(empty0 + 8 * s);
        mma_commit(accf0 + 8 * a);
        issued = kt;
      }
      // the MMAs in flight complete before the TMEM is freed
      if (issued >= 0) mbar_wait(accf0 + 8 * (issued % NACC), (issued / NACC) & 1);
    }
  } else {
    // drain: FP32 K-tile sums from TMEM added into TC registers
    const int q = warp & 3, half = (warp - 2) >> 2;
    TC acc[NCOL];
#pragma unroll
    for (int j = 0; j < NCOL; j++) acc[j] = (TC)0;
    bool ok = true;
    for (int kt = 0; kt < nkt; kt++) {
      const int a = kt % NACC;
      int good = 1;
      if (lane == 0) good = wait_or_abort(accf0 + 8 * a, (kt / NACC) & 1, abortf) ? 1 : 0;
      good = __shfl_sync(0xffffffffu, good, 0);
      if (!good) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      uint32_t r[NCOL];
      const uint32_t addr = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(a * BN + NCOL * half);
#pragma unroll
      for (int c16 = 0; c16 < NCOL / 16; c16++) {
        uint32_t* v = r + 16 * c16;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(addr + 16 * c16));
      }
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < NCOL; j++) acc[j] += (TC)__uint_as_float(r[j]);
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive1(acce0 + 8 * a);
    }
    if (ok && !*abortf) {
      const int row = t.row0 + 32 * q + lane;
      if (row < t.M) {
        TC* Cp = Cm + t.c_off + row;
#pragma unroll
        for (int j = 0; j < NCOL; j++) {
          const int col = t.col0 + NCOL * half + j;
          if (col < t.N) Cp[(size_t)col * t.ldc] = acc[j];
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (tid == 0 && *abortf) atomicExch(err, 1);
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
}

// Which form the products with a geometry-only operand take: 1 (default) the
// pre-split operands and k_tc_bulk where they fit, 0 the FP32 operands and
// k_gemm_tc_ring; ELFMM3D_SPLIT=0 or efmm_split_variant select the latter.
static int g_split = -1;
int split_variant() {
  if (g_split < 0) {
    const char* e = getenv("ELFMM3D_SPLIT");
    g_split = (e && e[0] == '0') ? 0 : 1;
  }
  return g_split;
}

template <class TC>
void launch_tc_bulk(cudaStream_t st, int ntask, const BulkTask* tasks, const float* A, const float* B, TC* C,
                    int* err, int bn) {
  if (ntask <= 0) return;
  if (bn == 64) {
    EFMM_CUDA_TRY(smem_raise(k_tc_bulk<64, TC>, BulkCfg<64>::SMEM));
    k_tc_bulk<64, TC><<<ntask, BULK_THREADS, BulkCfg<64>::SMEM, st>>>(tasks, A, B, C, err);
  } else {
    EFMM_CUDA_TRY(smem_raise(k_tc_bulk<128, TC>, BulkCfg<128>::SMEM));
    k_tc_bulk<128, TC><<<ntask, BULK_THREADS, BulkCfg<128>::SMEM, st>>>(tasks, A, B, C, err);
  }
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}
template void launch_tc_bulk<float>(cudaStream_t, int, const BulkTask*, const float*, const float*, float*, int*,
                                    int);
template void launch_tc_bulk<double>(cudaStream_t, int, const BulkTask*, const float*, const float*, double*, int*,
                                     int);

}  // namespace efmm

namespace {
// host restatement of tf32_head (tc_common.cuh): TF32 nearest, ties away
float tf32_head_host(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & ~0x1FFFu;
  float h;
  memcpy(&h, &u, 4);
  return h;
}

template <class TC>
int bulk_selfcheck(int M, int N, int K, int bn, unsigned seed, double* rel, int* timeout) {
  using namespace efmm;
  std::vector<float> hA((size_t)K * M), hB((size_t)N * K);
  unsigned long long st = seed * 6364136223846793005ull + 1;
  auto uni = [&]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return (float)(((st >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0);
  };
  for (auto& v : hA) v = uni();
  for (auto& v : hB) v = uni();
  const int nmt = (M + 127) / 128, nct = (N + bn - 1) / bn, nkt = (K + 31) / 32, bt = 2 * bn * 32;
  std::vector<float> tA((size_t)nmt * nkt * 8192, 0.0f), tB((size_t)nct * nkt * bt, 0.0f);
  for (int k = 0; k < K; k++) {
    const int kt = k >> 5, kl = k & 31;
    for (int m = 0; m < M; m++) {
      const int mt = m >> 7, ml = m & 127;
      const size_t idx = ((size_t)mt * nkt + kt) * 8192 + (kl & 3) + 4 * (ml & 7) + 32 * (kl >> 2) + 256 * (ml >> 3);
      const float v = hA[(size_t)k * M + m], h = tf32_head_host(v);
      tA[idx] = h;
      tA[idx + 4096] = v - h;
    }
    for (int n = 0; n < N; n++) {
      const int ct = n / bn, nl = n % bn;
      const size_t idx = ((size_t)ct * nkt + kt) * bt + (kl & 3) + 4 * (nl & 7) + 32 * (kl >> 2) + 256 * (nl >> 3);
      const float v = hB[(size_t)n * K + k], h = tf32_head_host(v);
      tB[idx] = h;
      tB[idx + bt / 2] = v - h;
    }
  }
  std::vector<BulkTask> tasks;
  for (int ct = 0; ct < nct; ct++)
    for (int mt = 0; mt < nmt; mt++)
      tasks.push_back({(long long)mt * nkt * 8192, (long long)ct * nkt * bt, 0, M, N, nkt, 128 * mt, bn * ct, M});
  std::vector<TC> hC((size_t)N * M, (TC)-7);
  float *dA = nullptr, *dB = nullptr;
  TC* dC = nullptr;
  int* dErr = nullptr;
  BulkTask* dT = nullptr;
  auto fail = [&]() {
    cudaFree(dA); cudaFree(dB); cudaFree(dC); cudaFree(dErr); cudaFree(dT);
    return 256;
  };
  if (cudaMalloc(&dA, tA.size() * 4 + 16) || cudaMalloc(&dB, tB.size() * 4 + 16) ||
      cudaMalloc(&dC, hC.size() * sizeof(TC)) || cudaMalloc(&dErr, 4) ||
      cudaMalloc(&dT, tasks.size() * sizeof(BulkTask) + 16))
    return fail();
  cudaMemcpy(dA, tA.data(), tA.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dB, tB.data(), tB.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dC, hC.data(), hC.size() * sizeof(TC), cudaMemcpyHostToDevice);
  cudaMemcpy(dT, tasks.data(), tasks.size() * sizeof(BulkTask), cudaMemcpyHostToDevice);
  cudaMemset(dErr, 0, 4);
  try {
    launch_tc_bulk<TC>(0, (int)tasks.size(), dT, dA, dB, dC, dErr, bn);
  } catch (const CudaError&) {
    return fail();
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return fail();
  cudaMemcpy(hC.data(), dC, hC.size() * sizeof(TC), cudaMemcpyDeviceToHost);
  int herr = 0;
  cudaMemcpy(&herr, dErr, 4, cudaMemcpyDeviceToHost);
  double num = 0, den = 0;
  for (int c = 0; c < N; c++)
    for (int r = 0; r < M; r++) {
      double ref = 0;
      for (int k = 0; k < K; k++) ref += (double)hA[(size_t)k * M + r] * (double)hB[(size_t)c * K + k];
      const double d = (double)hC[(size_t)c * M + r] - ref;
      num += d * d;
      den += ref * ref;
    }
  *rel = den > 0 ? sqrt(num / den) : sqrt(num);
  *timeout = herr;
  cudaFree(dA); cudaFree(dB); cudaFree(dC); cudaFree(dErr); cudaFree(dT);
  return 0;
}
}  // namespace

// The bulk-copy product on random FP32 A (K x M) and B (N x K) in [-1, 1)
// against an FP64 host product (relative l2 error in *rel; *timeout the
// kernel's error flag): the host writes the split tiles (128 x 32 of A,
// bn x 32 of B, head then tail, canonical layout) as the device splitters
// do, one task per (row tile, column tile); fp64 selects FP64 K-tile sums.
extern "C" int efmm_tc_bulk_selfcheck(int M, int N, int K, int bn, int fp64, unsigned seed, double* rel,
                                      int* timeout) {
  if (M < 1 || N < 1 || K < 0 || M > 8192 || N > 1024 || K > 65536 || (bn != 64 && bn != 128)) return 16;
  return fp64 ? bulk_selfcheck<double>(M, N, K, bn, seed, rel, timeout)
              : bulk_selfcheck<float>(M, N, K, bn, seed, rel, timeout);
}

// Select the form of the products with a geometry-only operand for this
// process (1 pre-split operands streamed by bulk copies, 0 FP32 operands
// split in shared memory); returns the previous form.  A plan rebuilds its
// split operands at its next mixed pass.
extern "C" int efmm_split_variant(int split) {
  const int old = efmm::split_variant();
  efmm::g_split = split ? 1 : 0;
  return old;
}
