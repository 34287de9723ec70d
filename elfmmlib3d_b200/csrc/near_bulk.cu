// near_bulk.cu -- the mixed replay of the stored near field as a stream of
// pre-split tensor-core tiles.
//
// The product of the mixed replay (per near leaf: C[r][KB e + c] = sum over
// the near triangles t and density components j of A[NJ t + j][KB e + c]
// sigma_r[NJ t + j]; M = KB x points rows, K = NJ x near triangles, N = R
// right-hand sides) runs on the tensor cores as the 3-term TF32 split
// A B ~ Ahi Bhi + Ahi Blo + Alo Bhi (x = hi + lo, hi = x rounded to TF32).
// A, the stored near field, depends on the geometry only, so it is split
// once per store (k_near_split_store, nearfield.cu): tiles of 128 rows x 32 k,
// each its TF32 head followed by its tail, both already in the canonical
// no-swizzle K-major layout of the tensor cores' shared-memory operands
// (element (row, k) at float (k % 4) + 4 (row % 8) + 32 (k / 4) +
// 256 (row / 8)).  The densities are split on every call the same way, into
// tiles of 64 columns x 32 k (k_near_sigma_split).  A K tile of the product
// is then two contiguous bulk copies (32 + 16 KB) from global into shared
// memory and twelve MMAs: no thread touches the operands on the way, so the
// kernel streams the store at the copy engines' rate, where the FP32 form
// (k_gemm_tc_ring) splits every tile in shared memory.  The head and the tail
// are full FP32 words, so the split store takes 8 bytes per element.
//
// k_near_tc_bulk: one CTA (320 threads) per (leaf, 128-row tile, 64-column
// tile).  Warp 0 issues the copies into a ring of 4 stages; one thread of
// warp 1 issues the MMAs, each K tile into its own TMEM accumulator of 64
// columns (8 of them); warps 2..9 drain every K tile's accumulator into FP64
// registers (warp w: TMEM lanes 32 (w % 4)..+31, columns 32 ((w - 2) / 4)..
// +31), so the K-tile sums are added in FP64 as in the FP32 form.
// mbarriers: full[s] (stage s landed), empty[s] (the MMAs reading stage s
// completed), accf[a] (accumulator a complete), acce[a] (accumulator a
// drained).  Every wait is bounded and watches a shared abort flag; a CTA
// that gives up sets *err, waits (bounded) for its copies and MMAs in
// flight, frees its TMEM and stores nothing.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <vector>
#include "common.cuh"
#include "kernels.h"
#include "tc_common.cuh"

namespace efmm {

namespace {

constexpr int NB_STAGES = 4, NB_ACC = 8, NB_THREADS = 320, NB_DRAIN_WARPS = 8;
constexpr int NB_AHALF = 16384, NB_BHALF = 8192;          // bytes: one A part, one B part
constexpr int NB_STAGE = 2 * NB_AHALF + 2 * NB_BHALF;     // 48 KB
constexpr uint32_t NB_LBO = 128, NB_SBO = 1024;
constexpr int NB_SMEM = NB_STAGES * NB_STAGE + 1024 + 256;  // stages, alignment, barriers

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

__global__ void __launch_bounds__(NB_THREADS, 1)
k_near_tc_bulk(const NearTcTask* __restrict__ tasks, const float* __restrict__ A, const float* __restrict__ B,
               double* __restrict__ Cm, int* __restrict__ err) {
  constexpr uint32_t IDESC = tc_idesc_mn(128, 64);
  extern __shared__ __align__(1024) unsigned char nb_raw[];
  const uint32_t raw = smem_u32(nb_raw);
  unsigned char* sm = nb_raw + ((1024 - (raw & 1023)) & 1023);
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + NB_STAGES * NB_STAGE);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * NB_STAGES + 2 * NB_ACC);
  volatile int* abortf = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const uint32_t bar0 = smem_u32(bars);
  const uint32_t full0 = bar0, empty0 = bar0 + 8 * NB_STAGES, accf0 = bar0 + 16 * NB_STAGES,
                 acce0 = accf0 + 8 * NB_ACC;
  const NearTcTask t = tasks[blockIdx.x];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 32) {
    for (int s = 0; s < NB_STAGES; s++) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int a = 0; a < NB_ACC; a++) {
      mbar_init(accf0 + 8 * a, 1);
      mbar_init(acce0 + 8 * a, NB_DRAIN_WARPS);
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
    // producer: K tile kt into stage kt % NB_STAGES once the MMAs of tile
    // kt - NB_STAGES have read it
    if (lane == 0) {
      int issued = -1;
      for (int kt = 0; kt < nkt; kt++) {
        const int s = kt % NB_STAGES;
        if (kt >= NB_STAGES && !wait_or_abort(empty0 + 8 * s, ((kt / NB_STAGES) - 1) & 1, abortf)) break;
        const uint32_t d = smem_u32(sm + s * NB_STAGE);
        mbar_expect_tx(full0 + 8 * s, NB_STAGE);
        bulk_g2s(d, A + t.a_off + (size_t)kt * (2 * NB_AHALF / 4), 2 * NB_AHALF, full0 + 8 * s);
        bulk_g2s(d + 2 * NB_AHALF, B + t.b_off + (size_t)kt * (2 * NB_BHALF / 4), 2 * NB_BHALF, full0 + 8 * s);
        issued = kt;
      }
      // no copy outlives the CTA: the last copies into every stage have landed
      for (int kt = issued - NB_STAGES + 1 > 0 ? issued - NB_STAGES + 1 : 0; kt <= issued; kt++)
        mbar_wait(full0 + 8 * (kt % NB_STAGES), (kt / NB_STAGES) & 1);
    }
  } else if (warp == 1) {
    // MMA issuer: tile kt into accumulator kt % NB_ACC once it is drained
    if (lane == 0) {
      int issued = -1;
      for (int kt = 0; kt < nkt; kt++) {
        const int s = kt % NB_STAGES, a = kt % NB_ACC;
        if (!wait_or_abort(full0 + 8 * s, (kt / NB_STAGES) & 1, abortf)) break;
        if (kt >= NB_ACC && !wait_or_abort(acce0 + 8 * a, ((kt / NB_ACC) - 1) & 1, abortf)) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t base = smem_u32(sm + s * NB_STAGE);
        const uint64_t dah = umma_desc(base, NB_LBO, NB_SBO), dal = umma_desc(base + NB_AHALF, NB_LBO, NB_SBO);
        const uint64_t dbh = umma_desc(base + 2 * NB_AHALF, NB_LBO, NB_SBO),
                       dbl = umma_desc(base + 2 * NB_AHALF + NB_BHALF, NB_LBO, NB_SBO);
        const uint32_t dacc = tmem + (uint32_t)a * 64;
#pragma unroll
        for (int i = 0; i < 4; i++) {
          // K step i: 2 i core matrices of 128 bytes further in the 16-byte address field
          const uint64_t o = (uint64_t)((2 * i * NB_LBO) >> 4);
          mma_tf32(dacc, dal + o, dbh + o, IDESC, i > 0 ? 1u : 0u);
          mma_tf32(dacc, dah + o, dbl + o, IDESC, 1u);
          mma_tf32(dacc, dah + o, dbh + o, IDESC, 1u);
        }
        mma_commit(empty0 + 8 * s);
        mma_commit(accf0 + 8 * a);
        issued = kt;
      }
      // the MMAs in flight complete before the TMEM is freed
      if (issued >= 0) mbar_wait(accf0 + 8 * (issued % NB_ACC), (issued / NB_ACC) & 1);
    }
  } else {
    // drain: FP32 K-tile sums from TMEM added into FP64 registers
    const int q = warp & 3, half = (warp - 2) >> 2;
    double acc[32];
#pragma unroll
    for (int j = 0; j < 32; j++) acc[j] = 0.0;
    bool ok = true;
    for (int kt = 0; kt < nkt; kt++) {
      const int a = kt % NB_ACC;
      int good = 1;
      if (lane == 0) good = wait_or_abort(accf0 + 8 * a, (kt / NB_ACC) & 1, abortf) ? 1 : 0;
      good = __shfl_sync(0xffffffffu, good, 0);
      if (!good) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      uint32_t r[32];
      const uint32_t addr = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)a * 64 + 32 * half;
#pragma unroll
      for (int c16 = 0; c16 < 2; c16++) {
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
      for (int j = 0; j < 32; j++) acc[j] += (double)__uint_as_float(r[j]);
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive1(acce0 + 8 * a);
    }
    if (ok && !*abortf) {
      const int row = t.row0 + 32 * q + lane;
      if (row < t.M) {
        double* Cp = Cm + t.c_off + row;
#pragma unroll
        for (int j = 0; j < 32; j++) {
          const int col = t.col0 + 32 * half + j;
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

// Which form the mixed replay of the stored near field takes: 1 (default)
// the pre-split store and k_near_tc_bulk, 0 the FP32 copy and
// k_gemm_tc_ring; ELFMM3D_NEAR_SPLIT=0 or efmm_near_variant select the latter.
static int g_near_split = -1;
int near_split_variant() {
  if (g_near_split < 0) {
    const char* e = getenv("ELFMM3D_NEAR_SPLIT");
    g_near_split = (e && e[0] == '0') ? 0 : 1;
  }
  return g_near_split;
}

void launch_near_tc_bulk(cudaStream_t st, int ntask, const NearTcTask* tasks, const float* A, const float* B,
                         double* C, int* err) {
  if (ntask <= 0) return;
  EFMM_CUDA_TRY(smem_raise(k_near_tc_bulk, NB_SMEM));
  k_near_tc_bulk<<<ntask, NB_THREADS, NB_SMEM, st>>>(tasks, A, B, C, err);
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}

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
}  // namespace

// The bulk-copy product on random FP32 A (K x M) and B (N x K) in [-1, 1)
// against an FP64 host product (relative l2 error in *rel; *timeout the
// kernel's error flag): the host writes the split tiles (128 x 32 of A,
// 64 x 32 of B, head then tail, canonical layout) as k_near_split_store and
// k_near_sigma_split do, one task per (row tile, column tile).
extern "C" int efmm_near_bulk_selfcheck(int M, int N, int K, unsigned seed, double* rel, int* timeout) {
  using namespace efmm;
  if (M < 1 || N < 1 || K < 0 || M > 4096 || N > 1024 || K > 65536) return 16;
  std::vector<float> hA((size_t)K * M), hB((size_t)N * K);
  unsigned long long st = seed * 6364136223846793005ull + 1;
  auto uni = [&]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return (float)(((st >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0);
  };
  for (auto& v : hA) v = uni();
  for (auto& v : hB) v = uni();
  const int nmt = (M + 127) / 128, nct = (N + 63) / 64, nkt = (K + 31) / 32;
  std::vector<float> tA((size_t)nmt * nkt * 8192, 0.0f), tB((size_t)nct * nkt * 4096, 0.0f);
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
      const int ct = n >> 6, nl = n & 63;
      const size_t idx = ((size_t)ct * nkt + kt) * 4096 + (kl & 3) + 4 * (nl & 7) + 32 * (kl >> 2) + 256 * (nl >> 3);
      const float v = hB[(size_t)n * K + k], h = tf32_head_host(v);
      tB[idx] = h;
      tB[idx + 2048] = v - h;
    }
  }
  std::vector<NearTcTask> tasks;
  for (int ct = 0; ct < nct; ct++)
    for (int mt = 0; mt < nmt; mt++)
      tasks.push_back({(long long)mt * nkt * 8192, (long long)ct * nkt * 4096, 0, M, N, nkt, 128 * mt, 64 * ct, M});
  std::vector<double> hC((size_t)N * M, -7.0);
  float *dA = nullptr, *dB = nullptr;
  double* dC = nullptr;
  int* dErr = nullptr;
  NearTcTask* dT = nullptr;
  auto fail = [&]() {
    cudaFree(dA); cudaFree(dB); cudaFree(dC); cudaFree(dErr); cudaFree(dT);
    return 256;
  };
  if (cudaMalloc(&dA, tA.size() * 4 + 16) || cudaMalloc(&dB, tB.size() * 4 + 16) || cudaMalloc(&dC, hC.size() * 8) ||
      cudaMalloc(&dErr, 4) || cudaMalloc(&dT, tasks.size() * sizeof(NearTcTask)))
    return fail();
  cudaMemcpy(dA, tA.data(), tA.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dB, tB.data(), tB.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dC, hC.data(), hC.size() * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(dT, tasks.data(), tasks.size() * sizeof(NearTcTask), cudaMemcpyHostToDevice);
  cudaMemset(dErr, 0, 4);
  try {
    launch_near_tc_bulk(0, (int)tasks.size(), dT, dA, dB, dC, dErr);
  } catch (const CudaError&) {
    return fail();
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return fail();
  cudaMemcpy(hC.data(), dC, hC.size() * 8, cudaMemcpyDeviceToHost);
  int herr = 0;
  cudaMemcpy(&herr, dErr, 4, cudaMemcpyDeviceToHost);
  double num = 0, den = 0;
  for (int c = 0; c < N; c++)
    for (int r = 0; r < M; r++) {
      double ref = 0;
      for (int k = 0; k < K; k++) ref += (double)hA[(size_t)k * M + r] * (double)hB[(size_t)c * K + k];
      const double d = hC[(size_t)c * M + r] - ref;
      num += d * d;
      den += ref * ref;
    }
  *rel = den > 0 ? sqrt(num / den) : sqrt(num);
  *timeout = herr;
  cudaFree(dA); cudaFree(dB); cudaFree(dC); cudaFree(dErr); cudaFree(dT);
  return 0;
}

// Select the form of the mixed near-field replay for this process (1 the
// pre-split store, 0 the FP32 copy); returns the previous form.  A plan
// rebuilds its copy of the store at its next mixed replay.
extern "C" int efmm_near_variant(int split) {
  const int old = efmm::near_split_variant();
  efmm::g_near_split = split ? 1 : 0;
  return old;
}
