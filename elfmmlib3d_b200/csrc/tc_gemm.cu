// tc_gemm.cu -- batched FP32 products on the 5th-generation tensor cores.
//
// The same contraction as k_gemm_tn<float> (fmm.cu):
//   C[col][row] = sum_k A[k][row] * B[col][k]
// over 128 x 128 output tiles (GemmTask), computed with tcgen05.mma
// kind::tf32 and FP32 accumulation in tensor memory.  FP32 accuracy comes
// from the 3-term split of each operand into a TF32 head and a TF32 tail
// (x = hi + lo, hi = x rounded to TF32): A B ~ Ahi Bhi + Ahi Blo + Alo Bhi,
// the dropped Alo Blo term being 2^-22 relative.
//
// One CTA (256 threads) per tile.  Each K tile of 32 is staged from global
// memory through registers into shared memory in the canonical no-swizzle
// K-major UMMA layout (core matrices of 8 rows x 4 k, 16 bytes per row; A is
// transposed on the way: a lane loads 4 k of one row, the lanes of a warp
// 32 consecutive rows), split into head and tail on the way, two
// stages deep; one thread issues the 12 MMAs of a K tile into one of two
// 128 x 128 TMEM accumulators and commits them to the stage's mbarrier; the
// threads then drain the previous tile's accumulator with tcgen05.ld (warp
// w: lanes 32 (w % 4).., columns 64 (w / 4)..) into FP32 registers while the
// tensor cores work on the current one.  Every wait is bounded: a wait that
// runs out sets *err, waits (bounded) for the MMAs in flight, frees the TMEM
// and returns without storing.
#include <cuda_runtime.h>
#include <cstdint>
#include <cmath>
#include <vector>
#include <cstdlib>
#include "common.cuh"
#include "fmm.h"
#include "tc_common.cuh"

namespace efmm {

namespace {

constexpr int TC_BM = 128, TC_BK = 32, TC_THREADS = 256;
constexpr int TC_TILE_BYTES = TC_BM * TC_BK * 4;          // one A part, 16 KB
// per stage: A hi, A lo (16 KB each), B hi, B lo (BN x 32 x 4 bytes each)
template <int BN>
__host__ __device__ constexpr int tc_stage_bytes() { return 2 * TC_TILE_BYTES + 2 * BN * TC_BK * 4; }
template <int BN>
__host__ __device__ constexpr int tc_smem() { return 2 * tc_stage_bytes<BN>() + 1024 + 64; }  // two stages, alignment, barriers
// A and B (K-major): element (row, k) at (k % 4) * 4 + (row % 8) * 16 + (k / 4) * 128 + (row / 8) * 1024
constexpr uint32_t TC_LBO = 128, TC_SBO = 1024;

struct Quad {
  float v[4];
};

}  // namespace

// TC: the accumulation (and output) type, float or double (the K-tile sums
// of the tensor cores added in FP64: the near-field replay)
template <int BN, class TC>
__global__ void __launch_bounds__(TC_THREADS, 1)
k_gemm_tc(const GemmTask* __restrict__ tasks, const float* __restrict__ A, const float* __restrict__ B,
          TC* __restrict__ Cm, int* __restrict__ err) {
  constexpr int TC_STAGE_BYTES = tc_stage_bytes<BN>(), TC_BTILE = BN * TC_BK * 4;
  constexpr int RG = BN / 8;       // 8-row groups of B
  constexpr int NB = BN / 32;      // B quads per thread and K tile
  constexpr int NHALF = BN / 2;    // accumulator columns drained per warp
  constexpr uint32_t IDESC = tc_idesc_mn(TC_BM, BN);
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  // 1024-byte aligned operand region
  const uint32_t raw = smem_u32(tc_smem_raw);
  unsigned char* sm = tc_smem_raw + ((1024 - (raw & 1023)) & 1023);
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + 2 * TC_STAGE_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + 2 * TC_STAGE_BYTES + 16);
  const GemmTask t = tasks[blockIdx.x];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(2 * BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(smem_u32(&bars[0]), 1);
    mbar_init(smem_u32(&bars[1]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  const float* Ab = A + t.a_off;
  const float* Bb = B + t.b_off;
  const int nkt = (t.K + TC_BK - 1) / TC_BK;
  // staging roles (4 quads of A and 4 of B per thread and K tile)
  Quad qa[4], qb[NB];
  const bool bvec = ((t.b_off & 3) == 0) && ((t.ldb & 3) == 0);  // 16-byte rows of B
  auto load = [&](int kt) {
    const int k0 = kt * TC_BK;
#pragma unroll
    for (int it = 0; it < 4; it++) {
      const int b = it * 8 + warp;
      // A: row 32 (b % 4) + lane, k chunk b / 4 (k = 4 (b / 4) .. + 3): the
      // lanes of a warp read 32 consecutive rows of each k
      const int m = 32 * (b & 3) + lane, ka = 4 * (b >> 2);
      const int gm = t.row0 + m, gk = k0 + ka;
#pragma unroll
      for (int j = 0; j < 4; j++)
        qa[it].v[j] = (gk + j < t.K && gm < t.M) ? Ab[(size_t)(gk + j) * t.lda + gm] : 0.0f;
    }
#pragma unroll
    for (int it = 0; it < NB; it++) {
      const int b = it * 8 + warp;
      // B: n = 8 (b % RG) + lane % 8, k chunk 4 (b / RG) + lane / 8
      const int n = 8 * (b % RG) + (lane & 7), kc = 4 * (b / RG) + (lane >> 3);
      const int gn = t.col0 + n, gk2 = k0 + 4 * kc;
      if (bvec && gn < t.N && gk2 + 3 < t.K) {
        const float4 v = *reinterpret_cast<const float4*>(Bb + (size_t)gn * t.ldb + gk2);
        qb[it].v[0] = v.x; qb[it].v[1] = v.y; qb[it].v[2] = v.z; qb[it].v[3] = v.w;
      } else {
#pragma unroll
        for (int j = 0; j < 4; j++)
          qb[it].v[j] = (gn < t.N && gk2 + j < t.K) ? Bb[(size_t)gn * t.ldb + gk2 + j] : 0.0f;
      }
    }
  };
  auto store = [&](int s) {
    unsigned char* st = sm + s * TC_STAGE_BYTES;
#pragma unroll
    for (int it = 0; it < 4; it++) {
      const int b = it * 8 + warp;
      const int m = 32 * (b & 3) + lane, ca = b >> 2;
      const uint32_t offa = (m & 7) * 16 + ca * TC_LBO + (m >> 3) * TC_SBO;
      float4 hi, lo;
      hi.x = tf32_head(qa[it].v[0]); lo.x = qa[it].v[0] - hi.x;
      hi.y = tf32_head(qa[it].v[1]); lo.y = qa[it].v[1] - hi.y;
      hi.z = tf32_head(qa[it].v[2]); lo.z = qa[it].v[2] - hi.z;
      hi.w = tf32_head(qa[it].v[3]); lo.w = qa[it].v[3] - hi.w;
      *reinterpret_cast<float4*>(st + offa) = hi;
      *reinterpret_cast<float4*>(st + TC_TILE_BYTES + offa) = lo;
    }
#pragma unroll
    for (int it = 0; it < NB; it++) {
      const int b = it * 8 + warp;
      float4 hi, lo;
      const int n = 8 * (b % RG) + (lane & 7), kc = 4 * (b / RG) + (lane >> 3);
      const uint32_t offb = (n & 7) * 16 + kc * TC_LBO + (n >> 3) * TC_SBO;
      hi.x = tf32_head(qb[it].v[0]); lo.x = qb[it].v[0] - hi.x;
      hi.y = tf32_head(qb[it].v[1]); lo.y = qb[it].v[1] - hi.y;
      hi.z = tf32_head(qb[it].v[2]); lo.z = qb[it].v[2] - hi.z;
      hi.w = tf32_head(qb[it].v[3]); lo.w = qb[it].v[3] - hi.w;
      *reinterpret_cast<float4*>(st + 2 * TC_TILE_BYTES + offb) = hi;
      *reinterpret_cast<float4*>(st + 2 * TC_TILE_BYTES + TC_BTILE + offb) = lo;
    }
  };

  // The tensor cores accumulate with truncation, so a long accumulation in
  // tensor memory drifts (relative error ~ K x 2^-27); each K tile is
  // therefore accumulated afresh in one of two TMEM accumulators and added
  // into FP32 registers (round to nearest), which keeps the product as
  // accurate as an FP32 dot product.  Accumulator (t & 1) holds tile t.
  const int quarter = warp & 3, half = warp >> 2;
  TC acc[NHALF];
#pragma unroll
  for (int j = 0; j < NHALF; j++) acc[j] = (TC)0;
  auto drain = [&](int u) {  // add the accumulator of tile u into acc
    const uint32_t col0 = (uint32_t)(u & 1) * BN + NHALF * half;
    // every load issued, then one wait
    uint32_t r[NHALF];
#pragma unroll
    for (int c16 = 0; c16 < NHALF / 16; c16++) {
      const uint32_t addr = tmem + ((uint32_t)(32 * quarter) << 16) + col0 + 16 * c16;
      uint32_t* q = r + 16 * c16;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15}, [%16];"
          : "=r"(q[0]), "=r"(q[1]), "=r"(q[2]), "=r"(q[3]), "=r"(q[4]), "=r"(q[5]), "=r"(q[6]), "=r"(q[7]),
            "=r"(q[8]), "=r"(q[9]), "=r"(q[10]), "=r"(q[11]), "=r"(q[12]), "=r"(q[13]), "=r"(q[14]), "=r"(q[15])
          : "r"(addr));
    }
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < NHALF; j++) acc[j] += (TC)__uint_as_float(r[j]);
  };
  bool ok = true;
  if (nkt > 0) load(0);
  for (int kt = 0; kt < nkt; kt++) {
    const int s = kt & 1;
    store(s);  // stage s is free: tile kt - 2 finished before tile kt - 1 was drained
    if (kt + 1 < nkt) load(kt + 1);  // in flight while the tensor cores work on tile kt
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t base = smem_u32(sm + s * TC_STAGE_BYTES);
      const uint32_t ahi = base, alo = base + TC_TILE_BYTES, bhi = base + 2 * TC_TILE_BYTES,
                     blo = bhi + TC_BTILE;
      const uint32_t dacc = tmem + (uint32_t)s * BN;
      // K step i: the step-0 descriptors + 2 i TC_LBO bytes in the 16-byte
      // address field (descriptor arithmetic kept off the issuing thread's path)
      const uint64_t dah = umma_desc(ahi, TC_LBO, TC_SBO), dal = umma_desc(alo, TC_LBO, TC_SBO);
      const uint64_t dbh = umma_desc(bhi, TC_LBO, TC_SBO), dbl = umma_desc(blo, TC_LBO, TC_SBO);
#pragma unroll
      for (int i = 0; i < TC_BK / 8; i++) {
        const uint64_t o = (uint64_t)((2 * i * TC_LBO) >> 4);
        mma_tf32(dacc, dal + o, dbh + o, IDESC, i > 0 ? 1u : 0u);
        mma_tf32(dacc, dah + o, dbl + o, IDESC, 1u);
        mma_tf32(dacc, dah + o, dbh + o, IDESC, 1u);
      }
      mma_commit(smem_u32(&bars[s]));
    }
    if (kt >= 1) {
      const int u = kt - 1;
      ok = mbar_wait(smem_u32(&bars[u & 1]), (u >> 1) & 1);
      ok = __syncthreads_and(ok);  // one decision for the whole CTA
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      drain(u);
    }
  }
  if (ok && nkt > 0) {
    const int u = nkt - 1;
    ok = mbar_wait(smem_u32(&bars[u & 1]), (u >> 1) & 1);
    ok = __syncthreads_and(ok);
    if (ok) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      drain(u);
    }
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    // give the MMAs in flight another bounded wait before freeing their accumulators
    for (int u = (nkt >= 2 ? nkt - 2 : 0); u < nkt; u++) mbar_wait(smem_u32(&bars[u & 1]), (u >> 1) & 1);
  } else {
    const int row = t.row0 + 32 * quarter + lane;
    if (row < t.M) {
      TC* Cp = Cm + t.c_off + row;
#pragma unroll
      for (int j = 0; j < NHALF; j++) {
        const int col = t.col0 + NHALF * half + j;
        if (col < t.N) Cp[(size_t)col * t.ldc] = acc[j];
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * BN) : "memory");
}

// ----------------------------------------------------------------------
// The same product with the operand tiles streamed by cp.async into a ring
// of raw FP32 tiles in shared memory, RING tiles ahead of the tensor cores
// (RING = 4 for 64-wide tiles, 3 for 128-wide), so that several K tiles of
// loads are in flight per SM while the threads split the current tile into
// its TF32 head and tail (shared memory to shared memory, into the canonical
// layout of k_gemm_tc) and the previous tile's accumulator is drained.  The
// raw A tile is [32 k][128 rows] (rows contiguous, as in A), the raw B tile
// [BN columns][32 k] with its 16-byte chunks XOR-swizzled by the column, so
// that the conversion's reads are free of bank conflicts.  Rows of A and B
// that are 16-byte aligned and complete are copied in 16-byte pieces, other
// elements one by one (zero-filled past the matrix).  Bounded waits and the
// per-K-tile FP32 drain as in k_gemm_tc.
template <int BN>
__host__ __device__ constexpr int tc_ring_depth() { return 3; }
constexpr int TC_RING_THREADS = 512;  // 16 warps: 4 TMEM lane quarters x 4 column parts
// split stages (and TMEM accumulators): the drain of a K tile trails its MMAs
// by tc_ring_stages - 1 tiles, so that the tensor cores' completion latency
// of that many tiles is hidden
template <int BN>
__host__ __device__ constexpr int tc_ring_stages() { return BN == 64 ? 3 : 2; }
template <int BN>
__host__ __device__ constexpr int tc_raw_bytes() { return TC_BM * TC_BK * 4 + BN * TC_BK * 4; }
template <int BN>
__host__ __device__ constexpr int tc_ring_smem() {
  return tc_ring_stages<BN>() * tc_stage_bytes<BN>() + tc_ring_depth<BN>() * tc_raw_bytes<BN>() + 1024 + 64;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int srcbytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(srcbytes) : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src, int srcbytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(srcbytes) : "memory");
}

template <int BN, class TC>
__global__ void __launch_bounds__(TC_RING_THREADS, 1)
k_gemm_tc_ring(const GemmTask* __restrict__ tasks, const float* __restrict__ A, const float* __restrict__ B,
               TC* __restrict__ Cm, int* __restrict__ err) {
  constexpr int TC_STAGE_BYTES = tc_stage_bytes<BN>(), TC_BTILE = BN * TC_BK * 4;
  constexpr int RING = tc_ring_depth<BN>(), RAW = tc_raw_bytes<BN>(), RAW_A = TC_BM * TC_BK * 4;
  constexpr int NST = tc_ring_stages<BN>(), LAG = NST - 1;
  constexpr uint32_t TMEM_COLS = NST * BN <= 256 ? 256 : 512;
  constexpr int RT = TC_RING_THREADS, NW = RT / 32;
  constexpr int RG = BN / 8, NBW = BN / 4 / NW, NPART = BN / 4;
  constexpr int NCA = TC_BM * TC_BK / 4 / RT;  // A chunks of 16 bytes per thread and tile (2)
  constexpr int NCB = BN * TC_BK / 4 / RT;     // B chunks per thread and tile (1 or 2)
  constexpr uint32_t IDESC = tc_idesc_mn(TC_BM, BN);
  extern __shared__ __align__(1024) unsigned char tc_ring_raw[];
  const uint32_t raw = smem_u32(tc_ring_raw);
  unsigned char* sm = tc_ring_raw + ((1024 - (raw & 1023)) & 1023);
  unsigned char* ring = sm + NST * TC_STAGE_BYTES;
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring + RING * RAW);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(ring + RING * RAW + 32);
  const GemmTask t = tasks[blockIdx.x];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < NST; i++) mbar_init(smem_u32(&bars[i]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  const float* Ab = A + t.a_off;
  const float* Bb = B + t.b_off;
  const int nkt = (t.K + TC_BK - 1) / TC_BK;
  const bool avec = ((t.a_off & 3) == 0) && ((t.lda & 3) == 0);
  const bool bvec = ((t.b_off & 3) == 0) && ((t.ldb & 3) == 0);
  // copies of K tile kt into ring slot kt % RING (nothing past the last tile)
  auto issue = [&](int kt) {
    if (kt >= nkt) return;
    const uint32_t slot = smem_u32(ring + (kt % RING) * RAW);
    const int k0 = kt * TC_BK;
#pragma unroll
    for (int it = 0; it < NCA; it++) {
      const int c = tid + RT * it, k = c >> 5, mc = c & 31;
      const int gk = k0 + k, gm = t.row0 + 4 * mc;
      const uint32_t d = slot + (uint32_t)(k * TC_BM + 4 * mc) * 4;
      const float* g = Ab + (size_t)gk * t.lda + gm;
      if (avec && gk < t.K && gm + 3 < t.M) {
        cp_async16(d, g, 16);
      } else {
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const bool ok = gk < t.K && gm + j < t.M;
          cp_async4(d + 4 * j, ok ? (const void*)(g + j) : (const void*)Ab, ok ? 4 : 0);
        }
      }
    }
#pragma unroll
    for (int it = 0; it < NCB; it++) {
      const int c = tid + RT * it, n = c >> 3, kc = c & 7;
      const int gn = t.col0 + n, gk = k0 + 4 * kc;
      const uint32_t d = slot + RAW_A + (uint32_t)(n * 128 + ((kc ^ (n & 7)) * 16));
      const float* g = Bb + (size_t)gn * t.ldb + gk;
      if (bvec && gn < t.N && gk + 3 < t.K) {
        cp_async16(d, g, 16);
      } else {
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const bool ok = gn < t.N && gk + j < t.K;
          cp_async4(d + 4 * j, ok ? (const void*)(g + j) : (const void*)Bb, ok ? 4 : 0);
        }
      }
    }
  };
  // ring slot of tile kt -> head / tail in conversion stage s (canonical layout)
  auto convert = [&](int kt, int s) {
    const unsigned char* slot = ring + (kt % RING) * RAW;
    const float* ra = reinterpret_cast<const float*>(slot);
    unsigned char* st = sm + s * TC_STAGE_BYTES;
#pragma unroll
    for (int it = 0; it < 32 / NW; it++) {
      const int b = it * NW + warp;
      const int m = 32 * (b & 3) + lane, ca = b >> 2;
      float v[4];
#pragma unroll
      for (int j = 0; j < 4; j++) v[j] = ra[(4 * ca + j) * TC_BM + m];
      const uint32_t offa = (m & 7) * 16 + ca * TC_LBO + (m >> 3) * TC_SBO;
      float4 hi, lo;
      hi.x = tf32_head(v[0]); lo.x = v[0] - hi.x;
      hi.y = tf32_head(v[1]); lo.y = v[1] - hi.y;
      hi.z = tf32_head(v[2]); lo.z = v[2] - hi.z;
      hi.w = tf32_head(v[3]); lo.w = v[3] - hi.w;
      *reinterpret_cast<float4*>(st + offa) = hi;
      *reinterpret_cast<float4*>(st + TC_TILE_BYTES + offa) = lo;
    }
#pragma unroll
    for (int it = 0; it < NBW; it++) {
      const int b = it * NW + warp;
      const int n = 8 * (b % RG) + (lane & 7), kc = 4 * (b / RG) + (lane >> 3);
      const float4 v = *reinterpret_cast<const float4*>(slot + RAW_A + n * 128 + ((kc ^ (n & 7)) * 16));
      const uint32_t offb = (n & 7) * 16 + kc * TC_LBO + (n >> 3) * TC_SBO;
      float4 hi, lo;
      hi.x = tf32_head(v.x); lo.x = v.x - hi.x;
      hi.y = tf32_head(v.y); lo.y = v.y - hi.y;
      hi.z = tf32_head(v.z); lo.z = v.z - hi.z;
      hi.w = tf32_head(v.w); lo.w = v.w - hi.w;
      *reinterpret_cast<float4*>(st + 2 * TC_TILE_BYTES + offb) = hi;
      *reinterpret_cast<float4*>(st + 2 * TC_TILE_BYTES + TC_BTILE + offb) = lo;
    }
  };
  // drain: warp w reads TMEM lanes 32 (w % 4) .. + 31 (rows), columns
  // NPART (w / 4) .. + NPART - 1
  const int quarter = warp & 3, part = warp >> 2;
  TC acc[NPART];
#pragma unroll
  for (int j = 0; j < NPART; j++) acc[j] = (TC)0;
  auto drain = [&](int u) {
    const uint32_t col0 = (uint32_t)(u % NST) * BN + NPART * part;
    // every load issued, then one wait
    uint32_t r[NPART];
#pragma unroll
    for (int c16 = 0; c16 < NPART / 16; c16++) {
      const uint32_t addr = tmem + ((uint32_t)(32 * quarter) << 16) + col0 + 16 * c16;
      uint32_t* q = r + 16 * c16;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15}, [%16];"
          : "=r"(q[0]), "=r"(q[1]), "=r"(q[2]), "=r"(q[3]), "=r"(q[4]), "=r"(q[5]), "=r"(q[6]), "=r"(q[7]),
            "=r"(q[8]), "=r"(q[9]), "=r"(q[10]), "=r"(q[11]), "=r"(q[12]), "=r"(q[13]), "=r"(q[14]), "=r"(q[15])
          : "r"(addr));
    }
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < NPART; j++) acc[j] += (TC)__uint_as_float(r[j]);
  };
  // the first RING - 1 tiles in flight (one commit group per tile, empty past the end)
#pragma unroll
  for (int q = 0; q < RING - 1; q++) {
    issue(q);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  bool ok = true;
  int issued = -1;  // last tile whose MMAs were issued
  for (int kt = 0; kt < nkt; kt++) {
    const int s = kt % NST;
    asm volatile("cp.async.wait_group %0;" ::"n"(RING - 2) : "memory");
    __syncthreads();  // tile kt landed for every thread; slot of tile kt - 1 converted
    issue(kt + RING - 1);
    asm volatile("cp.async.commit_group;" ::: "memory");
    convert(kt, s);  // stage s is free: tile kt - NST finished before tile kt - 1 - LAG was drained
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t base = smem_u32(sm + s * TC_STAGE_BYTES);
      const uint32_t ahi = base, alo = base + TC_TILE_BYTES, bhi = base + 2 * TC_TILE_BYTES, blo = bhi + TC_BTILE;
      const uint32_t dacc = tmem + (uint32_t)s * BN;
      // K step i: the step-0 descriptors + 2 i TC_LBO bytes in the 16-byte
      // address field (descriptor arithmetic kept off the issuing thread's path)
      const uint64_t dah = umma_desc(ahi, TC_LBO, TC_SBO), dal = umma_desc(alo, TC_LBO, TC_SBO);
      const uint64_t dbh = umma_desc(bhi, TC_LBO, TC_SBO), dbl = umma_desc(blo, TC_LBO, TC_SBO);
#pragma unroll
      for (int i = 0; i < TC_BK / 8; i++) {
        const uint64_t o = (uint64_t)((2 * i * TC_LBO) >> 4);
        mma_tf32(dacc, dal + o, dbh + o, IDESC, i > 0 ? 1u : 0u);
        mma_tf32(dacc, dah + o, dbl + o, IDESC, 1u);
        mma_tf32(dacc, dah + o, dbh + o, IDESC, 1u);
      }
      mma_commit(smem_u32(&bars[s]));
    }
    issued = kt;
    if (kt >= LAG) {
      const int u = kt - LAG;
      ok = mbar_wait(smem_u32(&bars[u % NST]), (u / NST) & 1);
      ok = __syncthreads_and(ok);
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      drain(u);
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");  // no copy outlives the CTA
  // the last LAG tiles
  for (int u = nkt > LAG ? nkt - LAG : 0; ok && u < nkt; u++) {
    ok = mbar_wait(smem_u32(&bars[u % NST]), (u / NST) & 1);
    ok = __syncthreads_and(ok);
    if (ok) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      drain(u);
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    for (int u = (issued >= LAG ? issued - LAG : 0); u <= issued; u++)
      mbar_wait(smem_u32(&bars[u % NST]), (u / NST) & 1);
  } else {
    const int row = t.row0 + 32 * quarter + lane;
    if (row < t.M) {
      TC* Cp = Cm + t.c_off + row;
#pragma unroll
      for (int j = 0; j < NPART; j++) {
        const int col = t.col0 + NPART * part + j;
        if (col < t.N) Cp[(size_t)col * t.ldc] = acc[j];
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

namespace {
__device__ int g_tc_err;
int* g_tc_err_addr[64] = {};
}  // namespace

int* tc_err_ptr() {
  int dev = 0;
  EFMM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw CudaError{(int)cudaErrorInvalidDevice};
  if (!g_tc_err_addr[dev]) {
    void* p = nullptr;
    EFMM_CUDA_TRY(cudaGetSymbolAddress(&p, g_tc_err));
    g_tc_err_addr[dev] = static_cast<int*>(p);
  }
  return g_tc_err_addr[dev];
}

bool tc_take_error() {
  int* p = tc_err_ptr();
  int h = 0;
  EFMM_CUDA_TRY(cudaMemcpy(&h, p, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) EFMM_CUDA_TRY(cudaMemset(p, 0, sizeof(int)));
  return h != 0;
}

// ELFMM3D_TC=0 keeps the FP32 products on the CUDA cores (k_gemm_tn<float>)
bool tc_enabled() {
  static const bool on = [] {
    const char* e = getenv("ELFMM3D_TC");
    return !(e && e[0] == '0');
  }();
  return on;
}

// Which form of the product runs: 1 (default) the cp.async ring
// (k_gemm_tc_ring), 0 the register-staged k_gemm_tc; ELFMM3D_TC_RING=0 or
// efmm_tc_variant select the latter.
static int g_tc_ring = -1;
int tc_ring_variant() {
  if (g_tc_ring < 0) {
    const char* e = getenv("ELFMM3D_TC_RING");
    g_tc_ring = (e && e[0] == '0') ? 0 : 1;
  }
  return g_tc_ring;
}

template <class TC>
static void launch_gemm_tc_t(cudaStream_t st, int ntask, const GemmTask* tasks, const float* A, const float* B,
                             TC* C, int* err, int bn) {
  if (ntask <= 0) return;
  if (tc_ring_variant()) {
    if (bn == 64) {
      EFMM_CUDA_TRY(smem_raise(k_gemm_tc_ring<64, TC>, (int)(tc_ring_smem<64>())));
      k_gemm_tc_ring<64, TC><<<ntask, TC_RING_THREADS, tc_ring_smem<64>(), st>>>(tasks, A, B, C, err);
    } else {
      EFMM_CUDA_TRY(smem_raise(k_gemm_tc_ring<128, TC>, (int)(tc_ring_smem<128>())));
      k_gemm_tc_ring<128, TC><<<ntask, TC_RING_THREADS, tc_ring_smem<128>(), st>>>(tasks, A, B, C, err);
    }
    count_launch();
    EFMM_CUDA_TRY(cudaGetLastError());
    return;
  }
  if (bn == 64) {
    EFMM_CUDA_TRY(smem_raise(k_gemm_tc<64, TC>, (int)(tc_smem<64>())));
    k_gemm_tc<64, TC><<<ntask, TC_THREADS, tc_smem<64>(), st>>>(tasks, A, B, C, err);
  } else {
    EFMM_CUDA_TRY(smem_raise(k_gemm_tc<128, TC>, (int)(tc_smem<128>())));
    k_gemm_tc<128, TC><<<ntask, TC_THREADS, tc_smem<128>(), st>>>(tasks, A, B, C, err);
  }
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}

void launch_gemm_tc(cudaStream_t st, int ntask, const GemmTask* tasks, const float* A, const float* B, float* C,
                    int* err, int bn) {
  launch_gemm_tc_t<float>(st, ntask, tasks, A, B, C, err, bn);
}

void launch_gemm_tc(cudaStream_t st, int ntask, const GemmTask* tasks, const float* A, const float* B, double* C,
                    int* err, int bn) {
  launch_gemm_tc_t<double>(st, ntask, tasks, A, B, C, err, bn);
}

}  // namespace efmm

// Device check of the tensor-core product against an FP64 host product:
// random A (K x M, lda = M + 3), B (N x K, ldb = K + 1) in [-1, 1), C = the
// tiles of k_gemm_tc.  Returns 0 and the relative l2 error in *rel (and
// *timeout != 0 if a bounded wait ran out).
extern "C" int efmm_tc_gemm_selfcheck_tile(int M, int N, int K, int bn, int aligned, unsigned seed, double* rel,
                                           int* timeout) {
  using namespace efmm;
  if (M < 1 || N < 1 || K < 0 || M > 4096 || N > 4096 || K > 65536) return 16;
  if (bn != 64 && bn != 128) return 16;
  // aligned: rows of A and B start on 16-byte boundaries (vector loads of
  // B); else odd leading dimensions (scalar loads)
  const int lda = aligned ? (M + 3) / 4 * 4 : M + 3, ldb = aligned ? (K + 3) / 4 * 4 : K + 1, ldc = M + 1;
  std::vector<float> hA((size_t)K * lda), hB((size_t)N * ldb), hC((size_t)N * ldc, -7.0f);
  unsigned long long st = seed * 6364136223846793005ull + 1;
  auto uni = [&]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return (float)(((st >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0);
  };
  for (auto& v : hA) v = uni();
  for (auto& v : hB) v = uni();
  std::vector<GemmTask> tasks;
  for (int c0 = 0; c0 < N; c0 += bn)
    for (int r0 = 0; r0 < M; r0 += 128) tasks.push_back({0, 0, 0, M, N, K, lda, ldb, ldc, r0, c0});
  float *dA = nullptr, *dB = nullptr, *dC = nullptr;
  int* dErr = nullptr;
  GemmTask* dT = nullptr;
  auto fail = [&]() {
    cudaFree(dA); cudaFree(dB); cudaFree(dC); cudaFree(dErr); cudaFree(dT);
    return 256;
  };
  if (cudaMalloc(&dA, hA.size() * 4 + 16) || cudaMalloc(&dB, hB.size() * 4 + 16) ||
      cudaMalloc(&dC, hC.size() * 4) || cudaMalloc(&dErr, 4) || cudaMalloc(&dT, tasks.size() * sizeof(GemmTask)))
    return fail();
  cudaMemcpy(dA, hA.data(), hA.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dB, hB.data(), hB.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dC, hC.data(), hC.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dT, tasks.data(), tasks.size() * sizeof(GemmTask), cudaMemcpyHostToDevice);
  cudaMemset(dErr, 0, 4);
  try {
    launch_gemm_tc(0, (int)tasks.size(), dT, dA, dB, dC, dErr, bn);
  } catch (const CudaError&) {
    return fail();
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return fail();
  cudaMemcpy(hC.data(), dC, hC.size() * 4, cudaMemcpyDeviceToHost);
  int herr = 0;
  cudaMemcpy(&herr, dErr, 4, cudaMemcpyDeviceToHost);
  double num = 0, den = 0;
  for (int c = 0; c < N; c++)
    for (int r = 0; r < M; r++) {
      double ref = 0;
      for (int k = 0; k < K; k++) ref += (double)hA[(size_t)k * lda + r] * (double)hB[(size_t)c * ldb + k];
      const double d = (double)hC[(size_t)c * ldc + r] - ref;
      num += d * d;
      den += ref * ref;
    }
  *rel = den > 0 ? sqrt(num / den) : sqrt(num);
  *timeout = herr;
  cudaFree(dA); cudaFree(dB); cudaFree(dC); cudaFree(dErr); cudaFree(dT);
  return 0;
}

// Select the form of the tensor-core product for this process (1 the
// cp.async ring, 0 register staging); returns the previous form.
extern "C" int efmm_tc_variant(int ring) {
  const int old = efmm::tc_ring_variant();
  efmm::g_tc_ring = ring ? 1 : 0;
  return old;
}

extern "C" int efmm_tc_gemm_selfcheck(int M, int N, int K, unsigned seed, double* rel, int* timeout) {
  return efmm_tc_gemm_selfcheck_tile(M, N, K, 128, 0, seed, rel, timeout);
}
