// rot_tc.cu -- the FP32 factored translations (M2M, M2L, L2L) on the
// 5th-generation tensor cores.
//
// A translation is Bk(d) Z(|d|) Fw(d) (rotations.h): block diagonal in the
// degree n (the rotations, blocks of 2n + 2 rows) or in the order m (the
// shift along z, blocks of 2(p - m + 1) rows).  Every group (one offset d,
// one operator) applies the same three factors to all of its columns (box
// pairs x expansion columns), so each factor is a batched block product
//     OUT[col][block rows] = OP_block x IN[col][block rows]
// with thousands of columns per operator block.  Here the columns are the M
// dimension of tcgen05.mma (128 columns per CTA, one TMEM lane each), the
// block's output rows the N dimension and its input rows K:
//     D[col][i] = sum_k X[col][k] OP[i][k],
// kind::tf32 with FP32 accumulation and the 3-term split of both operands
// (x = hi + lo, hi = x rounded to TF32; hi hi + hi lo + lo hi, FP32
// accuracy as in tc_gemm.cu).  The operator blocks are stored split and in
// the canonical no-swizzle K-major layout (built on the host), so a CTA
// copies them; the expansion rows are split while staged.  Accumulators are
// drained per K chunk of 32 (the tensor cores truncate their sums).
//
// The three factors run as three launches (stage 0 Fw, 1 Z, 2 Bk) through
// two intermediate arrays in device memory, laid out [row][column] per
// segment of columns so that the drains and the next stage's loads are
// coalesced: Y (after Fw) in order-major rows (order m: rows (n, m, re/im)
// for n = m..p, each order block padded to a multiple of 8 rows), W (after
// Z) in degree-major rows (each degree block padded likewise).  Stage 2 adds
// alpha x Bk W into the destination expansions (through a transpose in
// shared memory, so that the atomic adds are coalesced).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include "common.cuh"
#include "fmm.h"
#include "harmonics.cuh"
#include "rotations.h"
#include "tc_common.cuh"

namespace efmm {

namespace {

constexpr int RTC_M = 128, RTC_THREADS = 256, RTC_KMAX = 64;
constexpr int RTC_ABYTES = RTC_M * RTC_KMAX * 4;             // one A part: 32 KB
constexpr int RTC_BBYTES = RTC_KMAX * RTC_KMAX * 4;          // one B part: 16 KB
constexpr int RTC_STAGE = 2 * RTC_ABYTES + 2 * RTC_BBYTES;   // 96 KB
constexpr int RTC_TROW = 129;                                // transpose rows (floats), conflict-free
constexpr int RTC_SMEM = 2 * RTC_STAGE + 1024 + 2048;        // stages, alignment, barriers and tables

__host__ __device__ inline int ceil8(int x) { return (x + 7) & ~7; }
__host__ __device__ inline int ceil16(int x) { return (x + 15) & ~15; }

// block q of stage s at order p: rows (2q + 2 for the rotations, 2(p - q + 1)
// for the shift)
__host__ __device__ inline int rtc_rows(int s, int p, int q) { return s == 1 ? 2 * (p - q + 1) : 2 * q + 2; }

__device__ __forceinline__ void tmem_ld8(uint32_t addr, float* v) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 8; j++) v[j] = __uint_as_float(r[j]);
}

}  // namespace

size_t rot_tc_smem() { return RTC_SMEM; }

// One CTA per task (128 columns of one segment); the CTA runs every block of
// the stage: while the tensor cores multiply block q, the threads load block
// q + 1 into registers and drain block q - 1.  Waits are bounded: one that
// runs out sets *err, waits (bounded) for the MMAs in flight, frees the TMEM
// and returns.
__global__ void __launch_bounds__(RTC_THREADS, 1)
k_rot_tc(int stage, const RotTcTask* __restrict__ tasks, const RotTcSeg* __restrict__ segs,
         const TransPair* __restrict__ pairs, const RotTcOp* __restrict__ ops, const float* __restrict__ tiles,
         int D, int C, const float* __restrict__ src, float* __restrict__ ybuf, float* __restrict__ wbuf,
         float* __restrict__ dst, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char rtc_raw[];
  const uint32_t raw = smem_u32(rtc_raw);
  unsigned char* sm = rtc_raw + ((1024 - (raw & 1023)) & 1023);
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + 2 * RTC_STAGE);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + 2 * RTC_STAGE + 16);
  int* zpad = reinterpret_cast<int*>(sm + 2 * RTC_STAGE + 64);         // [33]
  int* npad = zpad + 34;                                               // [33]
  float* colalpha = reinterpret_cast<float*>(npad + 34);               // [128]
  long long* colbase = reinterpret_cast<long long*>(sm + 2 * RTC_STAGE + 1024);  // [128]
  const RotTcTask t = tasks[blockIdx.x];
  const RotTcSeg sg = segs[t.seg];
  const RotTcOp op = ops[sg.group];
  const int p = op.p, nblk = p + 1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // per tile column: the source expansion (stage 0) or the destination
  // expansion and its factor (stage 2); -1 past the segment's columns
  if (tid < RTC_M) {
    const int col = t.col0 + tid;
    long long base = -1;
    float al = 0.0f;
    if (col < sg.ncols && stage != 1) {
      const TransPair pr = pairs[sg.pair0 + col / C];
      base = ((long long)(stage == 0 ? pr.src : pr.dst) * C + col % C) * D;
      al = (float)pr.alpha;
    }
    colbase[tid] = base;
    colalpha[tid] = al;
  }
  if (tid == 0) {
    int z = 0, w = 0;
    for (int q = 0; q <= p + 1; q++) {
      zpad[q] = z;
      npad[q] = w;
      if (q <= p) {
        z += ceil8(2 * (p - q + 1));
        w += ceil8(2 * q + 2);
      }
    }
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(256)
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

  // loading roles: A (the expansion rows, X^T): thread -> column m, chunks of
  // 4 rows kc = kh, kh + 2, ...; B (the operator tile, already split and in
  // the canonical layout): float4 tid, tid + 256, ...
  const int m = tid & (RTC_M - 1), kh = tid >> 7;
  // this thread's input column: the source expansion (stage 0) or the
  // segment column of Y / W (stages 1, 2); -1 past the segment
  const long long mybase = stage == 0 ? colbase[m] : (t.col0 + m < sg.ncols ? (long long)(t.col0 + m) : -1LL);
  float4 ra[8], rb[8];
  auto tile_off = [&](int q) {
    long long o = op.tiles[stage];
    for (int j = 0; j < q; j++) {
      const int b = rtc_rows(stage, p, j);
      o += 2LL * ceil16(b) * ceil8(b);
    }
    return o;
  };
  // input rows of block q: the expansion (stage 0), Y (1) or W (2)
  auto in_row0 = [&](int q) { return stage == 0 ? q * (q + 1) : (stage == 1 ? zpad[q] : npad[q]); };
  const float* inb = stage == 1 ? ybuf + sg.ybase : wbuf + sg.wbase;
  auto load = [&](int q) {
    const int bb = rtc_rows(stage, p, q), Kp = ceil8(bb), Np = ceil16(bb), r0 = in_row0(q);
#pragma unroll
    for (int it = 0; it < 8; it++) {
      const int kc = kh + 2 * it, k0 = 4 * kc;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (k0 < Kp && mybase >= 0 && k0 < bb) {
        if (stage == 0) {
          // expansion rows r0 + k: 8-byte aligned pairs (D and r0 even), bb even
          const float2 a = *reinterpret_cast<const float2*>(src + mybase + r0 + k0);
          v.x = a.x;
          v.y = a.y;
          if (k0 + 2 < bb) {
            const float2 b = *reinterpret_cast<const float2*>(src + mybase + r0 + k0 + 2);
            v.z = b.x;
            v.w = b.y;
          }
        } else {
          const float* g = inb + (long long)(r0 + k0) * sg.ncols + mybase;
          v.x = g[0];
          v.y = g[sg.ncols];
          if (k0 + 2 < bb) {
            v.z = g[2LL * sg.ncols];
            v.w = g[3LL * sg.ncols];
          }
        }
      }
      ra[it] = v;
    }
    const float4* tb = reinterpret_cast<const float4*>(tiles + tile_off(q));
    const int nb4 = Np * Kp / 2;  // hi and lo parts, float4 count
#pragma unroll
    for (int it = 0; it < 8; it++) {
      const int idx = tid + RTC_THREADS * it;
      rb[it] = idx < nb4 ? tb[idx] : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };
  auto store = [&](int s, int q) {
    const int bb = rtc_rows(stage, p, q), Kp = ceil8(bb), Np = ceil16(bb);
    unsigned char* st = sm + s * RTC_STAGE;
    const uint32_t sbo = (uint32_t)Kp * 32;
#pragma unroll
    for (int it = 0; it < 8; it++) {
      const int kc = kh + 2 * it;
      if (4 * kc < Kp) {
        const uint32_t off = (m & 7) * 16 + kc * 128 + (m >> 3) * sbo;
        const float4 x = ra[it];
        float4 hi, lo;
        hi.x = tf32_head(x.x); lo.x = x.x - hi.x;
        hi.y = tf32_head(x.y); lo.y = x.y - hi.y;
        hi.z = tf32_head(x.z); lo.z = x.z - hi.z;
        hi.w = tf32_head(x.w); lo.w = x.w - hi.w;
        *reinterpret_cast<float4*>(st + off) = hi;
        *reinterpret_cast<float4*>(st + RTC_ABYTES + off) = lo;
      }
    }
    const int nb4 = Np * Kp / 2;
    float4* bs = reinterpret_cast<float4*>(st + 2 * RTC_ABYTES);
#pragma unroll
    for (int it = 0; it < 8; it++) {
      const int idx = tid + RTC_THREADS * it;
      if (idx < nb4) bs[idx] = rb[it];
    }
  };
  auto issue = [&](int s, int q) {
    const int bb = rtc_rows(stage, p, q), Kp = ceil8(bb), Np = ceil16(bb);
    const uint32_t base = smem_u32(sm + s * RTC_STAGE);
    const uint32_t ahi = base, alo = base + RTC_ABYTES, bhi = base + 2 * RTC_ABYTES, blo = bhi + Np * Kp * 4;
    const uint32_t sbo = (uint32_t)Kp * 32, idesc = tc_idesc_mn(RTC_M, Np);
    for (int i = 0; i < Kp / 8; i++) {
      const uint32_t dacc = tmem + (uint32_t)(2 * s + (i >> 2)) * 64;
      const uint64_t dah = umma_desc(ahi + 2 * i * 128, 128, sbo), dal = umma_desc(alo + 2 * i * 128, 128, sbo);
      const uint64_t dbh = umma_desc(bhi + 2 * i * 128, 128, sbo), dbl = umma_desc(blo + 2 * i * 128, 128, sbo);
      mma_tf32(dacc, dal, dbh, idesc, (i & 3) ? 1u : 0u);
      mma_tf32(dacc, dah, dbl, idesc, 1u);
      mma_tf32(dacc, dah, dbh, idesc, 1u);
    }
    mma_commit(smem_u32(&bars[s]));
  };
  const int quarter = warp & 3, half = warp >> 2;
  const int j = 32 * quarter + lane;  // the tile column (TMEM lane) this thread drains
  const long long cb = t.col0 + j < sg.ncols ? (long long)(t.col0 + j) : -1LL;  // its segment column
  auto drain = [&](int q) {
    const int s = q & 1, bb = rtc_rows(stage, p, q), Kp = ceil8(bb);
    float* T = reinterpret_cast<float*>(sm + s * RTC_STAGE);  // stage 2: [row][RTC_TROW]
#pragma unroll
    for (int c8 = 0; c8 < 4; c8++) {
      const int i0 = 32 * half + 8 * c8;
      if (i0 >= bb) break;  // warp-uniform
      float v[8], w[8];
      const uint32_t lanebase = tmem + ((uint32_t)(32 * quarter) << 16);
      tmem_ld8(lanebase + (uint32_t)(2 * s) * 64 + i0, v);
      if (Kp > 32) {
        tmem_ld8(lanebase + (uint32_t)(2 * s + 1) * 64 + i0, w);
#pragma unroll
        for (int e = 0; e < 8; e++) v[e] += w[e];
      }
#pragma unroll
      for (int e = 0; e < 8; e++) {
        const int i = i0 + e;
        if (i >= bb) break;
        if (stage == 2) {
          T[i * RTC_TROW + j] = v[e];
        } else if (cb >= 0) {
          const int part = i & 1;
          long long row;
          if (stage == 0) {  // degree q, order i / 2 -> order-major Y
            const int mm = i >> 1;
            row = zpad[mm] + 2 * (q - mm) + part;
            ybuf[sg.ybase + row * sg.ncols + cb] = v[e];
          } else {  // order q, degree q + i / 2 -> degree-major W
            const int n = q + (i >> 1);
            row = npad[n] + 2 * q + part;
            wbuf[sg.wbase + row * sg.ncols + cb] = v[e];
          }
        }
      }
    }
    if (stage == 2) {
      __syncthreads();
      const int r0 = q * (q + 1);
      for (int jj = warp; jj < RTC_M; jj += RTC_THREADS / 32) {
        const long long b = colbase[jj];
        if (b < 0) continue;
        const float al = colalpha[jj];
        for (int i = lane; i < bb; i += 32) atomicAdd(dst + b + r0 + i, al * T[i * RTC_TROW + jj]);
      }
      __syncthreads();  // T (stage s) is overwritten by a later store
    }
  };

  bool ok = true;
  int issued = -1;  // last block whose MMAs were issued (the same on every thread)
  if (nblk > 0) load(0);
  for (int q = 0; q < nblk; q++) {
    const int s = q & 1;
    store(s, q);
    if (q + 1 < nblk) load(q + 1);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      issue(s, q);
    }
    issued = q;
    if (q >= 1) {
      const int u = q - 1;
      ok = mbar_wait(smem_u32(&bars[u & 1]), (u >> 1) & 1);
      ok = __syncthreads_and(ok);
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      drain(u);
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
  }
  if (ok && nblk > 0) {
    const int u = nblk - 1;
    ok = mbar_wait(smem_u32(&bars[u & 1]), (u >> 1) & 1);
    ok = __syncthreads_and(ok);
    if (ok) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      drain(u);
    }
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    // give the MMAs in flight a bounded wait before their accumulators are freed
    for (int u = (issued >= 1 ? issued - 1 : 0); u <= issued; u++) mbar_wait(smem_u32(&bars[u & 1]), (u >> 1) & 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256) : "memory");
}

void launch_rot_tc(cudaStream_t st, int stage, int ntask, const RotTcTask* tasks, const RotTcSeg* segs,
                   const TransPair* pairs, const RotTcOp* ops, const float* tiles, int D, int C, const float* src,
                   float* ybuf, float* wbuf, float* dst, int* err) {
  if (ntask <= 0) return;
  EFMM_CUDA_TRY(smem_raise(k_rot_tc, RTC_SMEM));
  k_rot_tc<<<ntask, RTC_THREADS, RTC_SMEM, st>>>(stage, tasks, segs, pairs, ops, tiles, D, C, src, ybuf, wbuf, dst,
                                                 err);
  count_launch();
  EFMM_CUDA_TRY(cudaGetLastError());
}

// TF32 value nearest to x, ties away from zero (cvt.rna.tf32.f32): the head
// of the 3-term split, on the host
static float tf32_rna_host(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return x;
  u = (u + 0x1000u) & ~0x1FFFu;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

int rot_tc_rows(int stage, int p, int q) { return rtc_rows(stage, p, q); }

int rot_tc_pad_rows(int stage, int p) {
  int r = 0;
  for (int q = 0; q <= p; q++) r += ceil8(rtc_rows(stage, p, q));
  return r;
}

void build_rot_tc_tiles(const std::vector<RotOp>& ops, const std::vector<float>& pool_rowmajor,
                        std::vector<RotTcOp>& tops, std::vector<float>& tiles) {
  const int ng = (int)ops.size();
  tops.resize(ng);
  long long tot = 0;
  for (int g = 0; g < ng; g++) {
    tops[g].p = ops[g].p;
    tops[g].pad = 0;
    for (int s = 0; s < 3; s++) {
      tops[g].tiles[s] = tot;
      for (int q = 0; q <= ops[g].p; q++) {
        const int b = rtc_rows(s, ops[g].p, q);
        tot += 2LL * ceil16(b) * ceil8(b);
      }
    }
  }
  tiles.assign((size_t)tot, 0.0f);
  for (int g = 0; g < ng; g++) {
    const int p = ops[g].p;
    if (p > 31) continue;  // blocks wider than 64 rows: the CUDA-core kernels serve them
    for (int s = 0; s < 3; s++) {
      long long o = tops[g].tiles[s];
      for (int q = 0; q <= p; q++) {
        const int b = rtc_rows(s, p, q), Kp = ceil8(b), Np = ceil16(b);
        // the block, row-major b x b (output row, input column)
        long long src;
        if (s == 0)
          src = ops[g].fw + 2LL * q * (q + 1) * (2 * q + 1) / 3;
        else if (s == 2)
          src = ops[g].bk + 2LL * q * (q + 1) * (2 * q + 1) / 3;
        else {
          // order blocks m' < q of sizes (2(p - m' + 1))^2 precede block q
          long long zo = 0;
          for (int mm = 0; mm < q; mm++) zo += 4LL * (p - mm + 1) * (p - mm + 1);
          src = ops[g].z + zo;
        }
        float* hi = &tiles[(size_t)o];
        float* lo = hi + (size_t)Np * Kp;
        for (int i = 0; i < b; i++)
          for (int k = 0; k < b; k++) {
            const float v = pool_rowmajor[(size_t)(src + (long long)i * b + k)];
            const float h = tf32_rna_host(v);
            const size_t e = (size_t)(k & 3) + (size_t)(i & 7) * 4 + (size_t)(k >> 2) * 32 + (size_t)(i >> 3) * Kp * 8;
            hi[e] = h;
            lo[e] = v - h;
          }
        o += 2LL * Np * Kp;
      }
    }
  }
}

}  // namespace efmm

// Host emulation of the three tensor-core stages (the same tiles, the same
// canonical-layout addressing, the same row maps between the stages, the
// 3-term split and the FP32 sums per K chunk of 32) on random normalised
// expansions, for one M2L, one M2M and one L2L group of order p, against the
// factored product of the same FP32 operators in FP64.  Returns the largest
// relative l2 difference in *rel (about 1e-7 when every map is right).
extern "C" int efmm_rot_tc_selfcheck(int p, unsigned seed, double* rel) {
  using namespace efmm;
  if (p < 1 || p > 31 || !rel) return 16;
  const std::vector<int> kinds = {0, 1, 2};
  const std::vector<int> orders = {p, p, p};
  const std::vector<double> offs = {2.0, -1.0, 3.0, 0.25, -0.25, 0.25, -0.25, 0.25, -0.25};
  std::vector<RotOp> rops;
  std::vector<double> pool;
  build_factored_ops(p, kinds, orders, offs, rops, pool);
  std::vector<double> w(2 * (size_t)ncoef(p));
  for (int n = 0; n <= p; n++)
    for (int m = 0; m <= n; m++)
      w[2 * cidx(n, m)] = w[2 * cidx(n, m) + 1] = std::exp(0.5 * (std::lgamma(n + m + 1.0) + std::lgamma(n - m + 1.0)));
  std::vector<float> poolf;
  normalise_factored_ops(kinds, rops, pool, w, poolf);
  std::vector<RotTcOp> tops;
  std::vector<float> tiles;
  build_rot_tc_tiles(rops, poolf, tops, tiles);
  const int dim = (p + 1) * (p + 2);
  std::vector<int> zpad(p + 2), npad(p + 2);
  for (int q = 0, z = 0, wn = 0; q <= p + 1; q++) {
    zpad[q] = z;
    npad[q] = wn;
    if (q <= p) {
      z += ceil8(2 * (p - q + 1));
      wn += ceil8(2 * q + 2);
    }
  }
  unsigned long long st = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto uni = [&]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return (float)(((st >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0);
  };
  double worst = 0.0;
  for (int g = 0; g < 3; g++) {
    std::vector<float> x(dim), Y(zpad[p + 1], 0.f), W(npad[p + 1], 0.f), out(dim, 0.f);
    for (int n = 0; n <= p; n++)
      for (int s = 0; s < 2 * n + 2; s++) x[n * (n + 1) + s] = s == 1 ? 0.f : uni();
    // one stage: input rows (a[k], k < b) -> output D[i], the kernel's arithmetic
    auto block = [&](int stage, int q, const float* a) {
      const int b = rtc_rows(stage, p, q), Kp = ceil8(b), Np = ceil16(b);
      long long o = tops[g].tiles[stage];
      for (int j = 0; j < q; j++) {
        const int bj = rtc_rows(stage, p, j);
        o += 2LL * ceil16(bj) * ceil8(bj);
      }
      const float* hi = &tiles[(size_t)o];
      const float* lo = hi + (size_t)Np * Kp;
      std::vector<float> D(b);
      for (int i = 0; i < b; i++) {
        float acc = 0.f;
        for (int c = 0; c < Kp; c += 32) {
          float part = 0.f;
          for (int k = c; k < std::min(Kp, c + 32); k++) {
            const float av = k < b ? a[k] : 0.f, ah = tf32_rna_host(av), al = av - ah;
            const size_t e = (size_t)(k & 3) + (size_t)(i & 7) * 4 + (size_t)(k >> 2) * 32 + (size_t)(i >> 3) * Kp * 8;
            part += al * hi[e] + ah * lo[e] + ah * hi[e];
          }
          acc += part;
        }
        D[i] = acc;
      }
      return D;
    };
    for (int n = 0; n <= p; n++) {
      const std::vector<float> D = block(0, n, &x[n * (n + 1)]);
      for (int i = 0; i < 2 * n + 2; i++) Y[zpad[i >> 1] + 2 * (n - (i >> 1)) + (i & 1)] = D[i];
    }
    for (int m = 0; m <= p; m++) {
      const std::vector<float> D = block(1, m, &Y[zpad[m]]);
      for (int i = 0; i < 2 * (p - m + 1); i++) W[npad[m + (i >> 1)] + 2 * m + (i & 1)] = D[i];
    }
    for (int n = 0; n <= p; n++) {
      const std::vector<float> D = block(2, n, &W[npad[n]]);
      for (int i = 0; i < 2 * n + 2; i++) out[n * (n + 1) + i] = D[i];
    }
    // FP64 product of the same FP32 blocks: Bk Z Fw x
    const RotOp& ro = rops[g];
    std::vector<double> f(dim, 0.0), zz(dim, 0.0), r(dim, 0.0);
    for (int n = 0; n <= p; n++) {
      const int bb = 2 * n + 2, r0 = n * (n + 1);
      const float* B = &poolf[ro.fw + 2LL * n * (n + 1) * (2 * n + 1) / 3];
      for (int i = 0; i < bb; i++)
        for (int k = 0; k < bb; k++) f[r0 + i] += (double)B[i * bb + k] * x[r0 + k];
    }
    long long zo = 0;
    for (int m = 0; m <= p; m++) {
      const int bz = 2 * (p - m + 1);
      const float* Z = &poolf[ro.z + zo];
      zo += (long long)bz * bz;
      for (int a = 0; a < bz; a++)
        for (int c = 0; c < bz; c++)
          zz[2 * cidx(m + a / 2, m) + (a & 1)] += (double)Z[a * bz + c] * f[2 * cidx(m + c / 2, m) + (c & 1)];
    }
    for (int n = 0; n <= p; n++) {
      const int bb = 2 * n + 2, r0 = n * (n + 1);
      const float* B = &poolf[ro.bk + 2LL * n * (n + 1) * (2 * n + 1) / 3];
      for (int i = 0; i < bb; i++)
        for (int k = 0; k < bb; k++) r[r0 + i] += (double)B[i * bb + k] * zz[r0 + k];
    }
    double num = 0, den = 0;
    for (int q = 0; q < dim; q++) {
      num += (out[q] - r[q]) * (out[q] - r[q]);
      den += r[q] * r[q];
    }
    worst = std::max(worst, std::sqrt(num / std::max(den, 1e-300)));
  }
  *rel = worst;
  return 0;
}

// Device check of the three tensor-core stages: one M2L, one M2M and one L2L
// group of order p, npair box pairs each with C columns per box (random
// normalised source expansions, pair factors alpha), against the factored
// product of the same FP32 operators in FP64 on the host.  Returns 0 and the
// relative l2 error of the destination expansions in *rel (*timeout != 0 if
// a bounded wait ran out).
extern "C" int efmm_rot_tc_selfcheck_device(int p, int C, int npair, unsigned seed, double* rel, int* timeout) {
  using namespace efmm;
  if (p < 1 || p > 31 || C < 1 || npair < 1 || C * npair > (1 << 20) || !rel || !timeout) return 16;
  const std::vector<int> kinds = {0, 1, 2};
  const std::vector<int> orders = {p, p, p};
  const std::vector<double> offs = {2.0, -1.0, 3.0, 0.25, -0.25, 0.25, -0.25, 0.25, -0.25};
  std::vector<RotOp> rops;
  std::vector<double> pool;
  build_factored_ops(p, kinds, orders, offs, rops, pool);
  std::vector<double> w(2 * (size_t)ncoef(p));
  for (int n = 0; n <= p; n++)
    for (int m = 0; m <= n; m++)
      w[2 * cidx(n, m)] = w[2 * cidx(n, m) + 1] = std::exp(0.5 * (std::lgamma(n + m + 1.0) + std::lgamma(n - m + 1.0)));
  std::vector<float> poolf;
  normalise_factored_ops(kinds, rops, pool, w, poolf);
  std::vector<RotTcOp> tops;
  std::vector<float> tiles;
  build_rot_tc_tiles(rops, poolf, tops, tiles);
  const int D = 2 * ncoef(p), dim = (p + 1) * (p + 2);
  // boxes: sources 0 .. 3 npair - 1, destinations 3 npair .. 3 npair + 2 (each
  // group's pairs add into one destination box, as M2L pairs do)
  const int nsrc = 3 * npair, nbox = nsrc + 3;
  unsigned long long st = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto uni = [&]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return (float)(((st >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0);
  };
  std::vector<float> hsrc((size_t)nbox * C * D, 0.f), hdst((size_t)nbox * C * D, 0.f);
  for (int b = 0; b < nsrc; b++)
    for (int c = 0; c < C; c++)
      for (int n = 0; n <= p; n++)
        for (int s = 0; s < 2 * n + 2; s++) hsrc[((size_t)b * C + c) * D + n * (n + 1) + s] = s == 1 ? 0.f : uni();
  std::vector<TransPair> hp;
  std::vector<RotTcSeg> segs;
  std::vector<RotTcTask> tasks;
  long long ny = 0, nw = 0;
  for (int g = 0; g < 3; g++) {
    for (int k = 0; k < npair; k++) hp.push_back({g * npair + k, nsrc + g, 0.5 + 0.25 * k});
    const int ncols = npair * C, si = (int)segs.size();
    segs.push_back({g, g * npair, ncols, 0, ny, nw});
    for (int c0 = 0; c0 < ncols; c0 += 128) tasks.push_back({si, c0});
    ny += (long long)rot_tc_pad_rows(0, p) * ncols;
    nw += (long long)rot_tc_pad_rows(1, p) * ncols;
  }
  float *dsrc = nullptr, *ddst = nullptr, *dy = nullptr, *dw = nullptr, *dtiles = nullptr;
  TransPair* dp = nullptr;
  RotTcSeg* dseg = nullptr;
  RotTcTask* dtask = nullptr;
  RotTcOp* dops = nullptr;
  int* derr = nullptr;
  auto fail = [&]() {
    cudaFree(dsrc); cudaFree(ddst); cudaFree(dy); cudaFree(dw); cudaFree(dtiles);
    cudaFree(dp); cudaFree(dseg); cudaFree(dtask); cudaFree(dops); cudaFree(derr);
    return 256;
  };
  if (cudaMalloc(&dsrc, hsrc.size() * 4) || cudaMalloc(&ddst, hdst.size() * 4) || cudaMalloc(&dy, ny * 4) ||
      cudaMalloc(&dw, nw * 4) || cudaMalloc(&dtiles, tiles.size() * 4) || cudaMalloc(&dp, hp.size() * sizeof(TransPair)) ||
      cudaMalloc(&dseg, segs.size() * sizeof(RotTcSeg)) || cudaMalloc(&dtask, tasks.size() * sizeof(RotTcTask)) ||
      cudaMalloc(&dops, tops.size() * sizeof(RotTcOp)) || cudaMalloc(&derr, 4))
    return fail();
  cudaMemcpy(dsrc, hsrc.data(), hsrc.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(ddst, hdst.data(), hdst.size() * 4, cudaMemcpyHostToDevice);
  cudaMemset(dy, 0xff, ny * 4);  // NaN: every row a stage reads must be written or skipped
  cudaMemset(dw, 0xff, nw * 4);
  cudaMemcpy(dtiles, tiles.data(), tiles.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dp, hp.data(), hp.size() * sizeof(TransPair), cudaMemcpyHostToDevice);
  cudaMemcpy(dseg, segs.data(), segs.size() * sizeof(RotTcSeg), cudaMemcpyHostToDevice);
  cudaMemcpy(dtask, tasks.data(), tasks.size() * sizeof(RotTcTask), cudaMemcpyHostToDevice);
  cudaMemcpy(dops, tops.data(), tops.size() * sizeof(RotTcOp), cudaMemcpyHostToDevice);
  cudaMemset(derr, 0, 4);
  try {
    for (int stage = 0; stage < 3; stage++)
      launch_rot_tc(0, stage, (int)tasks.size(), dtask, dseg, dp, dops, dtiles, D, C, dsrc, dy, dw, ddst, derr);
  } catch (const CudaError&) {
    return fail();
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return fail();
  cudaMemcpy(hdst.data(), ddst, hdst.size() * 4, cudaMemcpyDeviceToHost);
  int herr = 0;
  cudaMemcpy(&herr, derr, 4, cudaMemcpyDeviceToHost);
  // host reference: dst(box) = sum over pairs alpha Bk Z Fw src(box), FP64
  double num = 0, den = 0;
  for (int g = 0; g < 3; g++) {
    const RotOp& ro = rops[g];
    for (int c = 0; c < C; c++) {
      std::vector<double> ref(dim, 0.0);
      for (int k = 0; k < npair; k++) {
        const float* x = &hsrc[((size_t)(g * npair + k) * C + c) * D];
        std::vector<double> f(dim, 0.0), zz(dim, 0.0);
        for (int n = 0; n <= p; n++) {
          const int bb = 2 * n + 2, r0 = n * (n + 1);
          const float* B = &poolf[ro.fw + 2LL * n * (n + 1) * (2 * n + 1) / 3];
          for (int i = 0; i < bb; i++)
            for (int q = 0; q < bb; q++) f[r0 + i] += (double)B[i * bb + q] * x[r0 + q];
        }
        long long zo = 0;
        for (int m = 0; m <= p; m++) {
          const int bz = 2 * (p - m + 1);
          const float* Z = &poolf[ro.z + zo];
          zo += (long long)bz * bz;
          for (int a = 0; a < bz; a++)
            for (int q = 0; q < bz; q++)
              zz[2 * cidx(m + a / 2, m) + (a & 1)] += (double)Z[a * bz + q] * f[2 * cidx(m + q / 2, m) + (q & 1)];
        }
        for (int n = 0; n <= p; n++) {
          const int bb = 2 * n + 2, r0 = n * (n + 1);
          const float* B = &poolf[ro.bk + 2LL * n * (n + 1) * (2 * n + 1) / 3];
          for (int i = 0; i < bb; i++)
            for (int q = 0; q < bb; q++) ref[r0 + i] += (0.5 + 0.25 * k) * (double)B[i * bb + q] * zz[r0 + q];
        }
      }
      const float* got = &hdst[((size_t)(nsrc + g) * C + c) * D];
      for (int q = 0; q < dim; q++) {
        num += (got[q] - ref[q]) * (got[q] - ref[q]);
        den += ref[q] * ref[q];
      }
    }
  }
  *rel = std::sqrt(num / std::max(den, 1e-300));
  *timeout = herr;
  fail();  // frees everything
  return 0;
}
