// rot_tc.cu -- the FP32 factored translations (M2M, M2L, L2L) on the
// 5th-generation tensor cores, the three factors of a translation in one
// pass through shared memory.
//
// A translation is Bk(d) Z(|d|) Fw(d) (rotations.h): block diagonal in the
// degree n (the rotations, blocks of 2n + 2 rows) or in the order m (the
// shift along z, blocks of 2(p - m + 1) rows), the same three factors for
// every column (box pair x expansion column) of a group (one offset d).  A
// persistent CTA takes 32 columns of one group at a time (a task) and keeps
// them in shared memory, X[column][row] in FP32 (degree-major rows, each
// degree padded to a multiple of 4), through all three factors.  Each K
// chunk (32 input rows) of each block of each factor is one product on the
// tensor cores,
//     D[i][col] = sum_k OP[i][k] X[col][k]   (M = 64 operator rows,
//                                             N = 32 columns, K = 8 per MMA),
// kind::tf32 with the 3-term split of both operands (x = hi + lo, hi = x
// rounded to TF32; hi hi + hi lo + lo hi: FP32 accuracy).  The operator
// chunks are split on the host and stored in the canonical no-swizzle
// K-major layout, so the CTA copies them with cp.async (a ring of three,
// two chunks ahead); the X rows are gathered and split while staged (the
// shift along z reads the rows (n, m), n >= m, of order m, which lie apart in
// the degree-major layout).  Accumulators live in TMEM, one per K chunk (the
// tensor cores truncate their sums: chunks are summed in FP32 registers),
// two blocks deep, so that a block drains while the next one multiplies.
// The first two factors write their results back into X in place (a block
// reads and writes the same rows); the third adds alpha x the result into
// the destination expansions with coalesced atomic adds.  While a CTA
// applies the third factor, the next task's source columns are copied into
// the rows of X that the third factor has finished reading, so a task's
// input is resident when it starts.  Every wait is bounded: one that runs
// out sets *err, the CTA waits (bounded) for its MMAs in flight, frees its
// TMEM and returns.
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

constexpr int RTC_NC = RTC_COLS, RTC_THREADS = 256, RTC_M = 64, RTC_KC = 32;
constexpr int RTC_APART = RTC_M * RTC_KC * 4;   // one part (head or tail) of an operator chunk: 8 KB
constexpr int RTC_ASLOT = 2 * RTC_APART;        // 16 KB
constexpr int RTC_BPART = RTC_NC * RTC_KC * 4;  // 4 KB
constexpr int RTC_BSLOT = 2 * RTC_BPART;        // 8 KB
constexpr int RTC_NA = 3;                       // operator ring slots
constexpr int RTC_TMEM_COLS = 128;              // 2 blocks x 2 K chunks x 32 columns

__host__ __device__ inline int ceil8(int x) { return (x + 7) & ~7; }

// block q of stage s at order p: rows (2q + 2 for the rotations, 2(p - q + 1)
// for the shift); K chunks of 32 of its ceil8(rows) input rows
__host__ __device__ inline int rtc_rows(int s, int p, int q) { return s == 1 ? 2 * (p - q + 1) : 2 * q + 2; }
__host__ __device__ inline int rtc_nchunk(int s, int p, int q) { return (ceil8(rtc_rows(s, p, q)) + 31) >> 5; }
// first X row of degree n: degrees padded to a multiple of 4 rows
__host__ __device__ inline int xpad(int n) { return n * (n + 1) + 2 * ((n + 1) / 2); }
// X column stride (floats) for orders <= pmax: 16-byte rows, 4 banks apart
__host__ __device__ inline int rtc_xs(int pmax) { return ((xpad(pmax + 1) + 31) & ~31) + 4; }

// offset (floats) of chunk c of block q of stage s in the group's tiles
__host__ __device__ inline long long rtc_tile_off(const RotTcOp& op, int s, int q, int c) {
  long long o = op.tiles[s];
  for (int j = 0; j < q; j++) {
    const int b = ceil8(rtc_rows(s, op.p, j));
    o += 2LL * b * b;
  }
  return o + 2LL * ceil8(rtc_rows(s, op.p, q)) * RTC_KC * c;
}

// one task's columns: source and destination expansion offsets (-1 past the
// segment), pair factor; the task's index, group and order
struct RtcTaskInfo {
  long long sbase[RTC_NC], dbase[RTC_NC];
  float alpha[RTC_NC];
  int ti, group, p, valid;
};

constexpr size_t rtc_smem_bytes(int xs) {
  return 1024 + (size_t)RTC_NA * RTC_ASLOT + 2 * RTC_BSLOT + (size_t)RTC_NC * xs * 4 + 2 * sizeof(RtcTaskInfo) + 64;
}

// a unit: K chunk c of block q of stage s of the CTA's t-th task
struct RtcUnit {
  int t, s, q, c, valid;
};

__device__ __forceinline__ void tmem_ld16(uint32_t addr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}

}  // namespace

size_t rot_tc_smem(int pmax) { return rtc_smem_bytes(rtc_xs(pmax)); }

__global__ void __launch_bounds__(RTC_THREADS, 1)
k_rot_tc(int ntask, const RotTcTask* __restrict__ tasks, const RotTcSeg* __restrict__ segs,
         const TransPair* __restrict__ pairs, const RotTcOp* __restrict__ ops, const float* __restrict__ tiles, int D,
         int C, int XS, const float* __restrict__ src, float* __restrict__ dst, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char rtc_raw[];
  const uint32_t raw = smem_u32(rtc_raw);
  unsigned char* sm = rtc_raw + ((1024 - (raw & 1023)) & 1023);
  const uint32_t sA = smem_u32(sm), sB = sA + RTC_NA * RTC_ASLOT;
  float* X = reinterpret_cast<float*>(sm + RTC_NA * RTC_ASLOT + 2 * RTC_BSLOT);
  unsigned char* tbl = sm + RTC_NA * RTC_ASLOT + 2 * RTC_BSLOT + (size_t)RTC_NC * XS * 4;
  RtcTaskInfo* info = reinterpret_cast<RtcTaskInfo*>(tbl);                      // [2], by task parity
  uint64_t* bars = reinterpret_cast<uint64_t*>(tbl + 2 * sizeof(RtcTaskInfo));  // stg[2], blk[2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 4);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // the table of the CTA's k-th task
  auto fill = [&](int k) {
    RtcTaskInfo& I = info[k & 1];
    const int ti = blockIdx.x + k * gridDim.x;
    if (tid < RTC_NC) {
      long long sb = -1, db = -1;
      float al = 0.0f;
      if (ti < ntask) {
        const RotTcTask t = tasks[ti];
        const RotTcSeg sg = segs[t.seg];
        const int col = t.col0 + tid;
        if (col < sg.ncols) {
          const TransPair pr = pairs[sg.pair0 + col / C];
          sb = ((long long)pr.src * C + col % C) * D;
          db = ((long long)pr.dst * C + col % C) * D;
          al = (float)pr.alpha;
        }
      }
      I.sbase[tid] = sb;
      I.dbase[tid] = db;
      I.alpha[tid] = al;
    }
    if (tid == 0) {
      I.ti = ti;
      I.valid = ti < ntask;
      if (ti < ntask) {
        I.group = segs[tasks[ti].seg].group;
        I.p = ops[I.group].p;
      } else {
        I.group = 0;
        I.p = 0;
      }
    }
  };
  auto next_unit = [&](RtcUnit u) {
    const int p = info[u.t & 1].p;
    if (u.c + 1 < rtc_nchunk(u.s, p, u.q)) {
      u.c++;
      return u;
    }
    u.c = 0;
    if (u.q < p) {
      u.q++;
      return u;
    }
    u.q = 0;
    if (u.s < 2) {
      u.s++;
      return u;
    }
    u.s = 0;
    u.t++;
    u.valid = info[u.t & 1].valid;
    return u;
  };
  // source rows of degrees n0..n1 of a task into X (pairs of floats: source
  // rows n(n+1) + 2j, X rows xpad(n) + 2j)
  auto load_x = [&](const RtcTaskInfo& I, int n0, int n1) {
    if (n1 < n0) return;
    const int g0 = n0 * (n0 + 1) / 2, np = (n1 + 1) * (n1 + 2) / 2 - g0;
    for (int idx = tid; idx < RTC_NC * np; idx += RTC_THREADS) {
      const int col = idx / np, g = g0 + idx % np;
      const long long sb = I.sbase[col];
      if (sb < 0) continue;
      int n = (int)((sqrtf(8.0f * g + 1.0f) - 1.0f) * 0.5f);
      while (n * (n + 1) / 2 > g) n--;
      while ((n + 1) * (n + 2) / 2 <= g) n++;
      const int j = g - n * (n + 1) / 2;
      cp_async8(smem_u32(X + (size_t)col * XS + xpad(n) + 2 * j), src + sb + 2 * g);
    }
  };
  // operator chunk of unit u into ring slot `slot`
  auto load_a = [&](const RtcUnit& u, int slot) {
    const RotTcOp op = ops[info[u.t & 1].group];
    const int Mr = ceil8(rtc_rows(u.s, op.p, u.q)), Kc = min(RTC_KC, Mr - RTC_KC * u.c);
    const float* g = tiles + rtc_tile_off(op, u.s, u.q, u.c);
    const int n16 = Mr * Kc / 4;
    for (int i = tid; i < 2 * n16; i += RTC_THREADS) {
      const int part = i >= n16, j = i - part * n16;
      cp_async16(sA + slot * RTC_ASLOT + part * RTC_APART + j * 16, g + (size_t)part * Mr * Kc + 4 * j);
    }
  };
  // X rows of unit u, split into head and tail, into staging buffer `buf`
  // (N = 32 columns x K = Kc, canonical K-major)
  auto convert = [&](const RtcUnit& u, int buf) {
    const int p = info[u.t & 1].p, bb = rtc_rows(u.s, p, u.q), Kc = min(RTC_KC, ceil8(bb) - RTC_KC * u.c);
    const int col = tid & 31, kq = tid >> 5, k0 = 4 * kq, kk = RTC_KC * u.c + k0;
    if (k0 >= Kc) return;
    const float* xc = X + (size_t)col * XS;
    float v[4];
    if (u.s != 1) {
      const float4 w = *reinterpret_cast<const float4*>(xc + xpad(u.q) + kk);
      v[0] = w.x; v[1] = w.y; v[2] = w.z; v[3] = w.w;
      for (int e = 0; e < 4; e++)
        if (kk + e >= bb) v[e] = 0.0f;
    } else {
      // order q: K index k -> degree q + k / 2, part k & 1
      const int n = u.q + (kk >> 1);
      float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
      if (kk < bb) a = *reinterpret_cast<const float2*>(xc + xpad(n) + 2 * u.q);
      if (kk + 2 < bb) b = *reinterpret_cast<const float2*>(xc + xpad(n + 1) + 2 * u.q);
      v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
    float4 hi, lo;
    hi.x = tf32_head(v[0]); lo.x = v[0] - hi.x;
    hi.y = tf32_head(v[1]); lo.y = v[1] - hi.y;
    hi.z = tf32_head(v[2]); lo.z = v[2] - hi.z;
    hi.w = tf32_head(v[3]); lo.w = v[3] - hi.w;
    unsigned char* b = sm + RTC_NA * RTC_ASLOT + buf * RTC_BSLOT + (col & 7) * 16 + kq * 128 + (col >> 3) * Kc * 32;
    *reinterpret_cast<float4*>(b) = hi;
    *reinterpret_cast<float4*>(b + RTC_BPART) = lo;
  };
  uint32_t tmem = 0;
  // block (stage s, block q) of task slot ts, TMEM blocks bp: rows 16 w + lane
  // of sub-partition w (the M = 64 layout: row r in lane 32 (r / 16) + r % 16)
  auto drain = [&](int ts, int s, int q, int bp) {
    const RtcTaskInfo& I = info[ts];
    const int bb = rtc_rows(s, I.p, q), w4 = warp & 3, h = warp >> 2;
    if (16 * w4 >= bb) return;  // warp-uniform: no rows of this block in the sub-partition
    const uint32_t ta = tmem + ((uint32_t)(32 * w4) << 16) + (uint32_t)(2 * bp) * 32 + 16 * h;
    float v[16];
    tmem_ld16(ta, v);
    if (rtc_nchunk(s, I.p, q) > 1) {
      float w[16];
      tmem_ld16(ta + 32, w);
#pragma unroll
      for (int j = 0; j < 16; j++) v[j] += w[j];
    }
    const int i = 16 * w4 + lane;
    if (lane >= 16 || i >= bb) return;
    if (s == 2) {
      const int row = q * (q + 1) + i;
#pragma unroll
      for (int j = 0; j < 16; j++) {
        const long long db = I.dbase[16 * h + j];
        if (db >= 0) atomicAdd(dst + db + row, I.alpha[16 * h + j] * v[j]);
      }
    } else {
      const int xrow = s == 0 ? xpad(q) + i : xpad(q + (i >> 1)) + 2 * q + (i & 1);
#pragma unroll
      for (int j = 0; j < 16; j++) X[(size_t)(16 * h + j) * XS + xrow] = v[j];
    }
  };

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(RTC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int b = 0; b < 4; b++) mbar_init(smem_u32(&bars[b]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fill(0);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  tmem = *tmem_slot;
  const uint32_t stg[2] = {smem_u32(&bars[0]), smem_u32(&bars[1])};
  const uint32_t blk[2] = {smem_u32(&bars[2]), smem_u32(&bars[3])};
  const uint32_t idesc = tc_idesc_mn(RTC_M, RTC_NC);

  RtcUnit cur{0, 0, 0, 0, info[0].valid};
  RtcUnit pf1 = cur, pf2 = cur;
  if (cur.valid) {
    load_x(info[0], 0, info[0].p);
    asm volatile("cp.async.commit_group;" ::: "memory");
    load_a(cur, 0);
    asm volatile("cp.async.commit_group;" ::: "memory");
    pf1 = next_unit(cur);
    load_a(pf1, 1);
    asm volatile("cp.async.commit_group;" ::: "memory");
    pf2 = next_unit(pf1);
  }
  long long un = 0;  // units issued so far (staging buffer un & 1, ring slot un % 3)
  int bseq = 0;      // blocks committed so far (TMEM blocks and blk barrier bseq & 1)
  bool pend = false;
  int pts = 0, pss = 0, pq = 0, pseq = 0;  // the committed block not yet drained
  bool ok = true;
  auto drain_pending = [&]() {
    ok = mbar_wait(blk[pseq & 1], (pseq >> 1) & 1);
    ok = __syncthreads_and(ok);
    if (!ok) return;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    drain(pts, pss, pq, pseq & 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    pend = false;
  };
  while (cur.valid) {
    const bool task_start = cur.s == 0 && cur.q == 0 && cur.c == 0;
    const bool stage_start = cur.q == 0 && cur.c == 0;
    if (task_start)
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    else
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    __syncthreads();
    // a stage reads what the previous one wrote; a new task's table slot is
    // the one the pending block of the previous task still uses
    if (pend && stage_start) {
      drain_pending();
      if (!ok) break;
      __syncthreads();
    }
    if (task_start) {
      fill(cur.t + 1);
      __syncthreads();
    }
    const RtcTaskInfo& I = info[cur.t & 1];
    const int buf = (int)(un & 1);
    if (un >= 2) ok = mbar_wait(stg[buf], ((un - 2) >> 1) & 1);  // the MMAs of unit un - 2 read this buffer
    convert(cur, buf);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    ok = __syncthreads_and(ok);
    if (!ok) break;
    const int nch = rtc_nchunk(cur.s, I.p, cur.q);
    const bool last_chunk = cur.c + 1 == nch;
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int Kc = min(RTC_KC, ceil8(rtc_rows(cur.s, I.p, cur.q)) - RTC_KC * cur.c);
      const uint32_t ahi = sA + (uint32_t)(un % RTC_NA) * RTC_ASLOT, alo = ahi + RTC_APART;
      const uint32_t bhi = sB + (uint32_t)buf * RTC_BSLOT, blo = bhi + RTC_BPART;
      const uint32_t sbo = (uint32_t)Kc * 32;
      const uint32_t dacc = tmem + (uint32_t)(2 * (bseq & 1) + cur.c) * 32;
      for (int j = 0; j < Kc / 8; j++) {
        const uint64_t dah = umma_desc(ahi + j * 256, 128, sbo), dal = umma_desc(alo + j * 256, 128, sbo);
        const uint64_t dbh = umma_desc(bhi + j * 256, 128, sbo), dbl = umma_desc(blo + j * 256, 128, sbo);
        mma_tf32(dacc, dal, dbh, idesc, j ? 1u : 0u);
        mma_tf32(dacc, dah, dbl, idesc, 1u);
        mma_tf32(dacc, dah, dbh, idesc, 1u);
      }
      mma_commit(stg[buf]);
      if (last_chunk) mma_commit(blk[bseq & 1]);
    }
    // the previous block drains while this one multiplies
    if (pend) {
      drain_pending();
      if (!ok) break;
    }
    if (last_chunk) {
      pend = true;
      pts = cur.t & 1;
      pss = cur.s;
      pq = cur.q;
      pseq = bseq;
      bseq++;
    }
    // ring slot of unit un + 2 held the operator of unit un - 1
    if (un >= 1) ok = mbar_wait(stg[(un - 1) & 1], ((un - 1) >> 1) & 1);
    if (pf2.valid) load_a(pf2, (int)((un + 2) % RTC_NA));
    // the last factor has read the rows of degree q: the next task's source
    // rows of that degree (and, after the last block, of its higher degrees)
    if (cur.s == 2 && last_chunk) {
      const RtcTaskInfo& N = info[(cur.t + 1) & 1];
      if (N.valid) {
        if (cur.q <= N.p) load_x(N, cur.q, cur.q);
        if (cur.q == I.p) load_x(N, I.p + 1, N.p);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    ok = __syncthreads_and(ok);
    if (!ok) break;
    un++;
    cur = pf1;
    pf1 = pf2;
    if (pf2.valid) pf2 = next_unit(pf2);
  }
  if (ok && pend) drain_pending();
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    // bounded waits for the MMAs in flight before their TMEM and shared memory go
    for (long long v = un >= 2 ? un - 2 : 0; v <= un; v++) mbar_wait(stg[v & 1], (v >> 1) & 1);
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(RTC_TMEM_COLS)
                 : "memory");
}

void launch_rot_tc(cudaStream_t st, int ntask, const RotTcTask* tasks, const RotTcSeg* segs, const TransPair* pairs,
                   const RotTcOp* ops, const float* tiles, int D, int C, int pmax, const float* src, float* dst,
                   int* err) {
  if (ntask <= 0) return;
  if (pmax < 0 || pmax > 31) throw CudaError{(int)cudaErrorInvalidValue};
  static int nsm = [] {
    int dev = 0, n = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n;
  }();
  const int xs = rtc_xs(pmax);
  const size_t smem = rtc_smem_bytes(xs);
  EFMM_CUDA_TRY(smem_raise(k_rot_tc, (int)smem));
  k_rot_tc<<<std::min(ntask, nsm), RTC_THREADS, smem, st>>>(ntask, tasks, segs, pairs, ops, tiles, D, C, xs, src, dst,
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

// element (i, k) of a part of a chunk with Kc columns (floats): the canonical
// K-major layout, 8 x 4 cores of 128 bytes, core columns along K 128 bytes
// apart, 8-row groups Kc x 32 bytes apart
static inline size_t rtc_elem(int i, int k, int Kc) {
  return (size_t)(k & 3) + (size_t)(i & 7) * 4 + (size_t)(k >> 2) * 32 + (size_t)(i >> 3) * Kc * 8;
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
      if (ops[g].p > 31) continue;  // blocks wider than 64 rows: the CUDA-core kernels serve them
      for (int q = 0; q <= ops[g].p; q++) {
        const int b = ceil8(rtc_rows(s, ops[g].p, q));
        tot += 2LL * b * b;
      }
    }
  }
  tiles.assign((size_t)tot, 0.0f);
  for (int g = 0; g < ng; g++) {
    const int p = ops[g].p;
    if (p > 31) continue;
    for (int s = 0; s < 3; s++) {
      for (int q = 0; q <= p; q++) {
        const int b = rtc_rows(s, p, q), Mr = ceil8(b);
        // the block, row-major b x b (output row, input column)
        long long sb;
        if (s == 0)
          sb = ops[g].fw + 2LL * q * (q + 1) * (2 * q + 1) / 3;
        else if (s == 2)
          sb = ops[g].bk + 2LL * q * (q + 1) * (2 * q + 1) / 3;
        else {
          // order blocks m' < q of sizes (2(p - m' + 1))^2 precede block q
          long long zo = 0;
          for (int mm = 0; mm < q; mm++) zo += 4LL * (p - mm + 1) * (p - mm + 1);
          sb = ops[g].z + zo;
        }
        for (int c = 0; c * RTC_KC < Mr; c++) {
          const int Kc = std::min(RTC_KC, Mr - RTC_KC * c);
          float* hi = &tiles[(size_t)rtc_tile_off(tops[g], s, q, c)];
          float* lo = hi + (size_t)Mr * Kc;
          for (int i = 0; i < b; i++)
            for (int k = 0; k < Kc && RTC_KC * c + k < b; k++) {
              const float v = pool_rowmajor[(size_t)(sb + (long long)i * b + RTC_KC * c + k)];
              const float h = tf32_rna_host(v);
              hi[rtc_elem(i, k, Kc)] = h;
              lo[rtc_elem(i, k, Kc)] = v - h;
            }
        }
      }
    }
  }
}

}  // namespace efmm

namespace {

// The factored product Bk Z Fw x of one group in FP64 from the FP32 blocks
// (rows of x and the result in the expansion layout, degree n at n(n+1)).
std::vector<double> rtc_reference(const efmm::RotOp& ro, const std::vector<float>& poolf, int p, const float* x) {
  using namespace efmm;
  const int dim = (p + 1) * (p + 2);
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
  return r;
}

// one M2L, one M2M and one L2L group of order p, normalised FP32 operators
void rtc_test_ops(int p, std::vector<efmm::RotOp>& rops, std::vector<float>& poolf) {
  using namespace efmm;
  const std::vector<int> kinds = {0, 1, 2};
  const std::vector<int> orders = {p, p, p};
  const std::vector<double> offs = {2.0, -1.0, 3.0, 0.25, -0.25, 0.25, -0.25, 0.25, -0.25};
  std::vector<double> pool;
  build_factored_ops(p, kinds, orders, offs, rops, pool);
  std::vector<double> w(2 * (size_t)ncoef(p));
  for (int n = 0; n <= p; n++)
    for (int m = 0; m <= n; m++)
      w[2 * cidx(n, m)] = w[2 * cidx(n, m) + 1] = std::exp(0.5 * (std::lgamma(n + m + 1.0) + std::lgamma(n - m + 1.0)));
  normalise_factored_ops(kinds, rops, pool, w, poolf);
}

struct RtcRng {
  unsigned long long st;
  explicit RtcRng(unsigned seed) : st(seed * 6364136223846793005ull + 1442695040888963407ull) {}
  float uni() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return (float)(((st >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0);
  }
};

}  // namespace

// Host emulation of the kernel's arithmetic (the same tiles and their
// canonical-layout addressing, the padded X rows, the row maps of the three
// factors, the 3-term split and the FP32 sums per K chunk of 32) for one
// column of random normalised expansions through one M2L, one M2M and one
// L2L group of order p, against the factored product of the same FP32
// operators in FP64.  Returns the largest relative l2 difference in *rel
// (about 1e-7 when every map is right).
extern "C" int efmm_rot_tc_selfcheck(int p, unsigned seed, double* rel) {
  using namespace efmm;
  if (p < 1 || p > 31 || !rel) return 16;
  std::vector<RotOp> rops;
  std::vector<float> poolf;
  rtc_test_ops(p, rops, poolf);
  std::vector<RotTcOp> tops;
  std::vector<float> tiles;
  build_rot_tc_tiles(rops, poolf, tops, tiles);
  const int dim = (p + 1) * (p + 2);
  RtcRng rng(seed);
  double worst = 0.0;
  for (int g = 0; g < 3; g++) {
    std::vector<float> x(dim), X(xpad(p + 1) + 8, 0.f), out(dim, 0.f);
    for (int n = 0; n <= p; n++)
      for (int s = 0; s < 2 * n + 2; s++) x[n * (n + 1) + s] = s == 1 ? 0.f : rng.uni();
    for (int n = 0; n <= p; n++)
      for (int s = 0; s < 2 * n + 2; s++) X[xpad(n) + s] = x[n * (n + 1) + s];
    for (int st = 0; st < 3; st++)
      for (int q = 0; q <= p; q++) {
        const int b = rtc_rows(st, p, q), Mr = ceil8(b);
        auto inrow = [&](int k) { return st == 1 ? xpad(q + k / 2) + 2 * q + (k & 1) : xpad(q) + k; };
        std::vector<float> Dv(b, 0.f);
        for (int c = 0; c * RTC_KC < Mr; c++) {
          const int Kc = std::min(RTC_KC, Mr - RTC_KC * c);
          const float* hi = &tiles[(size_t)rtc_tile_off(tops[g], st, q, c)];
          const float* lo = hi + (size_t)Mr * Kc;
          for (int i = 0; i < b; i++) {
            float part = 0.f;
            for (int k = 0; k < Kc; k++) {
              const int kk = RTC_KC * c + k;
              const float av = kk < b ? X[inrow(kk)] : 0.f, ah = tf32_rna_host(av), al = av - ah;
              const size_t e = rtc_elem(i, k, Kc);
              part += al * hi[e] + ah * lo[e] + ah * hi[e];
            }
            Dv[i] += part;
          }
        }
        for (int i = 0; i < b; i++) {
          if (st == 2)
            out[q * (q + 1) + i] = Dv[i];
          else
            X[st == 0 ? xpad(q) + i : xpad(q + i / 2) + 2 * q + (i & 1)] = Dv[i];
        }
      }
    const std::vector<double> r = rtc_reference(rops[g], poolf, p, x.data());
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

// Device check of the kernel: one M2L, one M2M and one L2L group of order p,
// npair box pairs each with C columns per box (random normalised source
// expansions, pair factors alpha, a destination box per group), in one
// launch, against the factored product of the same FP32 operators in FP64
// on the host.  Returns 0 and the relative l2 error of the destination
// expansions in *rel (*timeout != 0 if a bounded wait ran out).
extern "C" int efmm_rot_tc_selfcheck_device(int p, int C, int npair, unsigned seed, double* rel, int* timeout) {
  using namespace efmm;
  if (p < 1 || p > 31 || C < 1 || npair < 1 || C * npair > (1 << 20) || !rel || !timeout) return 16;
  std::vector<RotOp> rops;
  std::vector<float> poolf;
  rtc_test_ops(p, rops, poolf);
  std::vector<RotTcOp> tops;
  std::vector<float> tiles;
  build_rot_tc_tiles(rops, poolf, tops, tiles);
  const int D = 2 * ncoef(p), dim = (p + 1) * (p + 2);
  // boxes: sources 0 .. 3 npair - 1, destinations 3 npair .. 3 npair + 2
  const int nsrc = 3 * npair, nbox = nsrc + 3;
  RtcRng rng(seed);
  std::vector<float> hsrc((size_t)nbox * C * D, 0.f), hdst((size_t)nbox * C * D, 0.f);
  for (int b = 0; b < nsrc; b++)
    for (int c = 0; c < C; c++)
      for (int n = 0; n <= p; n++)
        for (int s = 0; s < 2 * n + 2; s++) hsrc[((size_t)b * C + c) * D + n * (n + 1) + s] = s == 1 ? 0.f : rng.uni();
  std::vector<TransPair> hp;
  std::vector<RotTcSeg> segs;
  std::vector<RotTcTask> tasks;
  for (int g = 0; g < 3; g++) {
    for (int k = 0; k < npair; k++) hp.push_back({g * npair + k, nsrc + g, 0.5 + 0.25 * k});
    const int ncols = npair * C, si = (int)segs.size();
    segs.push_back({g, g * npair, ncols, 0});
    for (int c0 = 0; c0 < ncols; c0 += RTC_COLS) tasks.push_back({si, c0});
  }
  float *dsrc = nullptr, *ddst = nullptr, *dtiles = nullptr;
  TransPair* dp = nullptr;
  RotTcSeg* dseg = nullptr;
  RotTcTask* dtask = nullptr;
  RotTcOp* dops = nullptr;
  int* derr = nullptr;
  auto release = [&]() {
    cudaFree(dsrc); cudaFree(ddst); cudaFree(dtiles); cudaFree(dp); cudaFree(dseg); cudaFree(dtask);
    cudaFree(dops); cudaFree(derr);
  };
  if (cudaMalloc(&dsrc, hsrc.size() * 4) || cudaMalloc(&ddst, hdst.size() * 4) ||
      cudaMalloc(&dtiles, tiles.size() * 4) || cudaMalloc(&dp, hp.size() * sizeof(TransPair)) ||
      cudaMalloc(&dseg, segs.size() * sizeof(RotTcSeg)) || cudaMalloc(&dtask, tasks.size() * sizeof(RotTcTask)) ||
      cudaMalloc(&dops, tops.size() * sizeof(RotTcOp)) || cudaMalloc(&derr, 4)) {
    release();
    return 256;
  }
  cudaMemcpy(dsrc, hsrc.data(), hsrc.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(ddst, hdst.data(), hdst.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dtiles, tiles.data(), tiles.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dp, hp.data(), hp.size() * sizeof(TransPair), cudaMemcpyHostToDevice);
  cudaMemcpy(dseg, segs.data(), segs.size() * sizeof(RotTcSeg), cudaMemcpyHostToDevice);
  cudaMemcpy(dtask, tasks.data(), tasks.size() * sizeof(RotTcTask), cudaMemcpyHostToDevice);
  cudaMemcpy(dops, tops.data(), tops.size() * sizeof(RotTcOp), cudaMemcpyHostToDevice);
  cudaMemset(derr, 0, 4);
  try {
    launch_rot_tc(0, (int)tasks.size(), dtask, dseg, dp, dops, dtiles, D, C, p, dsrc, ddst, derr);
  } catch (const CudaError&) {
    release();
    return 256;
  }
  if (cudaDeviceSynchronize() != cudaSuccess) {
    release();
    return 256;
  }
  cudaMemcpy(hdst.data(), ddst, hdst.size() * 4, cudaMemcpyDeviceToHost);
  int herr = 0;
  cudaMemcpy(&herr, derr, 4, cudaMemcpyDeviceToHost);
  release();
  // host reference: dst(box) = sum over pairs alpha Bk Z Fw src(box), FP64
  double num = 0, den = 0;
  for (int g = 0; g < 3; g++)
    for (int c = 0; c < C; c++) {
      std::vector<double> ref(dim, 0.0);
      for (int k = 0; k < npair; k++) {
        const std::vector<double> r = rtc_reference(rops[g], poolf, p, &hsrc[((size_t)(g * npair + k) * C + c) * D]);
        for (int q = 0; q < dim; q++) ref[q] += (0.5 + 0.25 * k) * r[q];
      }
      const float* got = &hdst[((size_t)(nsrc + g) * C + c) * D];
      for (int q = 0; q < dim; q++) {
        num += (got[q] - ref[q]) * (got[q] - ref[q]);
        den += ref[q] * ref[q];
      }
    }
  *rel = std::sqrt(num / std::max(den, 1e-300));
  *timeout = herr;
  return 0;
}
