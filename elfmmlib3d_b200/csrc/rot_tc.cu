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
// chunk (32 input rows) of each block of each factor (a unit) is one product
// on the tensor cores,
//     D[i][col] = sum_k OP[i][k] X[col][k]   (M = 64 operator rows,
//                                             N = 32 columns, K = 8 per MMA),
// kind::tf32 with the 3-term split of both operands (x = hi + lo, hi = x
// rounded to TF32; hi hi + hi lo + lo hi: FP32 accuracy), one FP32
// accumulator in TMEM per K chunk (the tensor cores truncate their sums:
// chunks are summed in FP32 registers).
//
// Warps have roles and meet only at mbarriers, so that several units are in
// flight: one thread copies each unit's operator chunk (split on the host,
// canonical no-swizzle K-major layout) with an untiled bulk copy into a byte
// ring; four warps gather the unit's X rows (the shift along z reads the
// rows (n, m), n >= m, of order m, which lie apart in the degree-major
// layout), split them and stage them; one thread issues the MMAs; four warps
// drain each block's accumulators from TMEM (8 blocks deep), back into X in
// place for the first two factors (a block reads and writes the same rows),
// and as alpha x the result with coalesced atomic adds into the destination
// expansions for the third.  While the third factor runs, the staging warps
// copy the next task's source columns into the rows of X it has finished
// reading.  Every wait is bounded: one that runs out makes every role stop,
// sets *err, and the CTA waits (bounded) for its copies and MMAs in flight
// before its TMEM and shared memory go.
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

constexpr int RTC_NC = RTC_COLS, RTC_M = 64, RTC_KC = 32;
constexpr int RTC_ARING = 48 * 1024;            // operator chunks in flight, each in its own size
constexpr int RTC_NA = 16;                       // at most this many of them
constexpr int RTC_BPART = RTC_NC * RTC_KC * 4;   // 4 KB
constexpr int RTC_BSLOT = 2 * RTC_BPART;         // 8 KB
constexpr int RTC_NB = 4;                        // staged X chunks in flight
// TMEM: per block 2 K chunks x 32 columns; 8 blocks in flight
constexpr int RTC_NACC = 8;
constexpr int RTC_TMEM_COLS = 512;
// roles: warps 0-3 stage X (and load the sources), warps 4-7 drain TMEM
// (warp 4 + i reads TMEM lanes 32 i .. 32 i + 31), warp 8 issues the MMAs,
// warp 9 copies the operator chunks
constexpr int RTC_THREADS = 320, RTC_CONV = 128, RTC_DRAIN = 128;

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

// barriers: A full / empty per operator slot, B full / empty per staging
// buffer, accumulator full / empty per TMEM block, X ready (the drains of a
// stage done), teardown
struct RtcBars {
  uint64_t afull[RTC_NA], aempty[RTC_NA], bfull[RTC_NB], bempty[RTC_NB], cfull[RTC_NACC], cempty[RTC_NACC];
  uint64_t xready, done;
};
// per-role tables (by task parity): source offsets of the staging warps,
// destination offsets and pair factors of the draining warps; the ring
// offset of each operator chunk in flight
struct RtcTables {
  long long sbase[2][RTC_NC], dbase[2][RTC_NC];
  float alpha[2][RTC_NC];
  uint32_t aoff[RTC_NA], alen[RTC_NA];
  uint32_t tmem;
  int abort_;
};

// shared memory: the operator ring (the MMAs of a chunk read 64 operator
// rows from its start; rows past the chunk's own land in the staging
// buffers that follow: garbage in output rows nobody reads), the staging
// buffers, X, barriers, tables
constexpr size_t rtc_smem_bytes(int xs) {
  return 1024 + (size_t)RTC_ARING + (size_t)RTC_NB * RTC_BSLOT + (size_t)RTC_NC * xs * 4 + sizeof(RtcBars) +
         sizeof(RtcTables);
}

// 16 columns of TMEM (this warp's 32 lanes) into r; complete after tmem_wait()
__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
}
__device__ __forceinline__ void tmem_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void bar_named(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
// named barrier that returns, to every participant, whether any of them passed true
__device__ __forceinline__ bool bar_any(int id, int n, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred q, p;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.or.pred p, %2, %3, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(id), "r"(n)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// untiled bulk copy global -> shared, completion counted on an mbarrier
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// bounded wait for phase `parity`, giving up at once when another role has
// given up (*abort_ set); false when it gave up
__device__ __forceinline__ bool rtc_wait(uint32_t bar, uint32_t parity, volatile int* abort_) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (*abort_ || clock64() - t0 > TC_WAIT_CYCLES) {
      *abort_ = 1;
      return false;
    }
  }
  return true;
}

// the task of this CTA's k-th turn: order, group, segment columns
struct RtcTask {
  int ti, p, group, pair0, ncols, col0;
};
__device__ __forceinline__ RtcTask rtc_task(int k, int ntask, const RotTcTask* tasks, const RotTcSeg* segs,
                                            const RotTcOp* ops) {
  RtcTask r;
  r.ti = blockIdx.x + k * gridDim.x;
  if (r.ti >= ntask) {
    r.p = -1;
    return r;
  }
  const RotTcTask t = tasks[r.ti];
  const RotTcSeg sg = segs[t.seg];
  r.group = sg.group;
  r.p = ops[sg.group].p;
  r.pair0 = sg.pair0;
  r.ncols = sg.ncols;
  r.col0 = t.col0;
  return r;
}

}  // namespace

size_t rot_tc_smem(int pmax) { return rtc_smem_bytes(rtc_xs(pmax)); }

// The units of a task, in the order every role walks them: stages 0, 1, 2;
// blocks 0..p; K chunks.  Units index the operator ring (u % RTC_NA) and the
// staging buffers (u % RTC_NB), blocks the TMEM blocks (b % nacc), each
// role counting its own.
__global__ void __launch_bounds__(RTC_THREADS, 1)
k_rot_tc(int ntask, const RotTcTask* __restrict__ tasks, const RotTcSeg* __restrict__ segs,
         const TransPair* __restrict__ pairs, const RotTcOp* __restrict__ ops, const float* __restrict__ tiles, int D,
         int C, int XS, const float* __restrict__ src, float* __restrict__ dst, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char rtc_raw[];
  constexpr int nacc = RTC_NACC;  // blocks in flight in TMEM, 64 columns each
  const uint32_t raw = smem_u32(rtc_raw);
  unsigned char* sm = rtc_raw + ((1024 - (raw & 1023)) & 1023);
  const uint32_t sA = smem_u32(sm), sB = sA + RTC_ARING;
  unsigned char* bstage = sm + RTC_ARING;
  float* X = reinterpret_cast<float*>(sm + RTC_ARING + RTC_NB * RTC_BSLOT);
  RtcBars* B = reinterpret_cast<RtcBars*>(sm + RTC_ARING + RTC_NB * RTC_BSLOT + (size_t)RTC_NC * XS * 4);
  RtcTables* T = reinterpret_cast<RtcTables*>(B + 1);
  volatile int* abort_ = &T->abort_;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  auto bar = [](const uint64_t& b) { return smem_u32(&b); };

  if (tid == 0) {
    for (int i = 0; i < RTC_NA; i++) {
      mbar_init(bar(B->afull[i]), 1);
      mbar_init(bar(B->aempty[i]), 1);
    }
    for (int i = 0; i < RTC_NB; i++) {
      mbar_init(bar(B->bfull[i]), RTC_CONV);
      mbar_init(bar(B->bempty[i]), 1);
    }
    for (int i = 0; i < RTC_NACC; i++) {
      mbar_init(bar(B->cfull[i]), 1);
      mbar_init(bar(B->cempty[i]), RTC_DRAIN);
    }
    mbar_init(bar(B->xready), RTC_DRAIN);
    mbar_init(bar(B->done), 1);
    T->abort_ = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 8) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&T->tmem)),
                 "r"(RTC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = T->tmem;

  if (warp < 4) {
    // ---- staging warps: X rows of each unit, split, into a staging buffer
    const int ct = tid;  // 0..127
    // the source offsets of task k's columns (table k & 1)
    auto fill_src = [&](int k, const RtcTask& tk) {
      if (ct < RTC_NC) {
        long long sb = -1;
        const int col = tk.col0 + ct;
        if (tk.p >= 0 && col < tk.ncols) {
          const TransPair pr = pairs[tk.pair0 + col / C];
          sb = ((long long)pr.src * C + col % C) * D;
        }
        T->sbase[k & 1][ct] = sb;
      }
    };
    // source rows of degrees n0..n1 into X (pairs of floats: source rows
    // n(n+1) + 2j, X rows xpad(n) + 2j)
    // (warp w: columns 8 w .. 8 w + 7, lanes along a degree's pairs)
    auto load_x = [&](int k, int n0, int n1) {
      for (int n = n0; n <= n1; n++)
        for (int cc = 0; cc < RTC_NC / 4; cc++) {
          const int col = 8 * warp + cc;
          const long long sb = T->sbase[k & 1][col];
          if (sb < 0) continue;
          for (int j = lane; j <= n; j += 32)
            cp_async8(smem_u32(X + (size_t)col * XS + xpad(n) + 2 * j), src + sb + n * (n + 1) + 2 * j);
        }
      asm volatile("cp.async.commit_group;" ::: "memory");
    };
    RtcTask tk = rtc_task(0, ntask, tasks, segs, ops);
    fill_src(0, tk);
    bar_named(1, RTC_CONV);
    load_x(0, 0, tk.p);
    long long u = 0;
    int xphase = 0;
    bool ok = true;
    for (int k = 0; tk.p >= 0 && ok; k++) {
      const RtcTask nx = rtc_task(k + 1, ntask, tasks, segs, ops);
      fill_src(k + 1, nx);
      asm volatile("cp.async.wait_group 0;" ::: "memory");
      bar_named(1, RTC_CONV);  // this task's X rows and the next task's table in place
      for (int s = 0; s < 3 && ok; s++) {
        if (s > 0) {
          // the previous stage's drains are all in X
          bool stop = false;
          if (ct == 0) stop = !rtc_wait(bar(B->xready), xphase & 1, abort_);
          xphase++;
          if (bar_any(1, RTC_CONV, stop)) ok = false;
        }
        for (int q = 0; q <= tk.p && ok; q++) {
          const int bb = rtc_rows(s, tk.p, q), nch = rtc_nchunk(s, tk.p, q);
          for (int c = 0; c < nch; c++, u++) {
            const int buf = (int)(u % RTC_NB);
            bool stop = false;
            if (ct == 0) stop = (u >= RTC_NB && !rtc_wait(bar(B->bempty[buf]), ((u / RTC_NB) - 1) & 1, abort_)) || *abort_;
            if (bar_any(1, RTC_CONV, stop)) {
              ok = false;
              break;
            }
            const int Kc = min(RTC_KC, ceil8(bb) - RTC_KC * c);
            // thread -> (column, K quad); two passes of 128 cover 32 columns x 8 quads
            for (int w = ct; w < RTC_NC * 8; w += RTC_CONV) {
              const int col = w & 31, kq = w >> 5, k0 = 4 * kq, kk = RTC_KC * c + k0;
              if (k0 >= Kc) continue;
              const float* xc = X + (size_t)col * XS;
              float v[4];
              if (s != 1) {
                const float4 x4 = *reinterpret_cast<const float4*>(xc + xpad(q) + kk);
                v[0] = x4.x; v[1] = x4.y; v[2] = x4.z; v[3] = x4.w;
                for (int e = 0; e < 4; e++)
                  if (kk + e >= bb) v[e] = 0.0f;
              } else {
                // order q: K index k -> degree q + k / 2, part k & 1
                const int n = q + (kk >> 1);
                float2 a2 = make_float2(0.f, 0.f), b2 = make_float2(0.f, 0.f);
                if (kk < bb) a2 = *reinterpret_cast<const float2*>(xc + xpad(n) + 2 * q);
                if (kk + 2 < bb) b2 = *reinterpret_cast<const float2*>(xc + xpad(n + 1) + 2 * q);
                v[0] = a2.x; v[1] = a2.y; v[2] = b2.x; v[3] = b2.y;
              }
              float4 hi, lo;
              hi.x = tf32_head(v[0]); lo.x = v[0] - hi.x;
              hi.y = tf32_head(v[1]); lo.y = v[1] - hi.y;
              hi.z = tf32_head(v[2]); lo.z = v[2] - hi.z;
              hi.w = tf32_head(v[3]); lo.w = v[3] - hi.w;
              unsigned char* b = bstage + buf * RTC_BSLOT + (col & 7) * 16 + kq * 128 + (col >> 3) * Kc * 32;
              *reinterpret_cast<float4*>(b) = hi;
              *reinterpret_cast<float4*>(b + RTC_BPART) = lo;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive(bar(B->bfull[buf]));
          }
          // the last factor has read the rows of degree q: the next task's
          // source rows of that degree (after the last block, its higher ones)
          if (s == 2 && ok && nx.p >= 0) {
            bar_named(1, RTC_CONV);
            if (q <= nx.p) load_x(k + 1, q, q);
            if (q == tk.p) load_x(k + 1, tk.p + 1, nx.p);
          }
        }
      }
      tk = nx;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
  } else if (warp < 8) {
    // ---- draining warps: TMEM lanes 32 w4 .. 32 w4 + 15 hold rows 16 w4 ..
    // 16 w4 + 15 of a block (the M = 64 layout)
    const int dt = tid - 128, w4 = warp - 4;
    long long b = 0;
    int bslot = 0, bwrap = 0;  // b = bwrap nacc + bslot
    bool ok = true;
    RtcTask tk = rtc_task(0, ntask, tasks, segs, ops);
    for (int k = 0; tk.p >= 0 && ok; k++) {
      if (dt < RTC_NC) {
        long long db = -1;
        float al = 0.0f;
        const int col = tk.col0 + dt;
        if (col < tk.ncols) {
          const TransPair pr = pairs[tk.pair0 + col / C];
          db = ((long long)pr.dst * C + col % C) * D;
          al = (float)pr.alpha;
        }
        T->dbase[k & 1][dt] = db;
        T->alpha[k & 1][dt] = al;
      }
      bar_named(2, RTC_DRAIN);
      for (int s = 0; s < 3 && ok; s++) {
        for (int q = 0; q <= tk.p; q++, b++) {
          const int slot = bslot;
          const int par = bwrap & 1;
          if (++bslot == nacc) {
            bslot = 0;
            bwrap++;
          }
          bool stop = false;
          if (dt == 0) stop = !rtc_wait(bar(B->cfull[slot]), par, abort_);
          if (bar_any(2, RTC_DRAIN, stop)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const int bb = rtc_rows(s, tk.p, q);
          float v[32];
          if (16 * w4 < bb) {
            // chunk 0 at columns 0..31 of the block, chunk 1 at 32..63: all
            // loads issued, then one wait
            const uint32_t ta = tmem + ((uint32_t)(32 * w4) << 16) + (uint32_t)slot * 64;
            uint32_t r0[16], r1[16], r2[16], r3[16];
            tmem_ld16(ta, r0);
            tmem_ld16(ta + 16, r1);
            if (rtc_nchunk(s, tk.p, q) > 1) {
              tmem_ld16(ta + 32, r2);
              tmem_ld16(ta + 48, r3);
              tmem_wait();
#pragma unroll
              for (int j = 0; j < 16; j++) {
                v[j] = __uint_as_float(r0[j]) + __uint_as_float(r2[j]);
                v[16 + j] = __uint_as_float(r1[j]) + __uint_as_float(r3[j]);
              }
            } else {
              tmem_wait();
#pragma unroll
              for (int j = 0; j < 16; j++) {
                v[j] = __uint_as_float(r0[j]);
                v[16 + j] = __uint_as_float(r1[j]);
              }
            }
          }
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          mbar_arrive(bar(B->cempty[slot]));
          const int i = 16 * w4 + lane;
          if (16 * w4 < bb && lane < 16 && i < bb) {
            if (s == 2) {
              const int row = q * (q + 1) + i;
#pragma unroll
              for (int j = 0; j < 32; j++) {
                const long long db = T->dbase[k & 1][j];
                if (db >= 0) atomicAdd(dst + db + row, T->alpha[k & 1][j] * v[j]);
              }
            } else {
              const int xrow = s == 0 ? xpad(q) + i : xpad(q + (i >> 1)) + 2 * q + (i & 1);
#pragma unroll
              for (int j = 0; j < 32; j++) X[(size_t)j * XS + xrow] = v[j];
            }
          }
        }
        if (s < 2 && ok) mbar_arrive(bar(B->xready));  // this stage's rows are in X
      }
      tk = rtc_task(k + 1, ntask, tasks, segs, ops);
    }
  } else if (warp == 8) {
    // ---- MMA issuer
    if (lane == 0) {
      const uint32_t idesc = tc_idesc_mn(RTC_M, RTC_NC);
      long long u = 0, b = 0;
      int bslot = 0, bwrap = 0;  // b = bwrap nacc + bslot
      bool ok = true;
      RtcTask tk = rtc_task(0, ntask, tasks, segs, ops);
      for (int k = 0; tk.p >= 0 && ok; k++) {
        for (int s = 0; s < 3 && ok; s++)
          for (int q = 0; q <= tk.p && ok; q++, b++) {
            const int slot = bslot;
            if (bwrap > 0) ok = rtc_wait(bar(B->cempty[slot]), (bwrap - 1) & 1, abort_);
            if (++bslot == nacc) {
              bslot = 0;
              bwrap++;
            }
            const int Mr = ceil8(rtc_rows(s, tk.p, q)), nch = rtc_nchunk(s, tk.p, q);
            for (int c = 0; c < nch && ok; c++, u++) {
              const int a = (int)(u % RTC_NA), buf = (int)(u % RTC_NB);
              ok = rtc_wait(bar(B->afull[a]), (u / RTC_NA) & 1, abort_) &&
                   rtc_wait(bar(B->bfull[buf]), (u / RTC_NB) & 1, abort_);
              if (!ok) break;
              asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
              const int Kc = min(RTC_KC, Mr - RTC_KC * c);
              const uint32_t ahi = sA + T->aoff[a], alo = ahi + (uint32_t)Mr * Kc * 4;
              const uint32_t bhi = sB + (uint32_t)buf * RTC_BSLOT, blo = bhi + RTC_BPART;
              const uint32_t sbo = (uint32_t)Kc * 32;
              const uint32_t dacc = tmem + (uint32_t)slot * 64 + (uint32_t)c * 32;
              // descriptors of K step j: the step-0 ones + 256 bytes per step
              // in the 16-byte address field
              const uint64_t dah = umma_desc(ahi, 128, sbo), dal = umma_desc(alo, 128, sbo);
              const uint64_t dbh = umma_desc(bhi, 128, sbo), dbl = umma_desc(blo, 128, sbo);
              const int J = Kc / 8;
#pragma unroll
              for (int j = 0; j < RTC_KC / 8; j++) {
                if (j < J) {
                  const uint64_t o = (uint64_t)(16 * j);
                  mma_tf32(dacc, dal + o, dbh + o, idesc, j ? 1u : 0u);
                  mma_tf32(dacc, dah + o, dbl + o, idesc, 1u);
                  mma_tf32(dacc, dah + o, dbh + o, idesc, 1u);
                }
              }
              mma_commit(bar(B->aempty[a]));
              mma_commit(bar(B->bempty[buf]));
            }
            if (ok) mma_commit(bar(B->cfull[slot]));
          }
        tk = rtc_task(k + 1, ntask, tasks, segs, ops);
      }
      // every MMA issued has completed before the TMEM and shared memory go
      mma_commit(bar(B->done));
      mbar_wait(bar(B->done), 0);
    }
  } else {
    // ---- operator copies: one bulk copy per part of each unit's chunk, into
    // a ring of bytes (each chunk contiguous, wrapping to the start when it
    // does not fit before the end); a chunk's space is taken back once the
    // MMAs of the oldest chunks in flight are done
    if (lane == 0) {
      long long u = 0, oldest = 0;
      uint32_t head = 0;
      bool ok = true;
      RtcTask tk = rtc_task(0, ntask, tasks, segs, ops);
      for (int k = 0; tk.p >= 0 && ok; k++) {
        const RotTcOp op = ops[tk.group];
        for (int s = 0; s < 3 && ok; s++)
          for (int q = 0; q <= tk.p && ok; q++) {
            const int Mr = ceil8(rtc_rows(s, tk.p, q)), nch = rtc_nchunk(s, tk.p, q);
            for (int c = 0; c < nch; c++, u++) {
              const int Kc = min(RTC_KC, Mr - RTC_KC * c);
              const uint32_t bytes = (uint32_t)Mr * Kc * 4, len = 2 * bytes;
              const uint32_t pos = head + len <= (uint32_t)RTC_ARING ? head : 0;
              // [pos, pos + len) must hold no chunk in flight; at most RTC_NA in flight
              while (oldest < u) {
                const int o = (int)(oldest % RTC_NA);
                const uint32_t a0 = T->aoff[o], a1 = a0 + T->alen[o];
                // the chunks in flight lie in the circular range [a0, head)
                const bool wrapped = a0 >= head;  // the range runs past the end to the start
                bool clear;
                if (!wrapped)
                  clear = pos >= head || pos + len <= a0;
                else
                  clear = pos >= head && pos + len <= a0;
                (void)a1;
                if (clear && u - oldest < RTC_NA) break;
                ok = rtc_wait(bar(B->aempty[o]), (oldest / RTC_NA) & 1, abort_);
                if (!ok) break;
                oldest++;
              }
              if (!ok) break;
              const int a = (int)(u % RTC_NA);
              T->aoff[a] = pos;
              T->alen[a] = len;
              head = pos + len;
              const float* g = tiles + rtc_tile_off(op, s, q, c);
              mbar_expect_tx(bar(B->afull[a]), len);
              bulk_g2s(sA + pos, g, bytes, bar(B->afull[a]));
              bulk_g2s(sA + pos + bytes, g + (size_t)Mr * Kc, bytes, bar(B->afull[a]));
            }
          }
        tk = rtc_task(k + 1, ntask, tasks, segs, ops);
      }
      // copies still in flight land before the shared memory goes
      for (long long v = u > RTC_NA ? u - RTC_NA : 0; v < u; v++)
        mbar_wait(bar(B->afull[v % RTC_NA]), (v / RTC_NA) & 1);
    }
  }
  __syncwarp();
  __syncthreads();
  if (tid == 0 && T->abort_) atomicExch(err, 1);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 8)
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

// The kernel on one M2L, one M2M and one L2L group of order p, npair box
// pairs each with C columns per box (random normalised source expansions,
// pair factors alpha, a destination box per group), in one launch; reps > 1
// launches it reps times more and returns the mean ms of those in *ms.  With
// rel: the relative l2 error of the destination expansions of the first
// launch against the factored product of the same FP32 operators in FP64 on
// the host.  *timeout != 0 if a bounded wait ran out.
static int rtc_device_run(int p, int C, int npair, unsigned seed, int reps, double* rel, int* timeout, double* ms) {
  using namespace efmm;
  if (p < 1 || p > 31 || C < 1 || npair < 1 || C * npair > (1 << 20) || !timeout) return 16;
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
  if (reps > 1 && ms) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, 0);
    try {
      for (int r = 0; r < reps; r++)
        launch_rot_tc(0, (int)tasks.size(), dtask, dseg, dp, dops, dtiles, D, C, p, dsrc, ddst, derr);
    } catch (const CudaError&) {
      release();
      return 256;
    }
    cudaEventRecord(e1, 0);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      release();
      return 256;
    }
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    *ms = t / reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  int herr = 0;
  cudaMemcpy(&herr, derr, 4, cudaMemcpyDeviceToHost);
  release();
  *timeout = herr;
  if (!rel) return 0;
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
  return 0;
}

// Device check of the kernel (rtc_device_run, one launch): returns 0 and
// the relative l2 error of the destination expansions in *rel.
extern "C" int efmm_rot_tc_selfcheck_device(int p, int C, int npair, unsigned seed, double* rel, int* timeout) {
  if (!rel) return 16;
  return rtc_device_run(p, C, npair, seed, 1, rel, timeout, nullptr);
}

// Timing of the kernel on the same inputs: mean ms of reps launches.
extern "C" int efmm_rot_tc_bench(int p, int C, int npair, int reps, double* ms, int* timeout) {
  if (reps < 1 || !ms) return 16;
  return rtc_device_run(p, C, npair, 1, reps + 1, nullptr, timeout, ms);
}
