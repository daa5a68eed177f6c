// Low-precision trailing update of the mixed-precision LU on the 5th-generation
// tensor cores:   C (fp32) -= sA[tile_m] * sB[tile_n] * (A16 B16^T)
// with A16 (m x k) and B16 (n x k) BF16 or FP16, both K-major (row-major with
// k contiguous), and FP32 accumulation in tensor memory.
//
// Pairs of CTAs (a 2-CTA cluster, one CTA per SM) compute 256 x 256 tiles with
// the two-SM MMA (tcgen05.mma.cta_group::2, M = 256, N = 256, K = 16): CTA r
// of the pair holds rows r*128 .. r*128+127 of the tile's A slice and rows
// r*128 .. r*128+127 of its B slice in its own shared memory, the MMA issued
// by CTA 0 reads both, and each CTA's TMEM receives its 128 x 256 part of the
// accumulator.  Per SM and k-block that is 32 KB of operands instead of the
// 48 KB a one-SM 128 x 256 tile needs, so six stages fit where four did and
// the operand feed from L2 keeps ahead of the MMAs.  320 threads per CTA:
//   warp 0      TMA producer (both CTAs): its A and B halves of each 64-deep
//               k-block (128-byte rows, 128B swizzle) into a 6-stage ring; the
//               loads of both CTAs complete on CTA 0's "full" barrier, whose
//               transaction count CTA 0 posts for the pair; each CTA loads only its own halves.
//   warp 1      allocates 512 TMEM columns in both CTAs (two accumulators,
//               collectively for the pair); in CTA 0 one lane issues the MMAs
//               and tcgen05.commit's with multicast to both CTAs' "empty" ring
//               barriers and "accumulator full" barriers.
//   warps 2..9  epilogue (both CTAs): tcgen05.ld of the accumulator rows their
//               TMEM lane group may read, scale, and C -= in FP32, then an
//               arrive on CTA 0's "accumulator drained" barrier (16 arrivals:
//               8 local, 8 from the peer).  Two accumulators let the epilogue
//               of one tile overlap the MMAs of the next.  When C allows a TMA
//               map (16-byte aligned base, ldc a multiple of 4) the epilogue
//               writes -scale * acc in 16-column chunks to a per-warp staging
//               buffer and hands each to a TMA reduce-add
//               (cp.reduce.async.bulk.tensor ... .add), so the read-modify-write
//               of C happens in L2; otherwise it loads, subtracts and stores C.
// Every mbarrier wait is bounded; on expiry the CTA records the site and the
// roles leave their loops; both CTAs then meet at a cluster barrier, release
// TMEM and exit.
#include <cstdlib>
#include <cstring>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.cuh"
#include "internal.h"

namespace hplb {

namespace {

constexpr int LBM = 128;               // tile rows per CTA (256 per pair)
constexpr int LBN = 256;               // tile columns (B rows; 128 per CTA)
// Ring depth and the epilogue's chunking are compile-time choices (defaults
// measured best on B200; -D overrides exist for tuning builds only).
#ifndef HPLB_LP_STAGES
#define HPLB_LP_STAGES 6
#endif
#ifndef HPLB_LP_EPI_COLS
#define HPLB_LP_EPI_COLS 16
#endif
#ifndef HPLB_LP_EPI_BUFS
#define HPLB_LP_EPI_BUFS 2
#endif
constexpr int LBK = 64, LSTAGES = HPLB_LP_STAGES;
constexpr int L_THREADS = 320;
constexpr int L_EPI_WARPS = 8;
constexpr int LA_BYTES = LBM * LBK * 2;        // 16 KB
constexpr int LB_BYTES = (LBN / 2) * LBK * 2;  // 16 KB: this CTA's half of B
constexpr int LSTAGE_BYTES = LA_BYTES + LB_BYTES;
constexpr int L_SMEM = LSTAGES * LSTAGE_BYTES + 1024 + 256;
constexpr int L_EPI_COLS = HPLB_LP_EPI_COLS;          // columns per staged chunk
constexpr int L_EPI_BUFS = HPLB_LP_EPI_BUFS;          // staging buffers per warp
constexpr int L_STG_BYTES = L_EPI_COLS * 32 * 4;      // one warp's chunk
constexpr int L_STG_TOTAL = L_EPI_WARPS * L_EPI_BUFS * L_STG_BYTES;
static_assert(L_EPI_COLS == 16 || L_EPI_COLS == 32, "epilogue chunks of 16 or 32 columns");
constexpr int L_SMEM_TMA = L_SMEM + L_STG_TOTAL;
constexpr int L_GROUP_N = 8;  // column tiles per group (A and B stay in L2)

HPLB_DEV uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

HPLB_DEV void bar_init(uint64_t* b, int c) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(c) : "memory");
}
HPLB_DEV void bar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)),
               "r"(bytes)
               : "memory");
}
HPLB_DEV bool bar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
HPLB_DEV bool bar_wait(uint64_t* b, uint32_t parity, volatile int* abort) {
  if(bar_try(b, parity)) return true;
  const unsigned long long t0 = globaltimer();
  while(!bar_try(b, parity)) {
    if(*abort) return false;
    if(globaltimer() - t0 > kWaitBudgetNs) return false;
  }
  return true;
}
HPLB_DEV uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// The shared::cluster address of the same shared-memory offset in CTA `rank`.
HPLB_DEV uint32_t mapa_shared(uint32_t addr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
HPLB_DEV void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n"
               "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
HPLB_DEV void bar_arrive_cluster(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr)
               : "memory");
}
// Tiled load into this CTA's shared memory whose completion is counted on the
// pair's barrier at bar (CTA 0's, for both CTAs).
HPLB_DEV void tma2d_pair(void* dst, const CUtensorMap* map, uint32_t bar, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(su32(dst)),
      "l"(map), "r"(bar), "r"(c0), "r"(c1)
      : "memory");
}


// Shared-memory matrix descriptor: K-major, 128B swizzle, 8-row atoms of
// 1024 bytes stacked densely (SBO = 1024 B), descriptor version 1.
HPLB_DEV uint64_t umma_desc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;              // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;    // stride byte offset
  d |= (uint64_t)1 << 46;              // version
  d |= (uint64_t)2 << 61;              // SWIZZLE_128B
  return d;
}

HPLB_DEV void umma_f16_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                            uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// Arrive once on the barrier at this offset in every CTA of `mask` when the
// MMAs issued so far have completed.
HPLB_DEV void umma_commit_pair(uint64_t* bar, uint16_t mask) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64"
      " [%0], %1;" ::"r"(su32(bar)),
      "h"(mask)
      : "memory");
}

// 16 or 32 consecutive accumulator columns of this warp's 32 TMEM lanes.
template <int NC>
HPLB_DEV void tmem_ld_cols(uint32_t taddr, uint32_t (&r)[NC]) {
  if constexpr(NC == 16) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,"
        "%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
  } else {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,"
        "%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31},"
        " [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
  }
}

// Wait until at most N of this thread's committed bulk groups still read
// shared memory.
template <int N>
HPLB_DEV void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

// C(x, y) += smem chunk, x = row (inner), y = column; out-of-range parts of
// the box are skipped by the TMA unit.
HPLB_DEV void tma_reduce_add2d(const CUtensorMap* map, const void* src, int c0, int c1) {
  asm volatile(
      "cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group"
      " [%0, {%2, %3}], [%1];" ::"l"(map),
      "r"(su32(src)), "r"(c0), "r"(c1)
      : "memory");
}

HPLB_DEV void tile_of(int t, int tiles_m, int tiles_n, int& tm, int& tn) {
  const int per = tiles_m * L_GROUP_N;
  const int grp = t / per;
  const int r   = t - grp * per;
  const int gn  = min(L_GROUP_N, tiles_n - grp * L_GROUP_N);
  tm            = r / gn;
  tn            = grp * L_GROUP_N + (r - tm * gn);
}

template <bool BF16, bool TMA_EPI>
__global__ void __launch_bounds__(L_THREADS, 1)
gemm_lp_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
               const __grid_constant__ CUtensorMap tmC, int m, int n, int k,
               float* __restrict__ C, int64_t ldc, const float* __restrict__ sA,
               const float* __restrict__ sB, int tiles_m, int tiles_n, int tpc, int* status) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* ringA = base;
  unsigned char* ringB = base + LSTAGES * LA_BYTES;
  unsigned char* stage = base + LSTAGES * LSTAGE_BYTES;  // TMA_EPI: epilogue staging
  uint64_t* full  = (uint64_t*)(stage + (TMA_EPI ? L_STG_TOTAL : 0));
  uint64_t* empty = full + LSTAGES;
  uint64_t* accf  = empty + LSTAGES;  // accumulator ready (MMA -> epilogue), both CTAs
  uint64_t* acce  = accf + 2;         // accumulator drained (epilogues -> MMA), CTA 0's
  uint64_t* drain = acce + 2;         // every issued MMA finished (abort path)
  __shared__ uint32_t     s_tmem;
  __shared__ volatile int s_abort;

  const int      warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();  // 0: issues the MMAs; 1: its peer
  const int      ntiles  = tiles_m * tiles_n;  // 256 x 256 tiles
  const int      t_begin = (blockIdx.x >> 1) * tpc;
  const int      t_end   = min(ntiles, t_begin + tpc);
  const int      KB      = (k + LBK - 1) / LBK;

  if(threadIdx.x == 0) {
    for(int s = 0; s < LSTAGES; ++s) {
      bar_init(&full[s], 1);
      bar_init(&empty[s], 1);
    }
    for(int b = 0; b < 2; ++b) {
      bar_init(&accf[b], 1);
      bar_init(&acce[b], 2 * L_EPI_WARPS);
    }
    bar_init(drain, 1);
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if(warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(
                     su32(&s_tmem))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  cluster_sync();  // both CTAs' barriers initialised before any cross-CTA signal
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;

  if(warp == 0) {
    // ---------------- TMA producer (both CTAs) ----------------
    if(lane == 0) {
      int s = 0, issued = 0;
      uint32_t ph = 0;
      for(int t = t_begin; t < t_end && !s_abort; ++t) {
        int tm, tn;
        tile_of(t, tiles_m, tiles_n, tm, tn);
        const int arow = tm * 2 * LBM + (int)rank * LBM;
        const int brow = tn * LBN + (int)rank * (LBN / 2);
        for(int kb = 0; kb < KB; ++kb) {
          if(!bar_wait(&empty[s], ph ^ 1, &s_abort)) {
            atomicCAS(status + ST_TIMEOUT, 0, 31);
            s_abort = 1;
            break;
          }
          if(rank == 0) bar_expect_tx(&full[s], 2 * LSTAGE_BYTES);  // both CTAs' bytes
          const uint32_t fb = mapa_shared(su32(&full[s]), 0);  // CTA 0's full[s]
          tma2d_pair(ringA + s * LA_BYTES, &tmA, fb, kb * LBK, arow);
          tma2d_pair(ringB + s * LB_BYTES, &tmB, fb, kb * LBK, brow);
          ++issued;
          if(++s == LSTAGES) {
            s = 0;
            ph ^= 1;
          }
        }
      }
      if(s_abort && rank == 0) {
        // Bounded drain: the last LSTAGES stages are the only ones whose
        // copies (this CTA's and the peer's) can still be in flight.
        for(int q = issued > LSTAGES ? issued - LSTAGES : 0; q < issued; ++q) {
          const unsigned long long t0 = globaltimer();
          while(!bar_try(&full[q % LSTAGES], (uint32_t)((q / LSTAGES) & 1)) &&
                globaltimer() - t0 < kWaitBudgetNs) {
          }
        }
      }
    }
    __syncwarp();
  } else if(warp == 1) {
    // ---------------- MMA issuer (CTA 0) ----------------
    if(lane == 0 && rank == 0) {
      // D = F32 (bits 4-5), A/B = BF16 (1) or F16 (0) (bits 7-12), K-major,
      // N/8 at bits 17-22, M/16 at bits 24-28; M = 256 across the pair.
      const uint32_t fmt   = BF16 ? 1u : 0u;
      const uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(LBN >> 3) << 17) |
                             ((uint32_t)((2 * LBM) >> 4) << 24);
      int s = 0;
      uint32_t ph = 0;
      int it = 0;
      for(int t = t_begin; t < t_end && !s_abort; ++t, ++it) {
        const int      buf = it & 1;
        const uint32_t d   = tmem + (uint32_t)(buf * LBN);
        if(!bar_wait(&acce[buf], (uint32_t)(((it >> 1) & 1) ^ 1), &s_abort)) {
          atomicCAS(status + ST_TIMEOUT, 0, 32);
          s_abort = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        bool ok = true;
        for(int kb = 0; kb < KB; ++kb) {
          if(!bar_wait(&full[s], ph, &s_abort)) {
            atomicCAS(status + ST_TIMEOUT, 0, 33);
            s_abort = 1;
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a0 = su32(ringA + s * LA_BYTES);
          const uint32_t b0 = su32(ringB + s * LB_BYTES);
#pragma unroll
          for(int kk = 0; kk < LBK / 16; ++kk)
            umma_f16_pair(d, umma_desc(a0 + kk * 32), umma_desc(b0 + kk * 32), idesc,
                          (kb | kk) != 0 ? 1u : 0u);
          umma_commit_pair(&empty[s], 0x3);  // both CTAs' slot s free once read
          if(++s == LSTAGES) {
            s = 0;
            ph ^= 1;
          }
        }
        if(!ok) break;
        umma_commit_pair(&accf[buf], 0x3);  // accumulator complete in both CTAs
      }
      if(s_abort) {
        // Bounded wait for every MMA issued before TMEM goes away.
        umma_commit_pair(drain, 0x1);
        const unsigned long long t0 = globaltimer();
        while(!bar_try(drain, 0) && globaltimer() - t0 < kWaitBudgetNs) {
        }
      }
    }
    __syncwarp();
  } else {
    // ---------------- epilogue (both CTAs) ----------------
    const int      ew   = warp - 2;              // 0..7
    const int      sub  = warp & 3;              // TMEM lane group this warp may read
    const int      half = ew >> 2;               // column half of the tile
    const uint32_t drained0 = mapa_shared(su32(acce), 0);  // CTA 0's acce[0]
    int it = 0, chunk = 0;
    for(int t = t_begin; t < t_end; ++t, ++it) {
      const int buf = it & 1;
      if(!bar_wait(&accf[buf], (uint32_t)((it >> 1) & 1), &s_abort)) {
        if(lane == 0) atomicCAS(status + ST_TIMEOUT, 0, 34);
        s_abort = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      int tm, tn;
      tile_of(t, tiles_m, tiles_n, tm, tn);
      const int  rtile = tm * 2 + (int)rank;  // this CTA's 128-row tile
      const int  row0  = rtile * LBM + sub * 32;
      const bool live  = rtile * LBM < m;     // the pair's last tile may hang off m
      const float scale = live ? sA[rtile] * sB[tn] : 0.f;
      if constexpr(TMA_EPI) {
        // Chunks of 16 columns: TMEM -> registers -> -scale * acc into this
        // warp's staging buffer (column-major, 32 rows x 16) -> TMA reduce-add
        // into C.  Two buffers per warp; a buffer is rewritten only after the
        // reduce issued from it two chunks ago has read it.
        unsigned char* mine = stage + ew * L_EPI_BUFS * L_STG_BYTES;
        for(int c0 = half * (LBN / 2); live && c0 < (half + 1) * (LBN / 2); c0 += L_EPI_COLS) {
          uint32_t r[L_EPI_COLS];
          const uint32_t taddr =
              tmem + ((uint32_t)(sub * 32) << 16) + (uint32_t)(buf * LBN + c0);
          tmem_ld_cols<L_EPI_COLS>(taddr, r);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          float* sbuf = reinterpret_cast<float*>(mine + (chunk % L_EPI_BUFS) * L_STG_BYTES);
          if(lane == 0) bulk_wait_read<L_EPI_BUFS - 1>();
          __syncwarp();
#pragma unroll
          for(int j = 0; j < L_EPI_COLS; ++j) sbuf[j * 32 + lane] = -scale * __uint_as_float(r[j]);
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          __syncwarp();
          if(lane == 0) {
            tma_reduce_add2d(&tmC, sbuf, row0, tn * LBN + c0);
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
          }
          ++chunk;
        }
      } else {
        const int row = row0 + lane;
        for(int c0 = half * (LBN / 2); live && c0 < (half + 1) * (LBN / 2); c0 += 32) {
          uint32_t r[32];
          const uint32_t taddr =
              tmem + ((uint32_t)(sub * 32) << 16) + (uint32_t)(buf * LBN + c0);
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,"
              "%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31},"
              " [%32];"
              : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
                "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
                "=r"(r[30]), "=r"(r[31])
              : "r"(taddr));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          if(row < m) {
            float cv[32];
            const int col0 = tn * LBN + c0;
#pragma unroll
            for(int j = 0; j < 32; ++j)
              cv[j] = (col0 + j < n) ? C[(size_t)row + (size_t)(col0 + j) * ldc] : 0.f;
#pragma unroll
            for(int j = 0; j < 32; ++j)
              if(col0 + j < n)
                C[(size_t)row + (size_t)(col0 + j) * ldc] = cv[j] - scale * __uint_as_float(r[j]);
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if(lane == 0) bar_arrive_cluster(drained0 + (uint32_t)(buf * sizeof(uint64_t)));
    }
    // Every reduce this warp issued has finished (its staging reads and its
    // writes) before the CTA's shared memory goes away.
    if(TMA_EPI && lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    __syncwarp();
  }

  if(threadIdx.x == 0 && s_abort) {
    // After a timeout the peer's copies into this CTA (and this CTA's copies
    // counted on the peer's barrier) are not tracked here: give anything
    // still in flight a bounded moment to land before the memory is released.
    const unsigned long long t0 = globaltimer();
    while(globaltimer() - t0 < 100000ull) {
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  cluster_sync();  // neither CTA leaves while the other may still touch its memory
  if(warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
  }
}

PFN_cuTensorMapEncodeTiled_v12000 g_enc = nullptr;

bool lp_encoder() {
  if(g_enc) return true;
  cudaDriverEntryPointQueryResult q;
  void*                           fn = nullptr;
  if(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
         cudaSuccess ||
     q != cudaDriverEntryPointSuccess || !fn) {
    cudaGetLastError();
    return false;
  }
  g_enc = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  return true;
}

}  // namespace

int gemm_lp_tile_m() { return LBM; }
int gemm_lp_tile_n() { return LBN; }

// A16: m x k, row-major with leading dimension lda (elements, k contiguous);
// B16: n x k likewise.  sA: tiles_m scale factors, sB: tiles_n.
cudaError_t launch_gemm_lp(bool bf16, int m, int n, int k, const void* A16, int64_t lda,
                           const void* B16, int64_t ldb, const float* sA, const float* sB,
                           float* C, int64_t ldc, int* status, cudaStream_t stream) {
  if(m <= 0 || n <= 0 || k <= 0) return cudaSuccess;
  if(!lp_encoder()) return cudaErrorNotSupported;
  if((uintptr_t)A16 % 16 || (uintptr_t)B16 % 16 || (lda * 2) % 16 || (ldb * 2) % 16)
    return cudaErrorInvalidValue;
  const CUtensorMapDataType dt =
      bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
  CUtensorMap mA, mB;
  {
    cuuint64_t dims[2]    = {(cuuint64_t)k, (cuuint64_t)m};
    cuuint64_t strides[1] = {(cuuint64_t)lda * 2};
    cuuint32_t box[2]     = {LBK, LBM};
    cuuint32_t es[2]      = {1, 1};
    if(g_enc(&mA, dt, 2, (void*)A16, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return cudaErrorInvalidValue;
  }
  {
    cuuint64_t dims[2]    = {(cuuint64_t)k, (cuuint64_t)n};
    cuuint64_t strides[1] = {(cuuint64_t)ldb * 2};
    cuuint32_t box[2]     = {LBK, LBN / 2};
    cuuint32_t es[2]      = {1, 1};
    if(g_enc(&mB, dt, 2, (void*)B16, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return cudaErrorInvalidValue;
  }
  // C for the reduce-add epilogue: FP32, column-major, boxes of 32 rows x 16
  // columns (one epilogue warp's chunk).  Needs a 16-byte aligned base and a
  // leading dimension in whole 16-byte units; otherwise the plain epilogue.
  CUtensorMap mC;
  memset(&mC, 0, sizeof mC);
  bool tma_epi = (uintptr_t)C % 16 == 0 && (ldc * 4) % 16 == 0;
  if(tma_epi) {
    cuuint64_t dims[2]    = {(cuuint64_t)m, (cuuint64_t)n};
    cuuint64_t strides[1] = {(cuuint64_t)ldc * 4};
    cuuint32_t box[2]     = {32, L_EPI_COLS};
    cuuint32_t es[2]      = {1, 1};
    tma_epi = g_enc(&mC, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)C, dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  }
  static bool attr[4] = {false, false, false, false};
  const int   kind    = (bf16 ? 1 : 0) + (tma_epi ? 2 : 0);
  cudaError_t e       = cudaSuccess;
  if(!attr[kind]) {
    switch(kind) {
      case 0: e = cudaFuncSetAttribute(gemm_lp_kernel<false, false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, L_SMEM); break;
      case 1: e = cudaFuncSetAttribute(gemm_lp_kernel<true, false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, L_SMEM); break;
      case 2: e = cudaFuncSetAttribute(gemm_lp_kernel<false, true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, L_SMEM_TMA);
              break;
      default: e = cudaFuncSetAttribute(gemm_lp_kernel<true, true>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, L_SMEM_TMA);
    }
    if(e != cudaSuccess) return e;
    attr[kind] = true;
  }
  const int tiles_m = (m + 2 * LBM - 1) / (2 * LBM), tiles_n = (n + LBN - 1) / LBN;
  const long long ntiles = (long long)tiles_m * tiles_n;
  // Up to 6 tiles per CTA pair (pairs retire regularly, so the panel stream
  // running beside this kernel gets SMs), balanced so the pair count fills
  // whole waves of one pair per two SMs.  In the FP16x3 solve at N = 131072
  // the LU took 2% less time with 6 than with 4 or 8, and 1.5% more with 32
  // than with 8 (pairs that keep their SMs longer hold up the panel).
  static int sms = 0;
  if(sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if(sms < 2) sms = 2;
  }
  constexpr int tmax  = 6;  // tiles per pair at most
  const int     pairs = sms / 2;
  const long long waves = (ntiles + (long long)pairs * tmax - 1) / ((long long)pairs * tmax);
  const int tpc = (int)((ntiles + (long long)pairs * waves - 1) / ((long long)pairs * waves));
  const long long npairs = (ntiles + tpc - 1) / tpc;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim          = dim3((unsigned)(2 * npairs));
  cfg.blockDim         = dim3(L_THREADS);
  cfg.dynamicSmemBytes = tma_epi ? L_SMEM_TMA : L_SMEM;
  cfg.stream           = stream;
  cudaLaunchAttribute at[1];
  at[0].id               = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 2;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs              = at;
  cfg.numAttrs           = 1;
  switch(kind) {
    case 0:
      e = cudaLaunchKernelEx(&cfg, gemm_lp_kernel<false, false>, mA, mB, mC, m, n, k, C, ldc, sA,
                             sB, tiles_m, tiles_n, tpc, status);
      break;
    case 1:
      e = cudaLaunchKernelEx(&cfg, gemm_lp_kernel<true, false>, mA, mB, mC, m, n, k, C, ldc, sA,
                             sB, tiles_m, tiles_n, tpc, status);
      break;
    case 2:
      e = cudaLaunchKernelEx(&cfg, gemm_lp_kernel<false, true>, mA, mB, mC, m, n, k, C, ldc, sA,
                             sB, tiles_m, tiles_n, tpc, status);
      break;
    default:
      e = cudaLaunchKernelEx(&cfg, gemm_lp_kernel<true, true>, mA, mB, mC, m, n, k, C, ldc, sA,
                             sB, tiles_m, tiles_n, tpc, status);
  }
  if(e != cudaSuccess) return e;
  return cudaGetLastError();
}

}  // namespace hplb
