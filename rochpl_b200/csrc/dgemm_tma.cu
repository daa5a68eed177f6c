// Trailing-update DGEMM, TMA-fed and warp-specialised:  C -= A B  (FP64, DMMA).
//
// The hot kernel of the solve (rocblas_dgemm of src/pgesv/HPL_pdupdateTT.cpp:
// 131-163).  The Tensor Memory Accelerator streams A and B k-slices into a
// 6-deep shared memory ring with cp.async.bulk.tensor (each CTA loads its own tiles), signalling "full"
// mbarriers through the transaction count; eight warps wait on them and run
// m16n8k8 f64 MMAs out of the swizzled tiles.  There is no dedicated producer
// warp (a ninth warp would cap every warp at 168 registers): the warp that is
// last to finish with a slot, counted by a shared-memory atomic, refills it
// with the slice STAGES ahead, so no warp ever blocks to produce.  No
// __syncthreads in the main loop.
//
// Layouts (doubles):
//   A slice: [8 slabs][16 k][16 m], 128-byte rows, 128B TMA swizzle.  A is
//            M-contiguous (column-major L21), so A is described to TMA as a 3-D
//            tensor {16 rows, k, row-slab}: every A copy starts at x = 0.
//   B slice: [128 n][16 k], 128-byte rows, 128B TMA swizzle (B = U12 is
//            k-contiguous per column).
// A 64-bit shared load is served per half warp (lanes g = 0..3 or 4..7 with
// t = 0..3), so each half warp must hit 16 distinct 8-byte slots of a 128-byte
// row.  The reduction index can be relabelled freely as long as A and B agree:
// MMA k-step 0 takes lane t's k from {0,3,12,15} (a0/b0) and {2,1,14,13}
// (a2/b1) of the 16-deep slice, step 1 from {4,7,8,11} and {6,5,10,9}.  Those
// sets have distinct (bit0, bit3) -- what the B swizzle needs -- and distinct
// (bit1, bit2) -- what the A swizzle needs -- so both fragments load without
// bank conflicts.
// A CTA computes tpc consecutive 128 x 128 tiles of a grouped order (4 column
// tiles per A row-tile), so an A tile is fetched from HBM once and re-read
// from L2 three times.  Either CTAs retire every few tiles, so that the
// high-priority panel stream can get onto SMs as they free up, or (a cap on
// the grid) a fixed number of CTAs each walks a long run of tiles and the
// SMs beyond the cap stay free for the panel stream for the whole launch.
//
// Every mbarrier wait is bounded: a wait only expires when a copy never lands;
// the CTA then records the site in the status word and exits.
#include <cstdlib>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.cuh"
#include "internal.h"

namespace hplb {

namespace {

constexpr int BM = 128, BN = 128, BK = 16, STAGES = 6;
constexpr int NCONS   = 8;               // consumer warps (one of them refills each slot)
constexpr int THREADS = NCONS * 32;
constexpr int GROUP_N = 4;               // column tiles per group
constexpr int A_BYTES = BM * BK * 8;     // 16 KB
constexpr int B_BYTES = BN * BK * 8;     // 16 KB
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int SMEM_BYTES  = STAGES * STAGE_BYTES + 1024 /*align*/ + 128 /*barriers*/;

HPLB_DEV uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

HPLB_DEV void mbar_init(uint64_t* b, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
HPLB_DEV void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)),
               "r"(bytes)
               : "memory");
}
HPLB_DEV bool mbar_try_wait(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for phase `parity` of barrier b.  False on timeout or when
// another warp of the CTA has already given up (*abort != 0).
HPLB_DEV bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort) {
  if(mbar_try_wait(b, parity)) return true;
  const unsigned long long t0 = globaltimer();
  while(!mbar_try_wait(b, parity)) {
    if(*abort) return false;
    if(globaltimer() - t0 > kWaitBudgetNs) return false;
  }
  return true;
}

HPLB_DEV void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                          int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
HPLB_DEV void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
      : "memory");
}

HPLB_DEV void dmma(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// Grouped tile order: GROUP_N column tiles share each row tile.
HPLB_DEV void tile_coords(int t, int tiles_m, int tiles_n, int& tm, int& tn) {
  const int per = tiles_m * GROUP_N;
  const int grp = t / per;
  const int r   = t - grp * per;
  const int gn  = min(GROUP_N, tiles_n - grp * GROUP_N);
  tm            = r / gn;
  tn            = grp * GROUP_N + (r - tm * gn);
}

// Element offset (in doubles) of A(k, m-in-slab) in a swizzled 16-row slab.
HPLB_DEV int a_off(int slab, int k, int m16) {
  const int L = ((slab * BK + k) * 16 + m16) * 8;  // logical byte offset
  return (L ^ (((L >> 7) & 7) << 4)) >> 3;
}
// Element offset of B(k, n) in the [n][16 k] slice with 128B swizzle.
HPLB_DEV int b_off(int n, int k) {
  const int L = (n * BK + k) * 8;
  return (L ^ (((L >> 7) & 7) << 4)) >> 3;
}

// Issue the copies of k-slice q (tile t_begin + q / KT, k-slice q % KT) into
// ring slot q % STAGES.
HPLB_DEV void issue_slice(int q, int t_begin, int KT, int tiles_m, int tiles_n,
                          const CUtensorMap* tmA, const CUtensorMap* tmB, unsigned char* sA,
                          unsigned char* sB, uint64_t* full) {
  const int s = q % STAGES;
  int       tm, tn;
  tile_coords(t_begin + q / KT, tiles_m, tiles_n, tm, tn);
  const int kt = q % KT;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mbar_expect_tx(&full[s], STAGE_BYTES);
  tma_load_3d(sA + s * A_BYTES, tmA, &full[s], 0, kt * BK, tm * (BM / 16));
  tma_load_2d(sB + s * B_BYTES, tmB, &full[s], kt * BK, tn * BN);
}

template <bool ACCUM>
__global__ void __launch_bounds__(THREADS, 1)
dgemm_tma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                 int m, int n, int k, double* __restrict__ C, int64_t ldc, int tiles_m,
                 int tiles_n, int tpc, int* status) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* sA   = base;                      // [STAGES][A_BYTES]
  unsigned char* sB   = base + STAGES * A_BYTES;   // [STAGES][B_BYTES]
  uint64_t*      full = (uint64_t*)(base + STAGES * STAGE_BYTES);
  __shared__ int          s_done[STAGES];  // warps finished with the slot's slice
  __shared__ volatile int s_abort;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntiles  = tiles_m * tiles_n;
  const int t_begin = blockIdx.x * tpc;
  const int t_end   = min(ntiles, t_begin + tpc);
  const int KT      = (k + BK - 1) / BK;
  const int nslices = (t_end - t_begin) * KT;

  if(threadIdx.x == 0) {
    for(int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      s_done[s] = 0;
    }
    s_abort = 0;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    for(int q = 0; q < STAGES && q < nslices; ++q)
      issue_slice(q, t_begin, KT, tiles_m, tiles_n, &tmA, &tmB, sA, sB, full);
  }
  __syncthreads();

  const int g = lane >> 2, t4 = lane & 3;
  const int wm = (warp & 1) * 64;   // 2 warps along M
  const int wn = (warp >> 1) * 32;  // 4 warps along N
  // Relabelled reduction index (see the layout note at the top): this lane's
  // k for a0/b0 and for a2/b1, in MMA k-steps 0 and 1.
  int kk[2][2];
  kk[0][0] = (t4 & 1) * 3 + (t4 >> 1) * 12;         // {0, 3, 12, 15}
  kk[0][1] = ((t4 & 1) ? 1 : 2) + (t4 >> 1) * 12;     // {2, 1, 14, 13}
  kk[1][0] = 4 + (t4 & 1) * 3 + (t4 >> 1) * 4;      // {4, 7, 8, 11}
  kk[1][1] = ((t4 & 1) ? 5 : 6) + (t4 >> 1) * 4;      // {6, 5, 10, 9}
  // Swizzled element offsets of this lane's fragments, fixed for the whole
  // kernel: A rows g / g+8 of the warp's first slab, B column g of its first
  // n-tile.  Slab i adds i*256 and n-tile j adds j*128 doubles (immediates).
  int oA[2][2][2], oB[2][2];
#pragma unroll
  for(int st = 0; st < 2; ++st)
#pragma unroll
    for(int h = 0; h < 2; ++h) {
      oA[st][h][0] = a_off(wm >> 4, kk[st][h], g);
      oA[st][h][1] = a_off(wm >> 4, kk[st][h], g + 8);
      oB[st][h]    = b_off(wn + g, kk[st][h]);
    }
  int       q  = 0;                 // running k-slice index
  int       slot = 0;               // q % STAGES
  uint32_t  phase = 0;              // (q / STAGES) & 1
  for(int t = t_begin; t < t_end; ++t) {
    int tm, tn;
    tile_coords(t, tiles_m, tiles_n, tm, tn);
    const int m0 = tm * BM + wm, n0 = tn * BN + wn;
    // Pull this warp's 64 x 32 block of C into L2 while the tile is computed.
    {
      const int col = n0 + lane;
      if(ACCUM && col < n)
        for(int r = m0; r < min(m0 + 64, m); r += 16)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(C + (size_t)r + (size_t)col * ldc));
    }
    double acc[4][4][4];
#pragma unroll
    for(int i = 0; i < 4; ++i)
#pragma unroll
      for(int j = 0; j < 4; ++j)
#pragma unroll
        for(int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;

    for(int kt = 0; kt < KT; ++kt, ++q) {
      if(!mbar_wait(&full[slot], phase, &s_abort)) {
        if(lane == 0) atomicCAS(status + ST_TIMEOUT, 0, 22);
        s_abort = 1;
        return;
      }
      const double* a = (const double*)(sA + slot * A_BYTES);
      const double* b = (const double*)(sB + slot * B_BYTES);
#pragma unroll
      for(int st = 0; st < 2; ++st) {
        double af[4][4], bf[4][2];
#pragma unroll
        for(int i = 0; i < 4; ++i) {
          af[i][0] = a[oA[st][0][0] + i * 256];
          af[i][1] = a[oA[st][0][1] + i * 256];
          af[i][2] = a[oA[st][1][0] + i * 256];
          af[i][3] = a[oA[st][1][1] + i * 256];
        }
#pragma unroll
        for(int j = 0; j < 4; ++j) {
          bf[j][0] = b[oB[st][0] + j * 128];
          bf[j][1] = b[oB[st][1] + j * 128];
        }
#pragma unroll
        for(int i = 0; i < 4; ++i)
#pragma unroll
          for(int j = 0; j < 4; ++j) dmma(acc[i][j], af[i], bf[j]);
      }
      // The last warp to finish with the slot refills it with slice q + STAGES.
      __syncwarp();
      if(lane == 0) {
        if(atomicAdd(&s_done[slot], 1) == NCONS - 1) {
          s_done[slot] = 0;
          if(q + STAGES < nslices)
            issue_slice(q + STAGES, t_begin, KT, tiles_m, tiles_n, &tmA, &tmB, sA, sB, full);
        }
      }
      if(++slot == STAGES) {
        slot = 0;
        phase ^= 1u;
      }
    }

    // Epilogue: C -= acc, or C = acc in the store form (C rows/cols outside
    // m x n are never touched).  Two
    // halves; all loads of a half are issued before its stores, so they are
    // in flight together instead of one dependent round trip per element.
#pragma unroll
    for(int h = 0; h < 2; ++h) {
      double cv[2][4][4];
#pragma unroll
      for(int i = 0; i < 2; ++i)
#pragma unroll
        for(int j = 0; j < 4; ++j)
#pragma unroll
          for(int r = 0; r < 4; ++r) {
            const int row = m0 + (2 * h + i) * 16 + g + (r >> 1) * 8;
            const int col = n0 + j * 8 + 2 * t4 + (r & 1);
            cv[i][j][r] =
                (ACCUM && row < m && col < n) ? C[(size_t)row + (size_t)col * ldc] : 0.0;
          }
#pragma unroll
      for(int i = 0; i < 2; ++i)
#pragma unroll
        for(int j = 0; j < 4; ++j)
#pragma unroll
          for(int r = 0; r < 4; ++r) {
            const int row = m0 + (2 * h + i) * 16 + g + (r >> 1) * 8;
            const int col = n0 + j * 8 + 2 * t4 + (r & 1);
            if(row < m && col < n)
              C[(size_t)row + (size_t)col * ldc] =
                  ACCUM ? cv[i][j][r] - acc[2 * h + i][j][r] : acc[2 * h + i][j][r];
          }
    }
  }
  // Every issued slice was waited for above, so no copy is still in flight.
}

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

bool get_encoder() {
  if(g_encode) return true;
  cudaDriverEntryPointQueryResult q;
  void*                           fn = nullptr;
  if(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
         cudaSuccess ||
     q != cudaDriverEntryPointSuccess || !fn) {
    cudaGetLastError();
    return false;
  }
  g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  return true;
}

// Tiles per CTA.  Four (a whole group: the A tile fetched once and re-read
// from L2 by the group's other column tiles, one pipeline across them) for a
// large product, at least 256 tiles per SM -- the trailing update while it is
// the critical path -- and eight (two groups) from 1024 tiles per SM, where the
// panel beside it has ample slack: fewer pipeline fills and CTA starts
// (N = 131072 solve: DGEMM 31.89 -> 32.13 TFLOP/s, 48.02 -> 47.66 s).  Below
// 256, one: the panel's own updates spread over the SMs, and the trailing
// update's CTAs retire every tile, so the high-priority panel kernels (the
// critical path once the trailing matrix is small) wait less for SMs.
// Measured at N = 16384 (getrf, NB = 512, B200): 251 ms with four, 208 ms
// with one, identical bits.
int tiles_per_cta(long long ntiles) {
  static const int sms = [] {
    int dev = 0, n = 148;
    if(cudaGetDevice(&dev) != cudaSuccess ||
       cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
      cudaGetLastError();
      n = 148;
    }
    return n;
  }();
  return ntiles >= 1024LL * sms ? 8 : (ntiles >= 256LL * sms ? 4 : 1);
}

cudaError_t launch_tpc(const CUtensorMap& mA, const CUtensorMap& mB, int m, int n, int k,
                       double* C, int64_t ldc, int tiles_m, int tiles_n, int tpc, bool accumulate,
                       int* status, cudaStream_t stream) {
  static bool attr = false;
  if(!attr) {
    cudaError_t e = cudaFuncSetAttribute(dgemm_tma_kernel<true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    if(e == cudaSuccess)
      e = cudaFuncSetAttribute(dgemm_tma_kernel<false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    if(e != cudaSuccess) return e;
    attr = true;
  }
  const long long ntiles = (long long)tiles_m * tiles_n;
  const long long grid   = (ntiles + tpc - 1) / tpc;
  if(grid > 0x7fffffff) return cudaErrorInvalidValue;
  if(accumulate)
    dgemm_tma_kernel<true><<<(unsigned)grid, THREADS, SMEM_BYTES, stream>>>(
        mA, mB, m, n, k, C, ldc, tiles_m, tiles_n, tpc, status);
  else
    dgemm_tma_kernel<false><<<(unsigned)grid, THREADS, SMEM_BYTES, stream>>>(
        mA, mB, m, n, k, C, ldc, tiles_m, tiles_n, tpc, status);
  return cudaGetLastError();
}

}  // namespace

bool dgemm_tma_eligible(int m, int n, int k, const double* A, int64_t lda, const double* B,
                        int64_t ldb) {
  if(m <= 0 || n <= 0 || k <= 0) return false;
  if((uintptr_t)A % 16 || (uintptr_t)B % 16) return false;
  if(lda % 2 || ldb % 2) return false;
  // The last 16-row slab of A is read whole: it must stay inside the column.
  if(lda < ((int64_t)m + 15) / 16 * 16) return false;
  return get_encoder();
}

cudaError_t launch_dgemm_tma(int m, int n, int k, const double* A, int64_t lda, const double* B,
                             int64_t ldb, double* C, int64_t ldc, int* status, bool accumulate,
                             cudaStream_t stream, int max_ctas) {
  CUtensorMap mA, mB;
  {
    cuuint64_t dims[3]    = {16, (cuuint64_t)k, (cuuint64_t)((m + 15) / 16)};
    cuuint64_t strides[2] = {(cuuint64_t)lda * 8, 128};
    cuuint32_t box[3]     = {16, BK, BM / 16};
    cuuint32_t es[3]      = {1, 1, 1};
    CUresult r = g_encode(&mA, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void*)A, dims, strides, box,
                          es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if(r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  }
  {
    cuuint64_t dims[2]    = {(cuuint64_t)k, (cuuint64_t)n};
    cuuint64_t strides[1] = {(cuuint64_t)ldb * 8};
    cuuint32_t box[2]     = {BK, BN};
    cuuint32_t es[2]      = {1, 1};
    CUresult r = g_encode(&mB, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, (void*)B, dims, strides, box,
                          es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if(r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  }
  const int       tiles_m = (m + BM - 1) / BM, tiles_n = (n + BN - 1) / BN;
  const long long ntiles  = (long long)tiles_m * tiles_n;
  long long       tpc     = tiles_per_cta(ntiles);
  if(max_ctas > 0 && (ntiles + tpc - 1) / tpc > max_ctas) tpc = (ntiles + max_ctas - 1) / max_ctas;
  if(tpc > 0x7fffffff) return cudaErrorInvalidValue;
  return launch_tpc(mA, mB, m, n, k, C, ldc, tiles_m, tiles_n, (int)tpc, accumulate, status,
                    stream);
}

}  // namespace hplb
