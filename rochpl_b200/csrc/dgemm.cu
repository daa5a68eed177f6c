// Trailing-update DGEMM  C(m x n) -= A(m x k) B(k x n), column-major FP64,
// on the FP64 tensor-core path (DMMA, mma.sync ... .f64).
//
// Replaces the rocblas_dgemm call of src/pgesv/HPL_pdupdateTT.cpp:131-163
// (and the panel-local one of src/pfact/HPL_pdrpanrlT.cpp:140-155).  sm_100a's
// tcgen05 MMA has no f64 kind, so FP64 tensor work is the warp-level DMMA
// m16n8k8 shape; operands are staged through a multi-stage cp.async ring in
// padded shared memory so every fragment load is bank-conflict free.
//
// Tile: 128 x 128 per CTA, k-slices of 16, 8 warps each owning 64 x 32.  In HPL
// k = NB (512 at the benchmark size), so each CTA reads its C tile once and
// writes it once: 256 KB of C traffic per 16.8 MFLOP.
#include <cstdlib>
#include <cstring>

#include "common.cuh"
#include "internal.h"

namespace hplb {

namespace {

HPLB_DEV void cp_async8(void* smem, const void* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int      n = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n)
               : "memory");
}
HPLB_DEV void cp_async16(void* smem, const void* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int      n = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n)
               : "memory");
}
HPLB_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
HPLB_DEV void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// D = A B + D, m16n8k8, f64.  Fragment layout (g = lane / 4, t = lane % 4):
//   A 16x8: a0 (g, t) a1 (g+8, t) a2 (g, t+4) a3 (g+8, t+4)
//   B  8x8: b0 (t, g) b1 (t+4, g)
//   C 16x8: c0 (g, 2t) c1 (g, 2t+1) c2 (g+8, 2t) c3 (g+8, 2t+1)
HPLB_DEV void dmma_16x8x8(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

constexpr int BM = 128, BN = 128, BK = 16, STAGES = 4;
constexpr int WM = 64, WN = 32;
constexpr int NWARP_M = BM / WM, NWARP_N = BN / WN;
constexpr int NTHREADS = NWARP_M * NWARP_N * 32;  // 256
constexpr int LDSA = BM + 4;  // smem row pitch of an A k-slice (doubles), = 4 mod 16
constexpr int LDSB = BK + 4;  // smem pitch of a B column (doubles), = 4 mod 16
constexpr int A_STAGE = BK * LDSA;
constexpr int B_STAGE = BN * LDSB;
constexpr int SMEM_BYTES = STAGES * (A_STAGE + B_STAGE) * 8;
constexpr int MT = WM / 16, NT = WN / 8;

// VEC: 16-byte cp.async (needs 16-byte aligned pointers and even leading
// dimensions and row offsets; the host checks).
template <bool VEC, bool ACCUM>
__global__ void __launch_bounds__(NTHREADS, 1)
dgemm_sub_kernel(int m, int n, int k, const double* __restrict__ A, int64_t lda,
                 const double* __restrict__ B, int64_t ldb, double* __restrict__ C,
                 int64_t ldc) {
  extern __shared__ __align__(16) double smem[];
  double* As = smem;
  double* Bs = smem + STAGES * A_STAGE;

  const int tid  = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp % NWARP_M) * WM;
  const int wn = (warp / NWARP_M) * WN;
  const int m0 = blockIdx.x * BM;
  const int n0 = blockIdx.y * BN;
  const int KT = (k + BK - 1) / BK;

  auto load_stage = [&](int kt, int stage) {
    const int k0 = kt * BK;
    double* as = As + stage * A_STAGE;
    double* bs = Bs + stage * B_STAGE;
    if(VEC) {
      // A: BK columns x BM rows, 2 doubles per copy -> 1024 copies, 4 per thread.
#pragma unroll
      for(int i = 0; i < (BM * BK / 2) / NTHREADS; ++i) {
        const int idx = tid + i * NTHREADS;
        const int r = (idx % (BM / 2)) * 2, c = idx / (BM / 2);
        const int gr = m0 + r, gc = k0 + c;
        const bool p = (gr < m) && (gc < k);
        const double* src = p ? A + (size_t)gr + (size_t)gc * lda : A;
        cp_async16(as + c * LDSA + r, src, p);
      }
      // B: BN columns x BK rows.
#pragma unroll
      for(int i = 0; i < (BN * BK / 2) / NTHREADS; ++i) {
        const int idx = tid + i * NTHREADS;
        const int kk = (idx % (BK / 2)) * 2, nn = idx / (BK / 2);
        const int gk = k0 + kk, gn = n0 + nn;
        const bool p = (gk < k) && (gn < n);
        const double* src = p ? B + (size_t)gk + (size_t)gn * ldb : B;
        cp_async16(bs + nn * LDSB + kk, src, p);
      }
    } else {
#pragma unroll
      for(int i = 0; i < (BM * BK) / NTHREADS; ++i) {
        const int idx = tid + i * NTHREADS;
        const int r = idx % BM, c = idx / BM;
        const int gr = m0 + r, gc = k0 + c;
        const bool p = (gr < m) && (gc < k);
        const double* src = p ? A + (size_t)gr + (size_t)gc * lda : A;
        cp_async8(as + c * LDSA + r, src, p);
      }
#pragma unroll
      for(int i = 0; i < (BN * BK) / NTHREADS; ++i) {
        const int idx = tid + i * NTHREADS;
        const int kk = idx % BK, nn = idx / BK;
        const int gk = k0 + kk, gn = n0 + nn;
        const bool p = (gk < k) && (gn < n);
        const double* src = p ? B + (size_t)gk + (size_t)gn * ldb : B;
        cp_async8(bs + nn * LDSB + kk, src, p);
      }
    }
  };

  double acc[MT][NT][4];
#pragma unroll
  for(int i = 0; i < MT; ++i)
#pragma unroll
    for(int j = 0; j < NT; ++j)
#pragma unroll
      for(int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;

#pragma unroll
  for(int s = 0; s < STAGES - 1; ++s) {
    if(s < KT) load_stage(s, s);
    cp_async_commit();
  }

  for(int kt = 0; kt < KT; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    {
      const int nk = kt + STAGES - 1;
      if(nk < KT) load_stage(nk, nk % STAGES);
      cp_async_commit();
    }
    const double* as = As + (kt % STAGES) * A_STAGE;
    const double* bs = Bs + (kt % STAGES) * B_STAGE;
#pragma unroll
    for(int kk = 0; kk < BK; kk += 8) {
      double af[MT][4], bf[NT][2];
#pragma unroll
      for(int i = 0; i < MT; ++i) {
        const double* p = as + (kk + t) * LDSA + wm + i * 16 + g;
        af[i][0] = p[0];
        af[i][1] = p[8];
        af[i][2] = p[4 * LDSA];
        af[i][3] = p[4 * LDSA + 8];
      }
#pragma unroll
      for(int j = 0; j < NT; ++j) {
        const double* p = bs + (wn + j * 8 + g) * LDSB + kk + t;
        bf[j][0] = p[0];
        bf[j][1] = p[4];
      }
#pragma unroll
      for(int i = 0; i < MT; ++i)
#pragma unroll
        for(int j = 0; j < NT; ++j) dmma_16x8x8(acc[i][j], af[i], bf[j]);
    }
  }
  cp_async_wait<0>();

  // Epilogue: C -= acc, or C = acc in the store form.
#pragma unroll
  for(int i = 0; i < MT; ++i)
#pragma unroll
    for(int j = 0; j < NT; ++j) {
      const int r = m0 + wm + i * 16 + g;
      const int c = n0 + wn + j * 8 + 2 * t;
#pragma unroll
      for(int q = 0; q < 4; ++q) {
        const int rr = r + (q >> 1) * 8;
        const int cc = c + (q & 1);
        if(rr < m && cc < n) {
          double* p = C + (size_t)rr + (size_t)cc * ldc;
          *p = ACCUM ? *p - acc[i][j][q] : acc[i][j][q];
        }
      }
    }
}

}  // namespace

static cudaError_t launch_dgemm_any(int m, int n, int k, const double* A, int64_t lda,
                                    const double* B, int64_t ldb, double* C, int64_t ldc,
                                    int* status, bool accumulate, cudaStream_t stream,
                                    int max_ctas = 0) {
  if(m <= 0 || n <= 0) return cudaSuccess;
  if(k > 0 && status && dgemm_tma_eligible(m, n, k, A, lda, B, ldb)) {
    cudaError_t e = launch_dgemm_tma(m, n, k, A, lda, B, ldb, C, ldc, status, accumulate, stream,
                                     max_ctas);
    if(e == cudaSuccess) return e;
    cudaGetLastError();  // fall back to the cp.async kernel
  }
  return launch_dgemm_cpasync(m, n, k, A, lda, B, ldb, C, ldc, accumulate, stream);
}

cudaError_t launch_dgemm_sub(int m, int n, int k, const double* A, int64_t lda,
                             const double* B, int64_t ldb, double* C, int64_t ldc,
                             int* status, cudaStream_t stream, int max_ctas) {
  if(k <= 0) return cudaSuccess;
  return launch_dgemm_any(m, n, k, A, lda, B, ldb, C, ldc, status, true, stream, max_ctas);
}

cudaError_t launch_dgemm_set(int m, int n, int k, const double* A, int64_t lda,
                             const double* B, int64_t ldb, double* C, int64_t ldc,
                             int* status, cudaStream_t stream) {
  return launch_dgemm_any(m, n, k, A, lda, B, ldb, C, ldc, status, false, stream);
}

template <bool VEC, bool ACCUM>
static cudaError_t launch_cpasync_t(dim3 grid, int m, int n, int k, const double* A,
                                    int64_t lda, const double* B, int64_t ldb, double* C,
                                    int64_t ldc, cudaStream_t stream) {
  static bool attr = false;
  if(!attr) {
    cudaError_t e = cudaFuncSetAttribute(dgemm_sub_kernel<VEC, ACCUM>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    if(e != cudaSuccess) return e;
    attr = true;
  }
  dgemm_sub_kernel<VEC, ACCUM><<<grid, NTHREADS, SMEM_BYTES, stream>>>(m, n, k, A, lda, B, ldb,
                                                                       C, ldc);
  return cudaGetLastError();
}

cudaError_t launch_dgemm_cpasync(int m, int n, int k, const double* A, int64_t lda,
                                 const double* B, int64_t ldb, double* C, int64_t ldc,
                                 bool accumulate, cudaStream_t stream) {
  if(m <= 0 || n <= 0) return cudaSuccess;
  // Paired copies never straddle the logical edge: m and k must be even too.
  const bool vec = ((uintptr_t)A % 16 == 0) && ((uintptr_t)B % 16 == 0) && (lda % 2 == 0) &&
                   (ldb % 2 == 0) && (m % 2 == 0) && (k % 2 == 0);
  dim3 grid((m + BM - 1) / BM, (n + BN - 1) / BN);
  if(grid.y > 65535) return cudaErrorInvalidValue;
  if(vec)
    return accumulate ? launch_cpasync_t<true, true>(grid, m, n, k, A, lda, B, ldb, C, ldc, stream)
                      : launch_cpasync_t<true, false>(grid, m, n, k, A, lda, B, ldb, C, ldc, stream);
  return accumulate ? launch_cpasync_t<false, true>(grid, m, n, k, A, lda, B, ldb, C, ldc, stream)
                    : launch_cpasync_t<false, false>(grid, m, n, k, A, lda, B, ldb, C, ldc, stream);
}

}  // namespace hplb
