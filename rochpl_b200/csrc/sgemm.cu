// FP32 GEMM for the FP32 panel of the mixed-precision solve:
//   C -= A B  (accumulate) or  C = A B  (store),  all column-major FP32.
// The panel recursion's updates and U12 = L11^-1 W run in FP32 (the mixed
// form keeps the panel in FP32); only the trailing update goes to the 16-bit
// tensor cores.  128 x 128 tiles, 256 threads each owning an 8 x 8 block
// (rows ty*4 + {0..3, 64..67}, columns tx*4 + {0..3, 64..67}), k-slices of 8
// staged through double-buffered shared memory.
#include "common.cuh"
#include "internal.h"

namespace hplb {

namespace {

constexpr int SBM = 128, SBN = 128, SBK = 8, SPAD = 4;

template <bool ACCUM>
__global__ void __launch_bounds__(256)
sgemm_kernel(int m, int n, int k, const float* __restrict__ A, int64_t lda,
             const float* __restrict__ B, int64_t ldb, float* __restrict__ C, int64_t ldc) {
  __shared__ __align__(16) float As[2][SBK][SBM + SPAD];
  __shared__ __align__(16) float Bs[2][SBK][SBN + SPAD];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.x * SBM, n0 = blockIdx.y * SBN;

  float acc[8][8];
#pragma unroll
  for(int i = 0; i < 8; ++i)
#pragma unroll
    for(int j = 0; j < 8; ++j) acc[i][j] = 0.f;

  float ra[4], rb[4];
  auto fetch = [&](int k0) {
#pragma unroll
    for(int q = 0; q < 4; ++q) {
      const int idx = tid + q * 256;
      const int r = idx & (SBM - 1), c = idx >> 7;  // A: 128 rows x 8 k
      const int gr = m0 + r, gc = k0 + c;
      ra[q] = (gr < m && gc < k) ? A[(size_t)gr + (size_t)gc * lda] : 0.f;
      const int kk = idx & (SBK - 1), nn = idx >> 3;  // B: 8 k x 128 columns
      const int gk = k0 + kk, gn = n0 + nn;
      rb[q] = (gk < k && gn < n) ? B[(size_t)gk + (size_t)gn * ldb] : 0.f;
    }
  };
  auto stash = [&](int buf) {
#pragma unroll
    for(int q = 0; q < 4; ++q) {
      const int idx = tid + q * 256;
      As[buf][idx >> 7][idx & (SBM - 1)] = ra[q];
      Bs[buf][idx & (SBK - 1)][idx >> 3] = rb[q];
    }
  };

  const int KT = (k + SBK - 1) / SBK;
  if(KT > 0) {
    fetch(0);
    stash(0);
  }
  __syncthreads();
  for(int kt = 0; kt < KT; ++kt) {
    const int buf = kt & 1;
    if(kt + 1 < KT) fetch((kt + 1) * SBK);
#pragma unroll
    for(int kk = 0; kk < SBK; ++kk) {
      const float4 a0 = *(const float4*)&As[buf][kk][ty * 4];
      const float4 a1 = *(const float4*)&As[buf][kk][64 + ty * 4];
      const float4 b0 = *(const float4*)&Bs[buf][kk][tx * 4];
      const float4 b1 = *(const float4*)&Bs[buf][kk][64 + tx * 4];
      const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for(int i = 0; i < 8; ++i)
#pragma unroll
        for(int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    if(kt + 1 < KT) {
      stash(buf ^ 1);
      __syncthreads();
    }
  }

#pragma unroll
  for(int i = 0; i < 8; ++i) {
    const int r = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
    if(r >= m) continue;
#pragma unroll
    for(int j = 0; j < 8; ++j) {
      const int c = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4);
      if(c < n) {
        float* p = C + (size_t)r + (size_t)c * ldc;
        *p       = ACCUM ? *p - acc[i][j] : acc[i][j];
      }
    }
  }
}

}  // namespace

cudaError_t launch_sgemm(int m, int n, int k, const float* A, int64_t lda, const float* B,
                         int64_t ldb, float* C, int64_t ldc, bool accumulate,
                         cudaStream_t stream) {
  if(m <= 0 || n <= 0) return cudaSuccess;
  if(k <= 0 && accumulate) return cudaSuccess;
  dim3 grid((m + SBM - 1) / SBM, (n + SBN - 1) / SBN);
  if(grid.y > 65535) return cudaErrorInvalidValue;
  if(accumulate)
    sgemm_kernel<true><<<grid, 256, 0, stream>>>(m, n, k, A, lda, B, ldb, C, ldc);
  else
    sgemm_kernel<false><<<grid, 256, 0, stream>>>(m, n, k, A, lda, B, ldb, C, ldc);
  return cudaGetLastError();
}

}  // namespace hplb
