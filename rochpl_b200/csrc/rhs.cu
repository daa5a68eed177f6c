// Kernels for solves with the stored HPL factors and many right-hand sides
// (hplb_getrs) and for the fused rank-k product of the solve's adjoint
// (hplb_rank_k).  No counterpart in the reference (its solve carries a single
// b through the factorisation, src/pgesv/HPL_pdgesv.cpp).
//
//   transpose      dst = src^T, 32 x 32 tiles through shared memory
//   laswp_inverse  P^T applied to columns of B: the inverse of a panel's row
//                  map (new row x came from permU[x]; old top row s went to
//                  permU[jb + s] or stayed in the top block when that is -1)
//   rank_k         C = alpha A B^T (+ C), k <= 64: 64 x 64 output tiles, A and B
//                  slices in shared memory, streaming stores (C is written once)
//   check_ipiv     pivots in range before any kernel indexes with them
#include <algorithm>

#include "common.cuh"
#include "internal.h"

namespace hplb {

namespace {

template <typename T>
__global__ void transpose_kernel(int m, int n, const T* __restrict__ src, int64_t lds,
                                 T* __restrict__ dst, int64_t ldd) {
  __shared__ T tile[32][33];
  const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  for(int q = threadIdx.y; q < 32; q += blockDim.y) {
    const int r = r0 + threadIdx.x, c = c0 + q;
    if(r < m && c < n) tile[q][threadIdx.x] = src[(size_t)r + (size_t)c * lds];
  }
  __syncthreads();
  for(int q = threadIdx.y; q < 32; q += blockDim.y) {
    const int r = r0 + q, c = c0 + threadIdx.x;  // dst(c, r) = src(r, c)
    if(r < m && c < n) dst[(size_t)c + (size_t)r * ldd] = tile[threadIdx.x][q];
  }
}

// One column of B per block; all reads land in shared memory before any write,
// so the permutation is applied in place.
__global__ void laswp_inverse_kernel(double* B, int64_t ldb, int ia, int jb,
                                     const int* __restrict__ permU) {
  extern __shared__ double sm[];
  double* t_new = sm;       // B(ia + x) for the top rows (new order)
  double* t_dis = sm + jb;  // the row each displaced old top row moved to
  double* col   = B + (size_t)blockIdx.x * ldb + ia;
  for(int x = threadIdx.x; x < jb; x += blockDim.x) {
    t_new[x]    = col[x];
    const int d = permU[jb + x];
    t_dis[x]    = d >= 0 ? col[d] : 0.0;
  }
  __syncthreads();
  for(int x = threadIdx.x; x < jb; x += blockDim.x) col[permU[x]] = t_new[x];
  for(int x = threadIdx.x; x < jb; x += blockDim.x)
    if(permU[jb + x] >= 0) col[x] = t_dis[x];
}

constexpr int RK_T = 64, RK_K = 32;

template <bool ACCUM>
__global__ void __launch_bounds__(256)
rank_k_kernel(int m, int n, int k, double alpha, const double* __restrict__ A, int64_t lda,
              const double* __restrict__ B, int64_t ldb, double* __restrict__ C, int64_t ldc) {
  __shared__ double As[RK_K][RK_T];
  __shared__ double Bs[RK_K][RK_T];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.x * RK_T, n0 = blockIdx.y * RK_T;
  double acc[4][4] = {};
  for(int k0 = 0; k0 < k; k0 += RK_K) {
    const int kc = min(RK_K, k - k0);
    for(int idx = tid; idx < RK_K * RK_T; idx += 256) {
      const int r = idx & (RK_T - 1), kk = idx >> 6;
      As[kk][r] = (kk < kc && m0 + r < m) ? A[(size_t)(m0 + r) + (size_t)(k0 + kk) * lda] : 0.0;
      Bs[kk][r] = (kk < kc && n0 + r < n) ? B[(size_t)(n0 + r) + (size_t)(k0 + kk) * ldb] : 0.0;
    }
    __syncthreads();
    for(int kk = 0; kk < kc; ++kk) {
      double a[4], b[4];
#pragma unroll
      for(int i = 0; i < 4; ++i) a[i] = As[kk][tx + 16 * i];
#pragma unroll
      for(int j = 0; j < 4; ++j) b[j] = Bs[kk][ty + 16 * j];
#pragma unroll
      for(int i = 0; i < 4; ++i)
#pragma unroll
        for(int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for(int j = 0; j < 4; ++j) {
    const int c = n0 + ty + 16 * j;
    if(c >= n) continue;
#pragma unroll
    for(int i = 0; i < 4; ++i) {
      const int r = m0 + tx + 16 * i;
      if(r >= m) continue;
      double* p = C + (size_t)r + (size_t)c * ldc;
      if(ACCUM)
        *p += alpha * acc[i][j];
      else
        __stcs(p, alpha * acc[i][j]);
    }
  }
}

__global__ void unit_lower_view_kernel(int kind, int jb, const double* __restrict__ T,
                                       int64_t ldt, double* __restrict__ out,
                                       double* __restrict__ d) {
  const int c = blockIdx.x;
  for(int r = threadIdx.x; r < jb; r += blockDim.x) {
    double v = r == c ? 1.0 : 0.0;
    if(r > c) {
      if(kind == 0) {  // (J D^-1 U J)[r][c] = U[jb-1-r][jb-1-c] / U[jb-1-r][jb-1-r]
        const int ur = jb - 1 - r, uc = jb - 1 - c;
        v = T[(size_t)ur + (size_t)uc * ldt] / T[(size_t)ur + (size_t)ur * ldt];
      } else if(kind == 1) {  // (J L^T J)[r][c] = L[jb-1-c][jb-1-r]
        v = T[(size_t)(jb - 1 - c) + (size_t)(jb - 1 - r) * ldt];
      } else {  // ((D^-1 U)^T)[r][c] = U[c][r] / U[c][c]
        v = T[(size_t)c + (size_t)r * ldt] / T[(size_t)c + (size_t)c * ldt];
      }
    }
    out[(size_t)r + (size_t)c * jb] = v;
  }
  if(c == 0 && kind != 1)
    for(int i = threadIdx.x; i < jb; i += blockDim.x) d[i] = T[(size_t)i + (size_t)i * ldt];
}

__global__ void rows_xform_kernel(int jb, const double* __restrict__ in, int64_t ldi,
                                  double* __restrict__ out, int64_t ldo,
                                  const double* __restrict__ d, int flip, int scale) {
  const int c = blockIdx.x;
  for(int i = threadIdx.x; i < jb; i += blockDim.x) {
    const int src = flip ? jb - 1 - i : i;
    double    v   = in[(size_t)src + (size_t)c * ldi];
    if(scale) v = v / d[src];
    out[(size_t)i + (size_t)c * ldo] = v;
  }
}

// X (jb x ncols) <- L^-1 X for a unit-lower L and few right-hand sides: one
// CTA per column, the column in shared memory.  Per 32-row block the 16 warps
// split the dot products of the block's rows with the solved rows above (lane
// = row, so each step reads 32 consecutive entries of a column of L), a fixed
// order sum of the 16 slices, then the block's 32 x 32 inverse (dinv, from
// diag_inv) applied.
constexpr int kSmallThreads = 512;
__global__ void __launch_bounds__(kSmallThreads)
trsm_small_kernel(int jb, double* X, int64_t ldx, const double* __restrict__ L, int64_t ldl,
                  const double* __restrict__ dinv) {
  extern __shared__ double xs[];
  __shared__ double part[kSmallThreads / 32][33];
  __shared__ double tmp[32];
  double*   col  = X + (size_t)blockIdx.x * ldx;
  const int lane = threadIdx.x & 31, sl = threadIdx.x >> 5, nsl = kSmallThreads / 32;
  for(int i = threadIdx.x; i < jb; i += kSmallThreads) xs[i] = col[i];
  __syncthreads();
  for(int b0 = 0; b0 < jb; b0 += 32) {
    const int r   = b0 + lane;
    double    acc = 0.0, acc2 = 0.0;
    if(r < jb) {
      const double* lr = L + r;
      int           k  = sl;
      for(; k + 7 * nsl < b0; k += 8 * nsl) {  // eight loads in flight, two chains
        double a[8];
#pragma unroll
        for(int q = 0; q < 8; ++q) a[q] = lr[(size_t)(k + q * nsl) * ldl];
#pragma unroll
        for(int q = 0; q < 8; q += 2) {
          acc  = fma(a[q], xs[k + q * nsl], acc);
          acc2 = fma(a[q + 1], xs[k + (q + 1) * nsl], acc2);
        }
      }
      for(; k < b0; k += nsl) acc = fma(lr[(size_t)k * ldl], xs[k], acc);
      acc += acc2;
    }
    part[sl][lane] = acc;
    __syncthreads();
    if(threadIdx.x < 32) {
      double t = 0.0;
      for(int q = 0; q < nsl; ++q) t += part[q][lane];
      tmp[lane] = r < jb ? xs[r] - t : 0.0;
    }
    __syncthreads();
    if(threadIdx.x < 32 && r < jb) {
      const double* D = dinv + (size_t)(b0 / 32) * 1024;
      double        x = 0.0;
#pragma unroll 8
      for(int c = 0; c < 32; ++c) x += D[c * 32 + lane] * tmp[c];
      xs[r] = x;
    }
    __syncthreads();
  }
  for(int i = threadIdx.x; i < jb; i += kSmallThreads) col[i] = xs[i];
}

// Split-k partial products for C (jb x nrhs) -= M (jb x K) Y (K x nrhs) with
// K much larger than jb and nrhs: CTA (chunk, column block) writes
// part[chunk] = M[:, chunk] Y[chunk, 32 columns]; Y's slice in shared memory,
// each thread 32 accumulators per row it owns.
constexpr int kSkK = 128;
__global__ void __launch_bounds__(256)
splitk_partial_kernel(int jb, int nrhs, int K, const double* __restrict__ M, int64_t ldm,
                      const double* __restrict__ Y, int64_t ldy, double* __restrict__ part) {
  __shared__ double ys[kSkK][33];
  const int k0 = blockIdx.x * kSkK, c0 = blockIdx.y * 32;
  const int kc = min(kSkK, K - k0), ncb = min(32, nrhs - c0);
  for(int e = threadIdx.x; e < kSkK * 32; e += 256) {
    const int k = e % kSkK, c = e / kSkK;
    ys[k][c] = (k < kc && c < ncb) ? Y[(size_t)(k0 + k) + (size_t)(c0 + c) * ldy] : 0.0;
  }
  __syncthreads();
  double* out = part + ((size_t)blockIdx.x * gridDim.y + blockIdx.y) * 32 * (size_t)jb;
  for(int r = threadIdx.x; r < jb; r += 256) {
    double acc[32];
#pragma unroll
    for(int c = 0; c < 32; ++c) acc[c] = 0.0;
    const double* m = M + r + (size_t)k0 * ldm;
    int           k = 0;
    for(; k + 8 <= kc; k += 8) {  // eight loads in flight before their FMAs
      double a[8];
#pragma unroll
      for(int q = 0; q < 8; ++q) a[q] = m[(size_t)(k + q) * ldm];
#pragma unroll
      for(int q = 0; q < 8; ++q)
#pragma unroll
        for(int c = 0; c < 32; ++c) acc[c] = fma(a[q], ys[k + q][c], acc[c]);
    }
    for(; k < kc; ++k) {
      const double a = m[(size_t)k * ldm];
#pragma unroll
      for(int c = 0; c < 32; ++c) acc[c] = fma(a, ys[k][c], acc[c]);
    }
#pragma unroll
    for(int c = 0; c < 32; ++c) out[(size_t)c * jb + r] = acc[c];
  }
}

// C (m x nrhs) -= M (m x K) Y (K x nrhs) for tall M and few right-hand sides:
// 32 rows per CTA (lane = row), the CTA's 8 warps on interleaved slices of
// each 128-deep chunk of k (Y's chunk in shared memory), 32 accumulators per
// thread, 16 loads in flight per warp; the 8 slices are summed in a fixed
// order at the end (C read and written once).
__global__ void __launch_bounds__(256)
rows_sub_kernel(int m, int nrhs, int K, const double* __restrict__ M, int64_t ldm,
                const double* __restrict__ Y, int64_t ldy, double* __restrict__ C, int64_t ldc) {
  __shared__ double ys[kSkK][33];  // also the reduction buffer, 16 columns at a time
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r = blockIdx.x * 32 + lane, c0 = blockIdx.y * 32;
  const int ncb = min(32, nrhs - c0);
  double    acc[32];
#pragma unroll
  for(int c = 0; c < 32; ++c) acc[c] = 0.0;
  for(int k0 = 0; k0 < K; k0 += kSkK) {
    const int kc = min(kSkK, K - k0);
    __syncthreads();
    for(int e = threadIdx.x; e < kSkK * 32; e += 256) {
      const int k = e % kSkK, c = e / kSkK;
      ys[k][c] = (k < kc && c < ncb) ? Y[(size_t)(k0 + k) + (size_t)(c0 + c) * ldy] : 0.0;
    }
    __syncthreads();
    if(r < m) {
      // This warp's k: warp, warp + 8, ... within the chunk (16 of them).
      const double* mr = M + r + (size_t)k0 * ldm;
      double        a[kSkK / 8];
#pragma unroll
      for(int q = 0; q < kSkK / 8; ++q) {
        const int k = warp + 8 * q;
        a[q]        = k < kc ? mr[(size_t)k * ldm] : 0.0;
      }
#pragma unroll
      for(int q = 0; q < kSkK / 8; ++q) {
        const int k = warp + 8 * q;
#pragma unroll
        for(int c = 0; c < 32; ++c) acc[c] = fma(a[q], ys[k][c], acc[c]);
      }
    }
  }
  double(*red)[16][33] = reinterpret_cast<double(*)[16][33]>(&ys[0][0]);  // [8][16][33]
#pragma unroll
  for(int h = 0; h < 2; ++h) {
    __syncthreads();
#pragma unroll
    for(int c = 0; c < 16; ++c) red[warp][c][lane] = acc[h * 16 + c];
    __syncthreads();
    // Thread (column h*16 + c, row lane): sum the 8 slices in order.
    for(int c = warp; c < 16; c += 8) {
      double t = 0.0;
#pragma unroll
      for(int w = 0; w < 8; ++w) t += red[w][c][lane];
      if(r < m && h * 16 + c < ncb) C[(size_t)r + (size_t)(c0 + h * 16 + c) * ldc] -= t;
    }
  }
}

// C -= the sum of the partial products, chunk by chunk in order.
__global__ void splitk_reduce_kernel(int jb, int nrhs, int nchunks, int ncb,
                                     const double* __restrict__ part, double* C, int64_t ldc) {
  const int64_t total = (int64_t)jb * nrhs;
  for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
      e += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(e % jb), c = (int)(e / jb);
    const int cb = c / 32, cc = c % 32;
    double    t  = 0.0;
    for(int q = 0; q < nchunks; ++q)
      t += part[(((size_t)q * ncb + cb) * 32 + cc) * jb + r];
    C[(size_t)r + (size_t)c * ldc] -= t;
  }
}

// Entry i of ipiv (count entries) must lie in [first + i, nrows); the first
// entry that does not is recorded 1-based in status[ST_INFO].
__global__ void check_ipiv_kernel(int count, int first, int nrows, const int* __restrict__ ipiv,
                                  int* status) {
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    if(ipiv[i] < first + i || ipiv[i] >= nrows) record_info(status, i + 1);
}

}  // namespace

template <typename T>
cudaError_t launch_transpose(int m, int n, const T* src, int64_t lds, T* dst, int64_t ldd,
                             cudaStream_t st) {
  if(m <= 0 || n <= 0) return cudaSuccess;
  dim3 grid((m + 31) / 32, (n + 31) / 32);
  if(grid.y > 65535) return cudaErrorInvalidValue;
  transpose_kernel<T><<<grid, dim3(32, 8), 0, st>>>(m, n, src, lds, dst, ldd);
  return cudaGetLastError();
}
template cudaError_t launch_transpose<double>(int, int, const double*, int64_t, double*, int64_t,
                                              cudaStream_t);
template cudaError_t launch_transpose<float>(int, int, const float*, int64_t, float*, int64_t,
                                             cudaStream_t);

cudaError_t launch_laswp_inverse(double* B, int64_t ldb, int ia, int jb, const int* permU, int n,
                                 cudaStream_t st) {
  if(jb <= 0 || n <= 0) return cudaSuccess;
  if(jb > 2048 || n > 65535) return cudaErrorInvalidValue;
  laswp_inverse_kernel<<<n, 256, 2 * jb * sizeof(double), st>>>(B, ldb, ia, jb, permU);
  return cudaGetLastError();
}

cudaError_t launch_rank_k(int m, int n, int k, double alpha, const double* A, int64_t lda,
                          const double* B, int64_t ldb, double* C, int64_t ldc, bool accumulate,
                          cudaStream_t st) {
  if(m <= 0 || n <= 0) return cudaSuccess;
  if(k < 0 || k > 64) return cudaErrorInvalidValue;
  dim3 grid((m + RK_T - 1) / RK_T, (n + RK_T - 1) / RK_T);
  if(grid.y > 65535) return cudaErrorInvalidValue;
  if(accumulate)
    rank_k_kernel<true><<<grid, 256, 0, st>>>(m, n, k, alpha, A, lda, B, ldb, C, ldc);
  else
    rank_k_kernel<false><<<grid, 256, 0, st>>>(m, n, k, alpha, A, lda, B, ldb, C, ldc);
  return cudaGetLastError();
}

cudaError_t launch_unit_lower_view(int kind, int jb, const double* T, int64_t ldt, double* out,
                                   double* d, cudaStream_t st) {
  if(jb <= 0) return cudaSuccess;
  unit_lower_view_kernel<<<jb, 256, 0, st>>>(kind, jb, T, ldt, out, d);
  return cudaGetLastError();
}

cudaError_t launch_rows_xform(int jb, int n, const double* in, int64_t ldi, double* out,
                              int64_t ldo, const double* d, bool flip, bool scale,
                              cudaStream_t st) {
  if(jb <= 0 || n <= 0) return cudaSuccess;
  if(n > 65535) return cudaErrorInvalidValue;
  rows_xform_kernel<<<n, 256, 0, st>>>(jb, in, ldi, out, ldo, d, flip ? 1 : 0, scale ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_trsm_small(int jb, int ncols, double* X, int64_t ldx, const double* L,
                              int64_t ldl, const double* dinv, cudaStream_t st) {
  if(jb <= 0 || ncols <= 0) return cudaSuccess;
  if(jb > 4096 || ncols > 65535) return cudaErrorInvalidValue;
  trsm_small_kernel<<<ncols, kSmallThreads, (size_t)jb * sizeof(double), st>>>(jb, X, ldx, L, ldl,
                                                                              dinv);
  return cudaGetLastError();
}

size_t splitk_ws_doubles(int jb, int nrhs, int K) {
  const size_t nch = (size_t)(K + kSkK - 1) / kSkK, ncb = (size_t)(nrhs + 31) / 32;
  return nch * ncb * 32 * (size_t)jb;
}

cudaError_t launch_splitk_sub(int jb, int nrhs, int K, const double* M, int64_t ldm,
                              const double* Y, int64_t ldy, double* C, int64_t ldc, double* ws,
                              cudaStream_t st) {
  if(jb <= 0 || nrhs <= 0 || K <= 0) return cudaSuccess;
  const int nch = (K + kSkK - 1) / kSkK, ncb = (nrhs + 31) / 32;
  if(ncb > 65535) return cudaErrorInvalidValue;
  splitk_partial_kernel<<<dim3(nch, ncb), 256, 0, st>>>(jb, nrhs, K, M, ldm, Y, ldy, ws);
  const int64_t total = (int64_t)jb * nrhs;
  const int     grid  = (int)std::min<int64_t>((total + 255) / 256, 4096);
  splitk_reduce_kernel<<<grid, 256, 0, st>>>(jb, nrhs, nch, ncb, ws, C, ldc);
  return cudaGetLastError();
}

cudaError_t launch_rows_sub(int m, int nrhs, int K, const double* M, int64_t ldm,
                            const double* Y, int64_t ldy, double* C, int64_t ldc,
                            cudaStream_t st) {
  if(m <= 0 || nrhs <= 0 || K <= 0) return cudaSuccess;
  const int ncb = (nrhs + 31) / 32;
  if(ncb > 65535) return cudaErrorInvalidValue;
  rows_sub_kernel<<<dim3((m + 31) / 32, ncb), 256, 0, st>>>(m, nrhs, K, M, ldm, Y, ldy, C, ldc);
  return cudaGetLastError();
}

cudaError_t launch_check_ipiv_range(int count, int first, int nrows, const int* ipiv,
                                    int* status, cudaStream_t st) {
  if(count <= 0) return cudaSuccess;
  const int grid = (count + 255) / 256 < 1024 ? (count + 255) / 256 : 1024;
  check_ipiv_kernel<<<grid, 256, 0, st>>>(count, first, nrows, ipiv, status);
  return cudaGetLastError();
}

cudaError_t launch_check_ipiv(int n, const int* ipiv, int* status, cudaStream_t st) {
  return launch_check_ipiv_range(n, 0, n, ipiv, status, st);
}

}  // namespace hplb
