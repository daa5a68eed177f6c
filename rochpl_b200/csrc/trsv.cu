// Back-solve U x = y at P = Q = 1 (src/pgesv/HPL_pdtrsv_device.cpp:29-346).
//
// y is column n of the factored [A|b]; x is written to X.  Blocked from the
// bottom up in kTb-row blocks: a one-warp kernel solves the diagonal block out
// of shared memory, then a row-parallel GEMV removes that block's contribution
// from every row above it (rocblas_dtrsv + rocblas_dgemv in the reference).
// The GEMVs stream the upper triangle once: n^2/2 * 8 bytes, HBM-bound.
#include "common.cuh"
#include "internal.h"

namespace hplb {

namespace {

constexpr int kTb = 64;

// Solve the kb x kb upper block at (s, s) in place on X[s : s+kb].
__global__ void __launch_bounds__(32) trsv_diag_kernel(const double* A, int64_t ld, int s,
                                                       int kb, double* X) {
  __shared__ double U[kTb][kTb + 1];  // U[r][c]
  const int lane = threadIdx.x;
  for(int c = 0; c < kb; ++c)
    for(int r = lane; r < kb; r += 32) U[r][c] = A[(size_t)(s + r) + (size_t)(s + c) * ld];
  double y0 = lane < kb ? X[s + lane] : 0.0;
  double y1 = lane + 32 < kb ? X[s + lane + 32] : 0.0;
  __syncwarp();
  for(int i = kb - 1; i >= 0; --i) {
    const double yi = __shfl_sync(0xffffffffu, i < 32 ? y0 : y1, i & 31);
    const double xi = yi / U[i][i];
    if(lane == (i & 31)) {
      if(i < 32)
        y0 = xi;
      else
        y1 = xi;
    }
    if(lane < i) y0 -= U[lane][i] * xi;
    if(lane + 32 < i) y1 -= U[lane + 32][i] * xi;
  }
  if(lane < kb) X[s + lane] = y0;
  if(lane + 32 < kb) X[s + lane + 32] = y1;
}

// X[0:s] -= U[0:s, s:s+kb] X[s:s+kb]; one thread per row, coalesced columns.
__global__ void __launch_bounds__(256) trsv_gemv_kernel(const double* A, int64_t ld, int s,
                                                        int kb, double* X) {
  __shared__ double xs[kTb];
  if(threadIdx.x < kb) xs[threadIdx.x] = X[s + threadIdx.x];
  __syncthreads();
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if(r >= s) return;
  const double* a = A + (size_t)r + (size_t)s * ld;
  double acc = 0.0;
#pragma unroll 8
  for(int c = 0; c < kb; ++c) acc += a[(size_t)c * ld] * xs[c];
  X[r] -= acc;
}

}  // namespace

cudaError_t launch_trsv(const double* A, int64_t ld, int n, double* X, int* status,
                        cudaStream_t stream, int* launches) {
  (void)status;
  if(n <= 0) return cudaSuccess;
  cudaError_t e = cudaMemcpyAsync(X, A + (size_t)n * ld, (size_t)n * sizeof(double),
                                  cudaMemcpyDeviceToDevice, stream);
  if(e != cudaSuccess) return e;
  const int nblk = (n + kTb - 1) / kTb;
  for(int b = nblk - 1; b >= 0; --b) {
    const int s  = b * kTb;
    const int kb = min(kTb, n - s);
    trsv_diag_kernel<<<1, 32, 0, stream>>>(A, ld, s, kb, X);
    ++*launches;
    if(s > 0) {
      trsv_gemv_kernel<<<(s + 255) / 256, 256, 0, stream>>>(A, ld, s, kb, X);
      ++*launches;
    }
  }
  return cudaGetLastError();
}

}  // namespace hplb
