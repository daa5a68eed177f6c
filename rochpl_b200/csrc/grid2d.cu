// Local kernels of the P x Q process grid (rochpl_b200/grid2d.py), where a
// panel column's rows are spread over the processes of a process column:
//
//   col_argmax_kernel  the local part of the pivot search of one column (the
//                      per-process arg-max that HPL_pdmxswp combines across the
//                      process column, src/pfact/HPL_pdmxswp.cpp:19-126):
//                      the largest |a| over rows [r0, r1), the lowest row
//                      among equal values, one CTA;
//   col_rank1_kernel   the leaf's column step on the local rows: the
//                      multiplier l = a_k / pivot (division, as
//                      src/pfact/HPL_pdpanrlT_device.cpp:232) into column k,
//                      then a_c - l u_c for the leaf's later columns; a thread
//                      per row, each column a coalesced walk.
#include <algorithm>

#include "common.cuh"
#include "internal.h"

namespace hplb {

namespace {

constexpr int kArgmaxThreads = 1024;

HPLB_DEV bool better_row(double av, int ar, double bv, int br) {
  if(br < 0) return ar >= 0;
  if(ar < 0) return false;
  const double fa = fabs(av), fb = fabs(bv);
  if(fa > fb) return true;
  if(fa < fb) return false;
  return ar < br;
}

__global__ void __launch_bounds__(kArgmaxThreads)
col_argmax_kernel(const double* __restrict__ A, int64_t ld, int r0, int r1, int c,
                  double* __restrict__ out) {
  __shared__ double s_v[kArgmaxThreads / 32];
  __shared__ int    s_r[kArgmaxThreads / 32];
  const double* col = A + (size_t)c * (size_t)ld;
  double        v   = 0.0;
  int           r   = -1;
  for(int i = r0 + (int)threadIdx.x; i < r1; i += blockDim.x) {
    const double x = col[i];
    if(better_row(x, i, v, r)) {
      v = x;
      r = i;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  warp_argmax(v, r);
  if(lane == 0) {
    s_v[warp] = v;
    s_r[warp] = r;
  }
  __syncthreads();
  if(warp == 0) {
    const int nw = blockDim.x >> 5;
    v = lane < nw ? s_v[lane] : 0.0;
    r = lane < nw ? s_r[lane] : -1;
    warp_argmax(v, r);
    if(lane == 0) {
      out[0] = v;
      out[1] = (double)r;
    }
  }
}

__global__ void __launch_bounds__(256)
col_rank1_kernel(double* __restrict__ A, int64_t ld, int r0, int r1, int c0, int k, int kend,
                 double piv, const double* __restrict__ u) {
  const size_t lds = (size_t)ld;
  for(int i = r0 + blockIdx.x * blockDim.x + threadIdx.x; i < r1; i += gridDim.x * blockDim.x) {
    double*      a = A + i + (size_t)c0 * lds;
    const double l = a[(size_t)k * lds] / piv;
    a[(size_t)k * lds] = l;
    for(int c = k + 1; c < kend; ++c) a[(size_t)c * lds] = a[(size_t)c * lds] - l * u[c];
  }
}

}  // namespace

cudaError_t launch_col_argmax(const double* A, int64_t ld, int r0, int r1, int c, double* out,
                              cudaStream_t stream) {
  col_argmax_kernel<<<1, kArgmaxThreads, 0, stream>>>(A, ld, r0, r1, c, out);
  return cudaGetLastError();
}

cudaError_t launch_col_rank1(double* A, int64_t ld, int r0, int r1, int c0, int k, int kend,
                             double piv, const double* u, int num_sms, cudaStream_t stream) {
  if(r1 <= r0) return cudaSuccess;
  const int rows = r1 - r0;
  const int grid = std::max(1, std::min((rows + 255) / 256, 4 * std::max(num_sms, 1)));
  col_rank1_kernel<<<grid, 256, 0, stream>>>(A, ld, r0, r1, c0, k, kend, piv, u);
  return cudaGetLastError();
}

}  // namespace hplb
