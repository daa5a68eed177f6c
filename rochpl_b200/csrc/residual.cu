// HPL residual check (src/HPL_pdtest.cpp:307-438 with the norms of
// src/pauxil/HPL_pdlange_device.cpp:76-116), deterministic on the device.
//
// Two sources for [A|b]: a stored matrix (the reference regenerates A in
// place with HPL_pdrandmat before checking), or the LCG itself, regenerated
// inside the kernels with the same bit-exact value function, so the check
// needs no N x N buffer at all.
//
// Work split (all reductions in a fixed order, no floating-point atomics):
//   rows_partial : grid (row blocks, column chunks); per row and chunk the
//                  partial sums of a_ij x_j and |a_ij|.
//   rows_final   : per row r_i = b_i - sum, row sum of |a|; per block the
//                  maxima of |r|, row sums, |b|, |x| and the sum of |x|.
//   col_sums     : one warp per column: sum_i |a_ij|; per block the max.
//   finish       : one block folds the per-block values into the 8 outputs.
#include "common.cuh"
#include "internal.h"
#include "lcg.cuh"

namespace hplb {

namespace {

constexpr int kRowThreads = 256;
constexpr int kChunk      = 2048;  // columns per partial sum

struct ResTabs {
  Jump pow2[64];
  Jump col;     // jump by n (next column, same row)
  Jump step32;  // jump by 32 (same column, 32 rows down)
  uint64_t x1;  // X(1)
};

HPLB_DEV uint64_t state_of(const ResTabs& T, uint64_t k) {
  Jump acc{1, 0};
  for(int b = 0; k; ++b, k >>= 1)
    if(k & 1) acc = compose(acc, T.pow2[b]);
  return apply(acc, T.x1);
}

template <bool LCG>
__global__ void __launch_bounds__(kRowThreads)
rows_partial(int n, const double* __restrict__ A, int64_t ld, const double* __restrict__ X,
             const ResTabs* __restrict__ T, double* part_r, double* part_a) {
  const int i  = blockIdx.x * kRowThreads + threadIdx.x;
  const int j0 = blockIdx.y * kChunk;
  const int j1 = min(n, j0 + kChunk);
  if(i >= n) return;
  double acc = 0.0, asum = 0.0;
  if(LCG) {
    const Jump cj = T->col;
    uint64_t   s  = state_of(*T, (uint64_t)i + (uint64_t)j0 * (uint64_t)n);
    for(int j = j0; j < j1; ++j) {
      const double a = lcg_value(s);
      acc += a * X[j];
      asum += fabs(a);
      s = apply(cj, s);
    }
  } else {
    const double* a = A + (size_t)i + (size_t)j0 * ld;
#pragma unroll 4
    for(int j = j0; j < j1; ++j, a += ld) {
      const double v = *a;
      acc += v * X[j];
      asum += fabs(v);
    }
  }
  part_r[(size_t)blockIdx.y * n + i] = acc;
  part_a[(size_t)blockIdx.y * n + i] = asum;
}

HPLB_DEV double block_max(double v, double* sh) {
  for(int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if(lane == 0) sh[warp] = v;
  __syncthreads();
  v = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
  if(warp == 0)
    for(int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
  return v;  // valid in thread 0
}

HPLB_DEV double block_sum(double v, double* sh) {
  for(int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if(lane == 0) sh[warp] = v;
  __syncthreads();
  v = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
  if(warp == 0)
    for(int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  return v;  // valid in thread 0
}

template <bool LCG>
__global__ void __launch_bounds__(kRowThreads)
rows_final(int n, int nch, const double* __restrict__ A, int64_t ld, const double* __restrict__ X,
           const ResTabs* __restrict__ T, const double* part_r, const double* part_a,
           double* blk) {
  __shared__ double sh[32];
  const int i = blockIdx.x * kRowThreads + threadIdx.x;
  double rabs = 0.0, rsum = 0.0, babs = 0.0, xabs = 0.0, xs = 0.0;
  if(i < n) {
    double b;
    if(LCG)
      b = lcg_value(state_of(*T, (uint64_t)i + (uint64_t)n * (uint64_t)n));
    else
      b = A[(size_t)i + (size_t)n * ld];
    double acc = 0.0;
    for(int c = 0; c < nch; ++c) {
      acc += part_r[(size_t)c * n + i];
      rsum += part_a[(size_t)c * n + i];
    }
    rabs = fabs(b - acc);
    babs = fabs(b);
    xabs = fabs(X[i]);
    xs   = xabs;
  }
  const double m0 = block_max(rabs, sh);
  const double m1 = block_max(rsum, sh);
  const double m2 = block_max(babs, sh);
  const double m3 = block_max(xabs, sh);
  const double s4 = block_sum(xs, sh);
  if(threadIdx.x == 0) {
    double* o = blk + (size_t)blockIdx.x * 5;
    o[0] = m0;
    o[1] = m1;
    o[2] = m2;
    o[3] = m3;
    o[4] = s4;
  }
}

template <bool LCG>
__global__ void __launch_bounds__(256)
col_sums(int n, const double* __restrict__ A, int64_t ld, const ResTabs* __restrict__ T,
         double* blkc) {
  __shared__ double sh[32];
  const int lane = threadIdx.x & 31;
  const int j    = blockIdx.x * 8 + (threadIdx.x >> 5);
  double    s    = 0.0;
  if(j < n) {
    if(LCG) {
      const Jump st = T->step32;
      uint64_t   x  = state_of(*T, (uint64_t)lane + (uint64_t)j * (uint64_t)n);
      for(int i = lane; i < n; i += 32) {
        s += fabs(lcg_value(x));
        x = apply(st, x);
      }
    } else {
      const double* a = A + (size_t)j * ld;
      for(int i = lane; i < n; i += 32) s += fabs(a[i]);
    }
    for(int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  }
  // s valid in lane 0 of each warp; block max over the 8 columns.
  s = __shfl_sync(0xffffffffu, s, 0);
  const double m = block_max(lane == 0 ? s : 0.0, sh);
  if(threadIdx.x == 0) blkc[blockIdx.x] = m;
}

__global__ void __launch_bounds__(256) finish(int n, int nrb, int ncb, const double* blk,
                                              const double* blkc, double* out) {
  __shared__ double sh[32];
  double v[5] = {0, 0, 0, 0, 0};
  for(int b = threadIdx.x; b < nrb; b += blockDim.x) {
    const double* o = blk + (size_t)b * 5;
    v[0] = fmax(v[0], o[0]);
    v[1] = fmax(v[1], o[1]);
    v[2] = fmax(v[2], o[2]);
    v[3] = fmax(v[3], o[3]);
  }
  // The |x| sum in block order, one thread, for a fixed summation order.
  double cm = 0.0;
  for(int b = threadIdx.x; b < ncb; b += blockDim.x) cm = fmax(cm, blkc[b]);
  const double rn = block_max(v[0], sh);
  const double ai = block_max(v[1], sh);
  const double bn = block_max(v[2], sh);
  const double xi = block_max(v[3], sh);
  const double a1 = block_max(cm, sh);
  if(threadIdx.x == 0) {
    double x1 = 0.0;
    for(int b = 0; b < nrb; ++b) x1 += blk[(size_t)b * 5 + 4];
    const double eps = 0x1p-53;
    out[0] = n > 0 ? rn / (eps * (ai * xi + bn) * (double)n) : 0.0;
    out[1] = rn;
    out[2] = a1;
    out[3] = ai;
    out[4] = x1;
    out[5] = xi;
    out[6] = bn;
    out[7] = eps;
  }
}

}  // namespace

size_t residual_ws_doubles(int n) {
  const size_t nch = (size_t)(n + kChunk - 1) / kChunk;
  const size_t nrb = (size_t)(n + kRowThreads - 1) / kRowThreads;
  const size_t ncb = (size_t)(n + 7) / 8;
  const size_t tabs = (sizeof(ResTabs) + 7) / 8;
  return 2 * nch * (size_t)n + 5 * nrb + ncb + tabs + 16;
}

cudaError_t launch_residual(int n, const double* A, int64_t ld, bool lcg, uint64_t seed,
                            const double* X, double* ws, double* out8, cudaStream_t stream) {
  if(n <= 0) return cudaMemsetAsync(out8, 0, 8 * sizeof(double), stream);
  const int nch = (n + kChunk - 1) / kChunk;
  const int nrb = (n + kRowThreads - 1) / kRowThreads;
  const int ncb = (n + 7) / 8;
  double* part_r = ws;
  double* part_a = part_r + (size_t)nch * n;
  double* blk    = part_a + (size_t)nch * n;
  double* blkc   = blk + (size_t)nrb * 5;
  ResTabs* dT = reinterpret_cast<ResTabs*>(((uintptr_t)(blkc + ncb) + 63) & ~(uintptr_t)63);

  ResTabs T;
  Jump p{kLcgMult, kLcgAdd};
  for(int b = 0; b < 64; ++b) {
    T.pow2[b] = p;
    p         = compose(p, p);
  }
  T.col    = jump_by((uint64_t)n);
  T.step32 = jump_by(32);
  T.x1     = kLcgMult * seed + kLcgAdd;
  cudaError_t e = cudaMemcpyAsync(dT, &T, sizeof(T), cudaMemcpyHostToDevice, stream);
  if(e != cudaSuccess) return e;
  // The host copy of T must outlive the async copy.
  e = cudaStreamSynchronize(stream);
  if(e != cudaSuccess) return e;

  dim3 g1(nrb, nch);
  if(lcg) {
    rows_partial<true><<<g1, kRowThreads, 0, stream>>>(n, A, ld, X, dT, part_r, part_a);
    rows_final<true><<<nrb, kRowThreads, 0, stream>>>(n, nch, A, ld, X, dT, part_r, part_a, blk);
    col_sums<true><<<ncb, 256, 0, stream>>>(n, A, ld, dT, blkc);
  } else {
    rows_partial<false><<<g1, kRowThreads, 0, stream>>>(n, A, ld, X, dT, part_r, part_a);
    rows_final<false><<<nrb, kRowThreads, 0, stream>>>(n, nch, A, ld, X, dT, part_r, part_a, blk);
    col_sums<false><<<ncb, 256, 0, stream>>>(n, A, ld, dT, blkc);
  }
  finish<<<1, 256, 0, stream>>>(n, nrb, ncb, blk, blkc, out8);
  return cudaGetLastError();
}

namespace {

// y[i] = sum of the per-chunk partials of row i (fixed order).
__global__ void rows_sum(int n, int nch, const double* __restrict__ part, double* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) return;
  double acc = 0.0;
  for(int c = 0; c < nch; ++c) acc += part[(size_t)c * n + i];
  y[i] = acc;
}

// out[i] = A(i, col), from the stored matrix or regenerated from the LCG.
template <bool LCG>
__global__ void column_of(int n, int col, const double* __restrict__ A, int64_t ld,
                          const ResTabs* __restrict__ T, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) return;
  if(LCG)
    out[i] = lcg_value(state_of(*T, (uint64_t)i + (uint64_t)col * (uint64_t)n));
  else
    out[i] = A[(size_t)i + (size_t)col * ld];
}

cudaError_t upload_tabs(int n, uint64_t seed, ResTabs* dT, cudaStream_t stream) {
  ResTabs T;
  Jump p{kLcgMult, kLcgAdd};
  for(int b = 0; b < 64; ++b) {
    T.pow2[b] = p;
    p         = compose(p, p);
  }
  T.col    = jump_by((uint64_t)n);
  T.step32 = jump_by(32);
  T.x1     = kLcgMult * seed + kLcgAdd;
  cudaError_t e = cudaMemcpyAsync(dT, &T, sizeof(T), cudaMemcpyHostToDevice, stream);
  if(e != cudaSuccess) return e;
  return cudaStreamSynchronize(stream);  // T lives on this stack frame
}

}  // namespace

// y = A x for the n x n part of [A|b], FP64, from the stored matrix or the LCG.
// ws: residual_ws_doubles(n) doubles.
cudaError_t launch_gemv_hpl(int n, const double* A, int64_t ld, bool lcg, uint64_t seed,
                            const double* x, double* y, double* ws, cudaStream_t stream) {
  if(n <= 0) return cudaSuccess;
  const int nch = (n + kChunk - 1) / kChunk;
  const int nrb = (n + kRowThreads - 1) / kRowThreads;
  double*   part_r = ws;
  double*   part_a = part_r + (size_t)nch * n;
  ResTabs*  dT = reinterpret_cast<ResTabs*>(((uintptr_t)(part_a + (size_t)nch * n) + 63) &
                                            ~(uintptr_t)63);
  cudaError_t e = upload_tabs(n, seed, dT, stream);
  if(e != cudaSuccess) return e;
  dim3 g1(nrb, nch);
  if(lcg)
    rows_partial<true><<<g1, kRowThreads, 0, stream>>>(n, A, ld, x, dT, part_r, part_a);
  else
    rows_partial<false><<<g1, kRowThreads, 0, stream>>>(n, A, ld, x, dT, part_r, part_a);
  rows_sum<<<nrb, kRowThreads, 0, stream>>>(n, nch, part_r, y);
  return cudaGetLastError();
}

// out = column col of [A|b] (col = n gives b).
cudaError_t launch_column_hpl(int n, int col, const double* A, int64_t ld, bool lcg,
                              uint64_t seed, double* out, double* ws, cudaStream_t stream) {
  if(n <= 0) return cudaSuccess;
  ResTabs* dT = reinterpret_cast<ResTabs*>(((uintptr_t)ws + 63) & ~(uintptr_t)63);
  cudaError_t e = upload_tabs(n, seed, dT, stream);
  if(e != cudaSuccess) return e;
  const int nrb = (n + kRowThreads - 1) / kRowThreads;
  if(lcg)
    column_of<true><<<nrb, kRowThreads, 0, stream>>>(n, col, A, ld, dT, out);
  else
    column_of<false><<<nrb, kRowThreads, 0, stream>>>(n, col, A, ld, dT, out);
  return cudaGetLastError();
}

}  // namespace hplb

// ---------------------------------------------------------------------------
// Allocation-free residual check.
//
// For callers that must not allocate device memory at all: a host program that
// has handed every byte of device memory to its own pool, or a check that runs
// between solves in a loop where cudaMalloc's implicit device synchronisation is
// not allowed.  The scratch of the kernels above lives in the file-scope array
// below instead of a context workspace, so this entry point needs neither a
// context nor an allocation.  The array is fixed in size (it serves
// n <= HPLB_NOALLOC_MAX_N) and every GPU that loads the library holds it until
// the process exits.
// ---------------------------------------------------------------------------

#include <cstdio>
#include <mutex>

namespace hplb {
namespace {

constexpr int    kNoAllocMaxN = HPLB_NOALLOC_MAX_N;
constexpr size_t kNoAllocWs   = 2 * ((size_t)(kNoAllocMaxN + kChunk - 1) / kChunk) * kNoAllocMaxN +
                                5 * ((size_t)(kNoAllocMaxN + kRowThreads - 1) / kRowThreads) +
                                (size_t)(kNoAllocMaxN + 7) / 8 + (sizeof(ResTabs) + 7) / 8 + 16 + 8;

// Shared by every call on a device; it keeps the last call's contents.  No
// kernel of the check accumulates into it (every partial sum, per-block value
// and output is overwritten before it is read), so nothing has to be cleared.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocWs];

constexpr int kMaxDevices = 64;
std::mutex    g_noalloc_mu;
double*       g_noalloc_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device.  In host code the
// array's name is only a host-side stand-in, so the address is looked up once
// per device (with that device current) and cached.
cudaError_t noalloc_scratch(int dev, double** out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if(!g_noalloc_ptr[dev]) {
    void*       p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if(e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = (double*)p;
  }
  *out = g_noalloc_ptr[dev];
  return cudaSuccess;
}

}  // namespace
}  // namespace hplb

extern "C" hplb_status hplb_residual_lcg_noalloc(int n, uint64_t seed, const double* dX,
                                                 void* stream, hplb_resid* out) {
  using namespace hplb;
  if(!out || n < 0 || (n > 0 && !dX)) return HPLB_ERR_ARG;
  if(n > kNoAllocMaxN) {
    fprintf(stderr,
            "hplb_residual_lcg_noalloc: n = %d exceeds the static scratch limit "
            "HPLB_NOALLOC_MAX_N = %d; use hplb_residual_lcg\n",
            n, kNoAllocMaxN);
    return HPLB_ERR_ARG;
  }
  int dev = 0;
  if(cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return HPLB_ERR_CUDA;
  }
  double* ws = nullptr;
  if(noalloc_scratch(dev, &ws) != cudaSuccess) {
    cudaGetLastError();
    return HPLB_ERR_CUDA;
  }
  cudaStream_t st   = (cudaStream_t)stream;
  double*      out8 = ws + (kNoAllocWs - 8);
  if(launch_residual(n, nullptr, 0, true, seed, dX, ws, out8, st) != cudaSuccess) {
    cudaGetLastError();
    return HPLB_ERR_CUDA;
  }
  double o[8];
  if(cudaMemcpyAsync(o, out8, sizeof o, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
     cudaStreamSynchronize(st) != cudaSuccess) {
    cudaGetLastError();
    return HPLB_ERR_CUDA;
  }
  out->resid     = o[0];
  out->rnorm_inf = o[1];
  out->anorm_1   = o[2];
  out->anorm_inf = o[3];
  out->xnorm_1   = o[4];
  out->xnorm_inf = o[5];
  out->bnorm_inf = o[6];
  out->eps       = o[7];
  return HPLB_OK;
}
