// HPL_pdrandmat at P = Q = 1 (src/matgen/HPL_pdrandmat_device.cpp:84-201),
// written as a pure HBM store stream.
//
// Entry (i, j) of the m-row matrix is the LCG state X(1 + i + j m) with
// X(0) = seed.  A warp owns a run of 32*kRowsPerLane consecutive rows of one
// column: lane l starts at row run0 + l and advances 32 rows per step with the
// 32-step jump, so each store instruction writes 256 contiguous bytes.  The
// per-warp start state is one jump computed by lane 0 from a shared-memory
// table of the 2^k jumps.  The reference instead walks block and column jumps
// serially per thread (:49-56).
#include "common.cuh"
#include "internal.h"
#include "lcg.cuh"

namespace hplb {

namespace {

constexpr int kRowsPerLane = 16;           // rows per lane per column run
constexpr int kRun         = 32 * kRowsPerLane;
constexpr int kWarps       = 8;

struct MatgenTables {
  Jump pow2[64];  // jump by 2^k
  Jump lane[32];  // jump by l (lane offset)
  Jump step32;    // jump by 32
};

// Block (gi0, gj0) .. (gi0 + m, gj0 + n) of the global matrix with mg rows:
// local entry (i, j) is global entry (gi0 + i, gj0 + j).
template <typename T>
__global__ void __launch_bounds__(kWarps * 32)
matgen_kernel(int m, int n, int64_t ld, T* __restrict__ A, uint64_t x1, uint64_t mg,
              uint64_t gi0, uint64_t gj0, MatgenTables Tab) {
  __shared__ Jump s_pow2[64];
  __shared__ Jump s_lane[32];
  for(int i = threadIdx.x; i < 64; i += blockDim.x) s_pow2[i] = Tab.pow2[i];
  if(threadIdx.x < 32) s_lane[threadIdx.x] = Tab.lane[threadIdx.x];
  __syncthreads();

  const int lane   = threadIdx.x & 31;
  const int runs   = (m + kRun - 1) / kRun;
  const int64_t wg = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
  if(wg >= (int64_t)runs * n) return;
  const int     j  = (int)(wg / runs);
  const int     i0 = (int)(wg % runs) * kRun;

  // State of global (gi0 + i0, gj0 + j): X(1 + gi0 + i0 + (gj0 + j) mg), the
  // jump by gi0 + i0 + (gj0 + j) mg (mod 2^64) applied to X(1).
  uint64_t s = 0;
  if(lane == 0) {
    uint64_t k   = gi0 + (uint64_t)i0 + (gj0 + (uint64_t)j) * mg;
    Jump     acc = {1, 0};
    for(int b = 0; k; ++b, k >>= 1)
      if(k & 1) acc = compose(acc, s_pow2[b]);
    s = apply(acc, x1);
  }
  s = __shfl_sync(0xffffffffu, s, 0);
  s = apply(s_lane[lane], s);

  T* col = A + (size_t)j * (size_t)ld;
  const Jump st = Tab.step32;
  if(i0 + kRun <= m) {
#pragma unroll 4
    for(int r = 0; r < kRowsPerLane; ++r) {
      col[i0 + r * 32 + lane] = (T)lcg_value(s);
      s = apply(st, s);
    }
  } else {
    for(int r = 0; r < kRowsPerLane; ++r) {
      const int i = i0 + r * 32 + lane;
      if(i < m) col[i] = (T)lcg_value(s);
      s = apply(st, s);
    }
  }
}

}  // namespace

template <typename E>
static cudaError_t matgen_any(int m, int n, uint64_t seed, E* A, int64_t ld, int64_t mg,
                              int64_t gi0, int64_t gj0, cudaStream_t stream) {
  if(m <= 0 || n <= 0) return cudaSuccess;
  MatgenTables T;
  Jump p{kLcgMult, kLcgAdd};
  for(int b = 0; b < 64; ++b) {
    T.pow2[b] = p;
    p         = compose(p, p);
  }
  for(int l = 0; l < 32; ++l) T.lane[l] = jump_by((uint64_t)l);
  T.step32          = jump_by(32);
  const uint64_t x1 = kLcgMult * seed + kLcgAdd;
  const int64_t runs  = (m + kRun - 1) / kRun;
  const int64_t warps = runs * (int64_t)n;
  const int64_t grid  = (warps + kWarps - 1) / kWarps;
  matgen_kernel<E><<<(unsigned)grid, kWarps * 32, 0, stream>>>(
      m, n, ld, A, x1, (uint64_t)mg, (uint64_t)gi0, (uint64_t)gj0, T);
  return cudaGetLastError();
}

cudaError_t launch_matgen(int m, int n, uint64_t seed, double* A, int64_t ld,
                          cudaStream_t stream) {
  return matgen_any<double>(m, n, seed, A, ld, m, 0, 0, stream);
}

cudaError_t launch_matgen_block(int64_t mg, int64_t i0, int64_t j0, int m, int n, uint64_t seed,
                                double* A, int64_t ld, cudaStream_t stream) {
  return matgen_any<double>(m, n, seed, A, ld, mg, i0, j0, stream);
}

// The same matrix rounded to FP32 (the working copy of the mixed-precision solve).
cudaError_t launch_matgen_f32(int m, int n, uint64_t seed, float* W, int64_t ld,
                              cudaStream_t stream) {
  return matgen_any<float>(m, n, seed, W, ld, m, 0, 0, stream);
}

}  // namespace hplb
