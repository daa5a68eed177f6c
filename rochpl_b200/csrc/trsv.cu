// Back-solve U x = y at P = Q = 1 (src/pgesv/HPL_pdtrsv_device.cpp:29-346).
//
// y is column n of the factored [A|b] (or a vector of its own); x is written
// to X; A and y are not modified.
// The reference solves bottom-up in NB blocks: rocblas_dtrsv on the diagonal
// block, then rocblas_dgemv to remove that block's contribution from every row
// above, two serial library calls per block.  Here the whole solve is ONE
// persistent kernel, HBM-bound on the single pass over the upper triangle
// (n^2/2 * 8 bytes):
//
//  * CTA k (in the order CTAs start, from an atomic ticket) owns row block
//    bi = nblk - 1 - k of kTb rows, so row blocks are taken bottom first.
//  * It streams its row panel U[bi, j] for j = nblk-1 down to bi+1, 16-byte
//    column segments, the next tile loaded while it waits for the current one's
//    x block, and accumulates U[bi, j] x_j in registers (each warp owns 8 of
//    the 64 columns of every tile, each lane 2 rows).
//  * x_j is published by the CTA that owns row block j: a release store of
//    flag j after x_j is written; readers acquire it.  A CTA only waits for
//    row blocks below its own, whose tickets were taken by CTAs that started
//    before it, so every wait ends; each is also bounded (status site 41).
//  * While the first flag is awaited the CTA inverts its own diagonal block
//    U_ii in shared memory (off the critical path), so the serial chain
//    through the blocks costs one 64 x 64 product per block instead of a
//    64-step substitution: x_i = U_ii^-1 (y_i - sum_j U_ij x_j).
#include <algorithm>

#include "common.cuh"
#include "internal.h"

namespace hplb {

namespace {

constexpr int kTb          = 64;   // rows (and columns) per block
constexpr int kTrsvThreads = 256;  // 8 warps
constexpr int kTrsvWarps   = kTrsvThreads / 32;
constexpr int kColsPerWarp = kTb / kTrsvWarps;  // columns of a tile per warp
constexpr int kTrsvSite    = 41;

struct TrsvSmem {
  double T[kTb][kTb + 1];          // U_ii, then U_ii^-1 (upper triangular)
  double red[kTrsvWarps][kTb];     // per-warp partial row sums
  double r[kTb];                   // right-hand side of the diagonal block
  double tmp[kTb];
  int    ticket;
};

// Spin (bounded) until flag == 1; false once this or any block timed out.
HPLB_DEV bool wait_flag(const int* flag, int* status, int site = kTrsvSite) {
  if(ld_acquire_gpu(flag) != 0) return true;
  const unsigned long long t0 = globaltimer();
  for(unsigned polls = 1;; ++polls) {
    if(ld_acquire_gpu(flag) != 0) return true;
    if((polls & 31u) == 0) {
      if(ld_acquire_gpu(status + ST_TIMEOUT) != 0) return false;
      if(globaltimer() - t0 > kWaitBudgetNs) {
        atomicCAS(status + ST_TIMEOUT, 0, site);
        return false;
      }
    }
    __nanosleep(32);
  }
}

template <bool VEC>
HPLB_DEV void load_tile(const double* __restrict__ A, int64_t ld, int r0, int c0, int kc,
                        int lane, int warp, double2 (&v)[kColsPerWarp]) {
#pragma unroll
  for(int q = 0; q < kColsPerWarp; ++q) {
    const int c = warp + kTrsvWarps * q;
    if(c < kc) {
      const double* p = A + (size_t)(r0 + 2 * lane) + (size_t)(c0 + c) * (size_t)ld;
      if(VEC) {
        v[q] = __ldcs(reinterpret_cast<const double2*>(p));
      } else {
        v[q].x = __ldcs(p);
        v[q].y = __ldcs(p + 1);
      }
    } else {
      v[q] = make_double2(0.0, 0.0);
    }
  }
}

// In-place inverse of the upper triangular kTb x kTb block T (column by
// column, left to right: column j of the inverse is -T_jj^-1 times the
// already-inverted leading block applied to column j of U).  256 threads.
HPLB_DEV void invert_upper(double (*T)[kTb + 1]) {
  const int t = threadIdx.x, row = t >> 2, part = t & 3;
  for(int j = 0; j < kTb; ++j) {
    double s = 0.0;
    if(row < j)
      for(int k = row + part; k < j; k += 4) s = fma(T[row][k], T[k][j], s);
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    const double d = 1.0 / T[j][j];
    __syncthreads();
    if(part == 0 && row < j) T[row][j] = -d * s;
    if(t == 0) T[j][j] = d;
    __syncthreads();
  }
}

template <bool VEC>
__global__ void __launch_bounds__(kTrsvThreads)
trsv_kernel(const double* __restrict__ A, int64_t ld, int n, const double* __restrict__ Y,
            double* __restrict__ X, int* flags, int* status) {
  __shared__ TrsvSmem S;
  const int nblk = (n + kTb - 1) / kTb;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if(t == 0) S.ticket = atomicAdd(flags + nblk, 1);
  __syncthreads();
  const int bi = nblk - 1 - S.ticket;
  const int r0 = bi * kTb;
  const int kb = min(kTb, n - r0);

  // First tile of the row panel in flight before anything else.
  double2 cur[kColsPerWarp], nxt[kColsPerWarp];
#pragma unroll
  for(int q = 0; q < kColsPerWarp; ++q) cur[q] = nxt[q] = make_double2(0.0, 0.0);
  int     j = nblk - 1;
  if(j > bi) load_tile<VEC>(A, ld, r0, j * kTb, min(kTb, n - j * kTb), lane, warp, cur);

  // Diagonal block (identity beyond kb), inverted while the loads fly.
  for(int idx = t; idx < kTb * kTb; idx += kTrsvThreads) {
    const int c = idx / kTb, r = idx % kTb;
    double    v = (r == c) ? 1.0 : 0.0;
    if(r < kb && c < kb) v = r <= c ? A[(size_t)(r0 + r) + (size_t)(r0 + c) * (size_t)ld] : 0.0;
    S.T[r][c] = v;
  }
  if(t < kTb) S.r[t] = t < kb ? Y[r0 + t] : 0.0;
  __syncthreads();
  invert_upper(S.T);

  // Row panel: acc = sum_j U[bi, j] x_j over the rows 2 lane, 2 lane + 1.
  double acc0 = 0.0, acc1 = 0.0;
  bool   alive = true;
  for(; j > bi; --j) {
    if(j - 1 > bi) load_tile<VEC>(A, ld, r0, (j - 1) * kTb, kTb, lane, warp, nxt);
    if(alive) alive = wait_flag(flags + j, status);
    const double* xj = X + (size_t)j * kTb;
    const int     kc = min(kTb, n - j * kTb);
#pragma unroll
    for(int q = 0; q < kColsPerWarp; ++q) {
      const int    c  = warp + kTrsvWarps * q;
      const double xc = c < kc ? __ldcg(xj + c) : 0.0;
      acc0            = fma(cur[q].x, xc, acc0);
      acc1            = fma(cur[q].y, xc, acc1);
    }
#pragma unroll
    for(int q = 0; q < kColsPerWarp; ++q) cur[q] = nxt[q];
  }

  // r = y_i - sum_j U_ij x_j, then x_i = U_ii^-1 r.
  S.red[warp][2 * lane]     = acc0;
  S.red[warp][2 * lane + 1] = acc1;
  __syncthreads();
  if(t < kTb) {
    double s = 0.0;
#pragma unroll
    for(int w = 0; w < kTrsvWarps; ++w) s += S.red[w][t];
    S.tmp[t] = S.r[t] - s;
  }
  __syncthreads();
  {
    const int m = t & (kTb - 1), q = t / kTb;  // 4 quarters of the 64 columns
    double    s = 0.0;
#pragma unroll
    for(int k = 0; k < kTb / 4; ++k) s = fma(S.T[m][q * (kTb / 4) + k], S.tmp[q * (kTb / 4) + k], s);
    S.red[q][m] = s;
  }
  __syncthreads();
  if(t < kb) {
    X[r0 + t] = (S.red[0][t] + S.red[1][t]) + (S.red[2][t] + S.red[3][t]);
    __threadfence();
  }
  __syncthreads();
  if(t == 0) st_release_gpu(flags + bi, 1);
}

// ---- U X = Y for up to kNr right-hand sides per launch ----
//
// trsv_kernel's structure with a kTb x kNr block of unknowns per row block:
// CTA k (ticket order) owns row block bi = nblk - 1 - k and walks its row
// panel bottom-up.  Each 64 x 64 tile of U is staged in shared memory by
// asynchronous copies (two buffers: the next tile lands while the current one
// is used) beside the published block x_j, and every warp accumulates
// U[bi, j] x_j for its own kNr / 8 right-hand sides (lane = rows 2 lane and
// 2 lane + 1), so each element of U crosses HBM once and feeds kNr FMAs.
// Then x_bi = U_ii^-1 (y_bi - sum), with U_ii inverted while the first tile
// loads.  Waits are bounded (status site 42).  X may alias Y: block bi of Y is
// read only by its own CTA, before that CTA writes block bi of X.
constexpr int kNr        = 32;                // right-hand sides per launch
constexpr int kNrPerWarp = kNr / kTrsvWarps;  // 4
constexpr int kTrsmSite  = 42;

struct TrsmSmem {
  double U[2][kTb][kTb];      // staged tiles, [column][row]
  double X[2][kTb][kNr + 2];  // the staged tile's x_j, [row of block j][rhs]
  double T[kTb][kTb + 1];     // U_ii, then U_ii^-1
  double R[kTb][kNr + 1];     // y_bi - sum_j U_ij x_j, [row][rhs]
  int    ticket;
};

HPLB_DEV void cp_async16(void* dst, const void* src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(bytes)
               : "memory");
}
HPLB_DEV void cp_async8(void* dst, const void* src, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(bytes)
               : "memory");
}

// Copies of the tile rows r0 .. r0 + kb, columns c0 .. c0 + kc of A into U
// (zeros outside), as one commit group.  VEC: 16-byte copies of row pairs (A
// 16-byte aligned, ld even); else 8-byte copies.
template <bool VEC>
HPLB_DEV void stage_tile(double (*U)[kTb], const double* A, int64_t ld, int r0, int kb, int c0,
                         int kc) {
  if(VEC) {
    for(int id = threadIdx.x; id < kTb * kTb / 2; id += kTrsvThreads) {
      const int     c = id / (kTb / 2), p = id % (kTb / 2);
      const int     rows = c < kc ? min(2, max(0, kb - 2 * p)) : 0;
      const double* src  = rows ? A + (size_t)(r0 + 2 * p) + (size_t)(c0 + c) * (size_t)ld : A;
      cp_async16(&U[c][2 * p], src, 8 * rows);
    }
  } else {
    for(int id = threadIdx.x; id < kTb * kTb; id += kTrsvThreads) {
      const int  c = id / kTb, r = id % kTb;
      const bool in = c < kc && r < kb;
      cp_async8(&U[c][r], in ? A + (size_t)(r0 + r) + (size_t)(c0 + c) * (size_t)ld : A,
                in ? 8 : 0);
    }
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <bool VEC>
__global__ void __launch_bounds__(kTrsvThreads, 1)
trsm_upper_kernel(const double* __restrict__ A, int64_t ld, int n, int nrhs, const double* Y,
                  int64_t ldy, double* X, int64_t ldx, int* flags, int* status) {
  extern __shared__ __align__(16) unsigned char trsm_smem_raw[];
  TrsmSmem& S    = *reinterpret_cast<TrsmSmem*>(trsm_smem_raw);
  const int nblk = (n + kTb - 1) / kTb;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if(t == 0) S.ticket = atomicAdd(flags + nblk, 1);
  __syncthreads();
  const int bi = nblk - 1 - S.ticket;
  const int r0 = bi * kTb;
  const int kb = min(kTb, n - r0);
  const int q0 = warp * kNrPerWarp;  // this warp's right-hand sides

  int j = nblk - 1;
  if(j > bi) stage_tile<VEC>(S.U[j & 1], A, ld, r0, kb, j * kTb, min(kTb, n - j * kTb));

  // Diagonal block (identity beyond kb), inverted while the first tile lands.
  for(int idx = t; idx < kTb * kTb; idx += kTrsvThreads) {
    const int c = idx / kTb, r = idx % kTb;
    double    v = (r == c) ? 1.0 : 0.0;
    if(r < kb && c < kb) v = r <= c ? A[(size_t)(r0 + r) + (size_t)(r0 + c) * (size_t)ld] : 0.0;
    S.T[r][c] = v;
  }
  __syncthreads();
  invert_upper(S.T);

  double acc[2][kNrPerWarp];
#pragma unroll
  for(int h = 0; h < 2; ++h)
#pragma unroll
    for(int k = 0; k < kNrPerWarp; ++k) acc[h][k] = 0.0;
  bool alive = true;
  for(; j > bi; --j) {
    const int b  = j & 1;
    const int kc = min(kTb, n - j * kTb);
    if(alive) alive = wait_flag(flags + j, status, kTrsmSite);
    for(int id = t; id < kTb * kNr; id += kTrsvThreads) {
      const int r = id % kTb, q = id / kTb;
      S.X[b][r][q] =
          (r < kc && q < nrhs) ? __ldcg(X + (size_t)(j * kTb + r) + (size_t)q * (size_t)ldx) : 0.0;
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");  // this thread's copies of tile j
    __syncthreads();  // everyone's, and the other buffers are no longer read
    if(j - 1 > bi) stage_tile<VEC>(S.U[b ^ 1], A, ld, r0, kb, (j - 1) * kTb, kTb);
#pragma unroll 4
    for(int c = 0; c < kTb; ++c) {
      const double2 u   = *reinterpret_cast<const double2*>(&S.U[b][c][2 * lane]);
      const double2 x01 = *reinterpret_cast<const double2*>(&S.X[b][c][q0]);
      const double2 x23 = *reinterpret_cast<const double2*>(&S.X[b][c][q0 + 2]);
      acc[0][0] = fma(u.x, x01.x, acc[0][0]);
      acc[0][1] = fma(u.x, x01.y, acc[0][1]);
      acc[0][2] = fma(u.x, x23.x, acc[0][2]);
      acc[0][3] = fma(u.x, x23.y, acc[0][3]);
      acc[1][0] = fma(u.y, x01.x, acc[1][0]);
      acc[1][1] = fma(u.y, x01.y, acc[1][1]);
      acc[1][2] = fma(u.y, x23.x, acc[1][2]);
      acc[1][3] = fma(u.y, x23.y, acc[1][3]);
    }
  }

  // R = y_bi - sum, then x_bi = U_ii^-1 R (lane = rows lane and lane + 32).
#pragma unroll
  for(int h = 0; h < 2; ++h)
#pragma unroll
    for(int k = 0; k < kNrPerWarp; ++k) {
      const int    r = 2 * lane + h, q = q0 + k;
      const double y = (r < kb && q < nrhs) ? Y[(size_t)(r0 + r) + (size_t)q * (size_t)ldy] : 0.0;
      S.R[r][q]      = y - acc[h][k];
    }
  __syncthreads();
#pragma unroll
  for(int h = 0; h < 2; ++h) {
    const int r = lane + 32 * h;
    double    x[kNrPerWarp];
#pragma unroll
    for(int k = 0; k < kNrPerWarp; ++k) x[k] = 0.0;
    for(int m = r; m < kTb; ++m) {
      const double tv = S.T[r][m];
#pragma unroll
      for(int k = 0; k < kNrPerWarp; ++k) x[k] = fma(tv, S.R[m][q0 + k], x[k]);
    }
#pragma unroll
    for(int k = 0; k < kNrPerWarp; ++k)
      if(r < kb && q0 + k < nrhs) X[(size_t)(r0 + r) + (size_t)(q0 + k) * (size_t)ldx] = x[k];
  }
  __threadfence();
  __syncthreads();
  if(t == 0) st_release_gpu(flags + bi, 1);
}

// z[r] += sum_c U[r, c] x[c] for r < m, c < k: a thread per row (coalesced
// down each column), x staged in shared memory in chunks of 1024.
__global__ void __launch_bounds__(256)
gemv_acc_kernel(int m, int k, const double* __restrict__ U, int64_t ld,
                const double* __restrict__ x, double* __restrict__ z) {
  __shared__ double xs[1024];
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  double    acc = 0.0;
  for(int c0 = 0; c0 < k; c0 += 1024) {
    const int kc = min(1024, k - c0);
    __syncthreads();
    for(int i = threadIdx.x; i < kc; i += blockDim.x) xs[i] = x[c0 + i];
    __syncthreads();
    if(r < m) {
      const double* u = U + (size_t)r + (size_t)c0 * (size_t)ld;
#pragma unroll 8
      for(int c = 0; c < kc; ++c) acc = fma(u[(size_t)c * (size_t)ld], xs[c], acc);
    }
  }
  if(r < m) z[r] += acc;
}

__global__ void vsub_kernel(int n, const double* __restrict__ y, const double* __restrict__ s,
                            double* __restrict__ r) {
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    r[i] = y[i] - s[i];
}

}  // namespace

size_t trsv_flag_ints(int n) { return (size_t)(n + kTb - 1) / kTb + 1; }

cudaError_t launch_gemv_acc(int m, int k, const double* U, int64_t ld, const double* x,
                            double* z, cudaStream_t stream) {
  if(m <= 0 || k <= 0) return cudaSuccess;
  gemv_acc_kernel<<<(m + 255) / 256, 256, 0, stream>>>(m, k, U, ld, x, z);
  return cudaGetLastError();
}

cudaError_t launch_vsub(int n, const double* y, const double* s, double* r, cudaStream_t stream) {
  if(n <= 0) return cudaSuccess;
  vsub_kernel<<<(n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024, 256, 0, stream>>>(n, y, s, r);
  return cudaGetLastError();
}

cudaError_t launch_trsv(const double* A, int64_t ld, int n, double* X, int* flags, int* status,
                        cudaStream_t stream, int* launches) {
  return launch_trsv_y(A, ld, n, A + (size_t)n * (size_t)ld, X, flags, status, stream, launches);
}

cudaError_t launch_trsv_y(const double* A, int64_t ld, int n, const double* Y, double* X,
                          int* flags, int* status, cudaStream_t stream, int* launches) {
  if(n <= 0) return cudaSuccess;
  const int   nblk = (n + kTb - 1) / kTb;
  cudaError_t e    = cudaMemsetAsync(flags, 0, trsv_flag_ints(n) * sizeof(int), stream);
  if(e != cudaSuccess) return e;
  const bool vec = (reinterpret_cast<uintptr_t>(A) % 16 == 0) && (ld % 2 == 0);
  if(vec)
    trsv_kernel<true><<<nblk, kTrsvThreads, 0, stream>>>(A, ld, n, Y, X, flags, status);
  else
    trsv_kernel<false><<<nblk, kTrsvThreads, 0, stream>>>(A, ld, n, Y, X, flags, status);
  ++*launches;
  return cudaGetLastError();
}

cudaError_t launch_trsm_upper(const double* A, int64_t ld, int n, int nrhs, const double* Y,
                              int64_t ldy, double* X, int64_t ldx, int* flags, int* status,
                              cudaStream_t stream, int* launches) {
  if(n <= 0 || nrhs <= 0) return cudaSuccess;
  const int  nblk = (n + kTb - 1) / kTb;
  const bool vec  = (reinterpret_cast<uintptr_t>(A) % 16 == 0) && (ld % 2 == 0);
  static bool attr = false;
  if(!attr) {
    cudaError_t e = cudaFuncSetAttribute(trsm_upper_kernel<true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(TrsmSmem));
    if(e == cudaSuccess)
      e = cudaFuncSetAttribute(trsm_upper_kernel<false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TrsmSmem));
    if(e != cudaSuccess) return e;
    attr = true;
  }
  // One launch per group of kNr right-hand sides, each with fresh flags.
  for(int q = 0; q < nrhs; q += kNr) {
    const int   nr = std::min(kNr, nrhs - q);
    cudaError_t e  = cudaMemsetAsync(flags, 0, trsv_flag_ints(n) * sizeof(int), stream);
    if(e != cudaSuccess) return e;
    const double* Yq = Y + (size_t)q * (size_t)ldy;
    double*       Xq = X + (size_t)q * (size_t)ldx;
    if(vec)
      trsm_upper_kernel<true><<<nblk, kTrsvThreads, sizeof(TrsmSmem), stream>>>(
          A, ld, n, nr, Yq, ldy, Xq, ldx, flags, status);
    else
      trsm_upper_kernel<false><<<nblk, kTrsvThreads, sizeof(TrsmSmem), stream>>>(
          A, ld, n, nr, Yq, ldy, Xq, ldx, flags, status);
    ++*launches;
    e = cudaGetLastError();
    if(e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace hplb
