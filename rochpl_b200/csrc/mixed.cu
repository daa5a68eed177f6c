// Kernels of the mixed-precision solve (FP32 factors, 16-bit trailing update,
// GMRES iterative refinement in FP64).  No counterpart in the reference, which
// is FP64 only; the surrounding algorithm (panel recursion, pivoting, look-
// ahead order) is the same as the FP64 path.
//
//   f64_to_f32          W = fp32(A) for a stored FP64 [A|b]
//   pack_l / pack_u     L21 and U12 (FP32) to K-major BF16/FP16 with one
//                       power-of-two scale per 128-row / 256-column tile, so
//                       every tile uses the 16-bit range fully and FP16 cannot
//                       overflow; the GEMM epilogue multiplies the scales back.
//                       Optionally split into high and low 16-bit parts.
//   upper_flip_*        U11^-1 through the unit-lower inverse: with D = diag(U),
//                       U = D Ut and J the reversal, J Ut J is unit lower, so
//                       U^-1 = J (J Ut J)^-1 J D^-1
//   perm_vec, gemv_rows  the preconditioner M^-1 = U^-1 L^-1 P applied to an
//                       FP64 vector panel by panel (FP32 factors, FP64 sums)
//   dot / amax / axpy   deterministic FP64 vector kernels for GMRES
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "internal.h"

namespace hplb {

namespace {

__global__ void f64_to_f32_kernel(int m, int n, const double* __restrict__ A, int64_t lda,
                                  float* __restrict__ W, int64_t ldw) {
  for(int c = blockIdx.y; c < n; c += gridDim.y) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if(r < m) W[(size_t)r + (size_t)c * ldw] = (float)A[(size_t)r + (size_t)c * lda];
  }
}

HPLB_DEV float block_max_f(float v, float* sh) {
  for(int off = 16; off > 0; off >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, off));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if(lane == 0) sh[warp] = v;
  __syncthreads();
  v = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.f;
  if(warp == 0)
    for(int off = 16; off > 0; off >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, off));
  if(threadIdx.x == 0) sh[0] = v;
  __syncthreads();
  v = sh[0];
  __syncthreads();
  return v;
}

// Power-of-two scale s with max*s in [0.5, 1); the epilogue multiplies by 1/s.
HPLB_DEV void pow2_scale(float mx, float& s, float& inv) {
  if(!(mx > 0.f) || isinf(mx)) {
    s   = 1.f;
    inv = 1.f;
    return;
  }
  int e;
  frexpf(mx, &e);
  s   = ldexpf(1.f, -e);
  inv = ldexpf(1.f, e);
}

template <bool BF16>
HPLB_DEV unsigned short to16(float x) {
  if(BF16) return __bfloat16_as_ushort(__float2bfloat16_rn(x));
  return __half_as_ushort(__float2half_rn(x));
}
template <bool BF16>
HPLB_DEV float from16(unsigned short h) {
  if(BF16) return __bfloat162float(__ushort_as_bfloat16(h));
  return __half2float(__ushort_as_half(h));
}

// Writes x (already scaled) into the packed row.  With SPLIT the row holds
// three jb-wide segments, [hi | hi | lo] for L and [hi | lo | hi] for U, so a
// single GEMM over K = 3 jb computes Lhi Uhi + Lhi Ulo + Llo Uhi: the 16-bit
// rounding error of each operand is carried by its low part.
template <bool BF16, bool SPLIT, bool IS_L>
HPLB_DEV void put16(unsigned short* row, int k, int jb, float x) {
  const unsigned short hi = to16<BF16>(x);
  row[k] = hi;
  if(SPLIT) {
    const unsigned short lo = to16<BF16>(x - from16<BF16>(hi));
    row[jb + k]     = IS_L ? hi : lo;
    row[2 * jb + k] = IS_L ? lo : hi;
  }
}

// Eight consecutive values (already scaled) of one packed row, stored as one
// 16-byte vector per segment; VEC needs k and jb multiples of 8.
template <bool BF16, bool SPLIT, bool IS_L>
HPLB_DEV void put16x8(unsigned short* row, int k, int jb, const float (&x)[8]) {
  union {
    unsigned short h[8];
    uint4          v;
  } hi, lo;
#pragma unroll
  for(int i = 0; i < 8; ++i) {
    hi.h[i] = to16<BF16>(x[i]);
    lo.h[i] = SPLIT ? to16<BF16>(x[i] - from16<BF16>(hi.h[i])) : (unsigned short)0;
  }
  *reinterpret_cast<uint4*>(row + k) = hi.v;
  if(SPLIT) {
    *reinterpret_cast<uint4*>(row + jb + k)     = IS_L ? hi.v : lo.v;
    *reinterpret_cast<uint4*>(row + 2 * jb + k) = IS_L ? lo.v : hi.v;
  }
}

// L21 (m x jb, column-major, leading dimension ld) -> out (m x ldo row-major
// 16-bit), one 128-row tile per block: a max pass for the tile's scale, then
// 32-column chunks transposed through shared memory and stored 8 values (16
// bytes) at a time per segment.
template <bool BF16, bool SPLIT>
__global__ void __launch_bounds__(256)
pack_l_kernel(int m, int jb, const float* __restrict__ L, int64_t ld,
              unsigned short* __restrict__ out, int64_t ldo, float* __restrict__ sL, float sign) {
  __shared__ float tile[128][33];
  __shared__ float sh[32];
  const int r0 = blockIdx.x * 128;
  const int rr = threadIdx.x & 127, cq = threadIdx.x >> 7;
  float mx = 0.f;
  if(r0 + rr < m)
    for(int c = cq; c < jb; c += 2) mx = fmaxf(mx, fabsf(L[(size_t)(r0 + rr) + (size_t)c * ld]));
  mx = block_max_f(mx, sh);
  float s, inv;
  pow2_scale(mx, s, inv);
  if(threadIdx.x == 0) sL[blockIdx.x] = inv;
  s *= sign;
  const bool vec = (jb & 7) == 0;
  for(int cb = 0; cb < jb; cb += 32) {
    for(int c = cq; c < 32; c += 2)
      tile[rr][c] = (r0 + rr < m && cb + c < jb) ? L[(size_t)(r0 + rr) + (size_t)(cb + c) * ld]
                                                   : 0.f;
    __syncthreads();
    const int r = threadIdx.x >> 1, half = threadIdx.x & 1;
    if(r0 + r < m) {
      unsigned short* o = out + (size_t)(r0 + r) * ldo;
#pragma unroll
      for(int g8 = 0; g8 < 2; ++g8) {
        const int k = cb + half * 16 + g8 * 8;
        if(vec && k + 8 <= jb) {
          float x[8];
#pragma unroll
          for(int q = 0; q < 8; ++q) x[q] = tile[r][half * 16 + g8 * 8 + q] * s;
          put16x8<BF16, SPLIT, true>(o, k, jb, x);
        } else {
#pragma unroll
          for(int q = 0; q < 8; ++q)
            if(k + q < jb) put16<BF16, SPLIT, true>(o, k + q, jb, tile[r][half * 16 + g8 * 8 + q] * s);
        }
      }
    }
    __syncthreads();
  }
}

// U12 (jb x n, column-major, leading dimension ld) -> out (n x ldo row-major:
// column c's jb values contiguous), one 256-column tile per block of 1024
// threads: a max pass for the tile's scale, then the pack pass, both with
// float4 loads and 8-byte stores of four 16-bit values when jb, ld and U
// allow (VEC), else one value at a time.
template <bool BF16, bool SPLIT, bool VEC>
__global__ void __launch_bounds__(1024)
pack_u_kernel(int jb, int n, const float* __restrict__ U, int64_t ld,
              unsigned short* __restrict__ out, int64_t ldo, float* __restrict__ sU, float sign) {
  __shared__ float sh[32];
  const int c0 = blockIdx.x * 256;
  const int nc = min(256, n - c0);
  const int W  = VEC ? jb / 4 : jb;  // items per column
  float     mx = 0.f;
  for(int idx = threadIdx.x; idx < nc * W; idx += blockDim.x) {
    const int c = idx / W, k = idx - c * W;
    const float* col = U + (size_t)(c0 + c) * ld;
    if(VEC) {
      const float4 v = *reinterpret_cast<const float4*>(col + 4 * k);
      mx = fmaxf(mx, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
    } else {
      mx = fmaxf(mx, fabsf(col[k]));
    }
  }
  mx = block_max_f(mx, sh);
  float s, inv;
  pow2_scale(mx, s, inv);
  if(threadIdx.x == 0) sU[blockIdx.x] = inv;
  s *= sign;
  for(int idx = threadIdx.x; idx < nc * W; idx += blockDim.x) {
    const int c = idx / W, k = idx - c * W;
    const float*    col = U + (size_t)(c0 + c) * ld;
    unsigned short* o   = out + (size_t)(c0 + c) * ldo;
    if(VEC) {
      const float4 v = *reinterpret_cast<const float4*>(col + 4 * k);
      const float  x[4] = {v.x * s, v.y * s, v.z * s, v.w * s};
      union {
        unsigned short h[4];
        uint2          v;
      } hi, lo;
#pragma unroll
      for(int i = 0; i < 4; ++i) {
        hi.h[i] = to16<BF16>(x[i]);
        lo.h[i] = SPLIT ? to16<BF16>(x[i] - from16<BF16>(hi.h[i])) : (unsigned short)0;
      }
      *reinterpret_cast<uint2*>(o + 4 * k) = hi.v;
      if(SPLIT) {
        *reinterpret_cast<uint2*>(o + jb + 4 * k)     = lo.v;
        *reinterpret_cast<uint2*>(o + 2 * jb + 4 * k) = hi.v;
      }
    } else {
      put16<BF16, SPLIT, false>(o, k, jb, col[k] * s);
    }
  }
}

// Lf = J (D^-1 U) J for the jb x jb upper block U (leading dimension ld):
// unit lower, leading dimension jb.  d[i] = U(i, i).
template <typename T>
__global__ void upper_flip_in_kernel(int jb, const T* __restrict__ U, int64_t ld,
                                     T* __restrict__ Lf, T* __restrict__ d) {
  const int c = blockIdx.x;  // column of Lf
  for(int r = threadIdx.x; r < jb; r += blockDim.x) {
    const int ur = jb - 1 - r, uc = jb - 1 - c;
    T v = T(0);
    if(r >= c) v = U[(size_t)ur + (size_t)uc * ld] / U[(size_t)ur + (size_t)ur * ld];
    Lf[(size_t)r + (size_t)c * jb] = v;
  }
  if(c == 0)
    for(int i = threadIdx.x; i < jb; i += blockDim.x) d[i] = U[(size_t)i + (size_t)i * ld];
}

// Uinv = J Lfinv J D^-1 (all jb x jb, leading dimension jb).
template <typename T>
__global__ void upper_flip_out_kernel(int jb, const T* __restrict__ Lfinv,
                                      const T* __restrict__ d, T* __restrict__ Uinv) {
  const int c = blockIdx.x;
  for(int r = threadIdx.x; r < jb; r += blockDim.x)
    Uinv[(size_t)r + (size_t)c * jb] =
        (r <= c) ? Lfinv[(size_t)(jb - 1 - r) + (size_t)(jb - 1 - c) * jb] / d[c] : T(0);
}

// Apply a panel's row map to a vector: z[ia + x] <- z[ia + permU[x]] for the
// top jb rows, displaced top rows to their new rows.  One block; each thread
// handles at most 8 of the top rows.
__global__ void perm_vec_kernel(double* z, int ia, int jb, const int* __restrict__ permU) {
  extern __shared__ double top[];
  for(int x = threadIdx.x; x < jb; x += blockDim.x) top[x] = z[ia + x];
  __syncthreads();
  double v[8];
  int    nx = 0;
  for(int x = threadIdx.x; x < jb && nx < 8; x += blockDim.x, ++nx) {
    const int src = permU[x];
    v[nx] = src < jb ? top[src] : z[ia + src];
  }
  __syncthreads();
  for(int s = threadIdx.x; s < jb; s += blockDim.x) {
    const int dst = permU[jb + s];
    if(dst >= 0) z[ia + dst] = top[s];
  }
  nx = 0;
  for(int x = threadIdx.x; x < jb && nx < 8; x += blockDim.x, ++nx) z[ia + x] = v[nx];
}

// y = M x (SUB = false) or y -= M x (SUB = true) for an FP32 M (rows x cols,
// column-major) and FP64 x, y: 32 rows per block, the 8 warps on slices of the
// columns (lane = row, so each column's 32 rows are one 128-byte read), FP64
// accumulation, then a fixed-order sum of the 8 slices.  x and y must not
// overlap.
template <bool SUB>
__global__ void __launch_bounds__(256)
gemv_rows_kernel(int rows, int cols, const float* __restrict__ M, int64_t ld,
                 const double* __restrict__ x, double* __restrict__ y) {
  __shared__ double xs[512];
  __shared__ double part[8][33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r    = blockIdx.x * 32 + lane;
  double    acc  = 0.0;
  for(int c0 = 0; c0 < cols; c0 += 512) {
    const int nc = min(512, cols - c0);
    __syncthreads();
    for(int i = threadIdx.x; i < nc; i += 256) xs[i] = x[c0 + i];
    __syncthreads();
    const int cs = (nc + 7) / 8, a = warp * cs, b = min(nc, a + cs);
    if(r < rows) {
      const float* m = M + (size_t)r + (size_t)c0 * ld;
#pragma unroll 8
      for(int c = a; c < b; ++c) acc += (double)m[(size_t)c * ld] * xs[c];
    }
  }
  part[warp][lane] = acc;
  __syncthreads();
  if(warp == 0 && r < rows) {
    double t = 0.0;
#pragma unroll
    for(int w = 0; w < 8; ++w) t += part[w][lane];
    y[r] = SUB ? y[r] - t : t;
  }
}

// ---- FP64 vector kernels (fixed-order, deterministic reductions) ----
constexpr int kVecBlocks = 296;

__global__ void __launch_bounds__(256) dot_partial_kernel(int n, const double* __restrict__ a,
                                                          const double* __restrict__ b,
                                                          double* part) {
  __shared__ double sh[8];
  double s = 0.0;
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s += a[i] * b[i];
  for(int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if(threadIdx.x == 0) {
    double t = 0.0;
    for(int w = 0; w < 8; ++w) t += sh[w];
    part[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(256) amax_partial_kernel(int n, const double* __restrict__ a,
                                                           double* part) {
  __shared__ double sh[8];
  double s = 0.0;
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s = fmax(s, fabs(a[i]));
  for(int off = 16; off > 0; off >>= 1) s = fmax(s, __shfl_down_sync(0xffffffffu, s, off));
  if((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if(threadIdx.x == 0) {
    double t = 0.0;
    for(int w = 0; w < 8; ++w) t = fmax(t, sh[w]);
    part[blockIdx.x] = t;
  }
}

// MAXIMUM = true: out = max(part), else out = sum(part), in block order.
template <bool MAXIMUM>
__global__ void fold_kernel(int nb, const double* part, double* out) {
  if(threadIdx.x == 0 && blockIdx.x == 0) {
    double t = 0.0;
    for(int i = 0; i < nb; ++i) t = MAXIMUM ? fmax(t, part[i]) : t + part[i];
    *out = t;
  }
}

// Classical Gram-Schmidt pieces for GMRES: part[i * gridDim.x + b] = partial
// of V_i . w over the rows block b strides, for the k columns of V at once.
constexpr int kMdotBlocks = 128;

__global__ void __launch_bounds__(256)
mdot_partial_kernel(int n, int k, const double* __restrict__ V, int64_t ldv,
                    const double* __restrict__ w, double* part) {
  __shared__ double sh[8];
  const int i = blockIdx.y;
  const double* v = V + (size_t)i * ldv;
  double s = 0.0;
  for(int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    s += v[r] * w[r];
  for(int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if(threadIdx.x == 0) {
    double t = 0.0;
    for(int q = 0; q < 8; ++q) t += sh[q];
    part[(size_t)i * gridDim.x + blockIdx.x] = t;
  }
}

// out[i] = sum of part[i * nb .. i * nb + nb), one thread per i, block order.
__global__ void mfold_kernel(int k, int nb, const double* part, double* out) {
  const int i = threadIdx.x;
  if(i < k) {
    double t = 0.0;
    for(int b = 0; b < nb; ++b) t += part[(size_t)i * nb + b];
    out[i] = t;
  }
}

// w -= V h (k columns, h on the device); acc = h (add into the running sum).
__global__ void mgemv_sub_kernel(int n, int k, const double* __restrict__ V, int64_t ldv,
                                 const double* __restrict__ h, double* __restrict__ w,
                                 double* acc) {
  __shared__ double hs[64];
  for(int i = threadIdx.x; i < k; i += blockDim.x) hs[i] = h[i];
  __syncthreads();
  if(acc && blockIdx.x == 0)
    for(int i = threadIdx.x; i < k; i += blockDim.x) acc[i] += hs[i];
  for(int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    double t = w[r];
    for(int i = 0; i < k; ++i) t -= hs[i] * V[(size_t)i * ldv + r];
    w[r] = t;
  }
}

__global__ void axpy_kernel(int n, double a, const double* __restrict__ x, double* y) {
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] += a * x[i];
}

__global__ void scal_copy_kernel(int n, double a, const double* __restrict__ x, double* y) {
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = a * x[i];
}

__global__ void sub_kernel(int n, const double* __restrict__ a, const double* __restrict__ b,
                           double* c) {
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    c[i] = a[i] - b[i];
}

}  // namespace

cudaError_t launch_f64_to_f32(int m, int n, const double* A, int64_t lda, float* W, int64_t ldw,
                              cudaStream_t st) {
  if(m <= 0 || n <= 0) return cudaSuccess;
  dim3 grid((m + 255) / 256, min(n, 65535));
  f64_to_f32_kernel<<<grid, 256, 0, st>>>(m, n, A, lda, W, ldw);
  return cudaGetLastError();
}

cudaError_t launch_pack_l(bool bf16, bool split, int m, int jb, const float* L, int64_t ld,
                          void* out, int64_t ldo, float* sL, cudaStream_t st, float sign) {
  if(m <= 0 || jb <= 0) return cudaSuccess;
  if(ldo % 8) return cudaErrorInvalidValue;  // 16-byte rows for the vector stores
  const int       grid = (m + 127) / 128;
  unsigned short* o    = (unsigned short*)out;
  if(bf16 && split)
    pack_l_kernel<true, true><<<grid, 256, 0, st>>>(m, jb, L, ld, o, ldo, sL, sign);
  else if(bf16)
    pack_l_kernel<true, false><<<grid, 256, 0, st>>>(m, jb, L, ld, o, ldo, sL, sign);
  else if(split)
    pack_l_kernel<false, true><<<grid, 256, 0, st>>>(m, jb, L, ld, o, ldo, sL, sign);
  else
    pack_l_kernel<false, false><<<grid, 256, 0, st>>>(m, jb, L, ld, o, ldo, sL, sign);
  return cudaGetLastError();
}

template <bool BF16, bool SPLIT>
static void pack_u_any(bool vec, int grid, int jb, int n, const float* U, int64_t ld,
                       unsigned short* o, int64_t ldo, float* sU, float sign, cudaStream_t st) {
  if(vec)
    pack_u_kernel<BF16, SPLIT, true><<<grid, 1024, 0, st>>>(jb, n, U, ld, o, ldo, sU, sign);
  else
    pack_u_kernel<BF16, SPLIT, false><<<grid, 1024, 0, st>>>(jb, n, U, ld, o, ldo, sU, sign);
}

cudaError_t launch_pack_u(bool bf16, bool split, int jb, int n, const float* U, int64_t ld,
                          void* out, int64_t ldo, float* sU, cudaStream_t st, float sign) {
  if(n <= 0 || jb <= 0) return cudaSuccess;
  const int       grid = (n + 255) / 256;
  unsigned short* o    = (unsigned short*)out;
  const bool vec = (jb % 4 == 0) && (ld % 4 == 0) && ((uintptr_t)U % 16 == 0) && (ldo % 4 == 0) &&
                   ((uintptr_t)out % 16 == 0);
  if(bf16 && split)
    pack_u_any<true, true>(vec, grid, jb, n, U, ld, o, ldo, sU, sign, st);
  else if(bf16)
    pack_u_any<true, false>(vec, grid, jb, n, U, ld, o, ldo, sU, sign, st);
  else if(split)
    pack_u_any<false, true>(vec, grid, jb, n, U, ld, o, ldo, sU, sign, st);
  else
    pack_u_any<false, false>(vec, grid, jb, n, U, ld, o, ldo, sU, sign, st);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_upper_inverse(int jb, const T* U, int64_t ld, T* Uinv, T* work, T* dinv_work,
                                 cudaStream_t st) {
  if(jb <= 0) return cudaSuccess;
  // work: jb*jb (flipped unit lower) + jb*jb (its inverse) + jb (diagonal).
  T* Lf    = work;
  T* Lfinv = work + (size_t)jb * jb;
  T* d     = Lfinv + (size_t)jb * jb;
  upper_flip_in_kernel<T><<<jb, 128, 0, st>>>(jb, U, ld, Lf, d);
  cudaError_t e = cudaGetLastError();
  if(e != cudaSuccess) return e;
  if((e = launch_diag_inv<T>(Lf, jb, 0, 0, jb, dinv_work, st)) != cudaSuccess) return e;
  if((e = launch_unit_lower_inverse<T>(Lf, jb, jb, dinv_work, Lfinv, jb, st)) != cudaSuccess)
    return e;
  upper_flip_out_kernel<T><<<jb, 128, 0, st>>>(jb, Lfinv, d, Uinv);
  return cudaGetLastError();
}
template cudaError_t launch_upper_inverse<float>(int, const float*, int64_t, float*, float*,
                                                 float*, cudaStream_t);
template cudaError_t launch_upper_inverse<double>(int, const double*, int64_t, double*, double*,
                                                  double*, cudaStream_t);

cudaError_t launch_perm_vec(double* z, int ia, int jb, const int* permU, cudaStream_t st) {
  if(jb <= 0) return cudaSuccess;
  if(jb > 8 * 256) return cudaErrorInvalidValue;
  perm_vec_kernel<<<1, 256, jb * sizeof(double), st>>>(z, ia, jb, permU);
  return cudaGetLastError();
}

cudaError_t launch_gemv_sub(int rows, int cols, const float* M, int64_t ld, const double* x,
                            double* y, cudaStream_t st) {
  if(rows <= 0 || cols <= 0) return cudaSuccess;
  gemv_rows_kernel<true><<<(rows + 31) / 32, 256, 0, st>>>(rows, cols, M, ld, x, y);
  return cudaGetLastError();
}

cudaError_t launch_gemv_set(int rows, int cols, const float* M, int64_t ld, const double* x,
                            double* y, cudaStream_t st) {
  if(rows <= 0) return cudaSuccess;
  gemv_rows_kernel<false><<<(rows + 31) / 32, 256, 0, st>>>(rows, cols, M, ld, x, y);
  return cudaGetLastError();
}

int vec_partials() { return kVecBlocks; }

cudaError_t launch_dot(int n, const double* a, const double* b, double* part, double* out,
                       cudaStream_t st) {
  dot_partial_kernel<<<kVecBlocks, 256, 0, st>>>(n, a, b, part);
  fold_kernel<false><<<1, 32, 0, st>>>(kVecBlocks, part, out);
  return cudaGetLastError();
}

cudaError_t launch_amax(int n, const double* a, double* part, double* out, cudaStream_t st) {
  amax_partial_kernel<<<kVecBlocks, 256, 0, st>>>(n, a, part);
  fold_kernel<true><<<1, 32, 0, st>>>(kVecBlocks, part, out);
  return cudaGetLastError();
}

size_t mdot_partials(int k) { return (size_t)k * kMdotBlocks; }

cudaError_t launch_mdot(int n, int k, const double* V, int64_t ldv, const double* w,
                        double* part, double* out, cudaStream_t st) {
  if(k <= 0) return cudaSuccess;
  if(k > 64) return cudaErrorInvalidValue;
  mdot_partial_kernel<<<dim3(kMdotBlocks, k), 256, 0, st>>>(n, k, V, ldv, w, part);
  mfold_kernel<<<1, 64, 0, st>>>(k, kMdotBlocks, part, out);
  return cudaGetLastError();
}

cudaError_t launch_mgemv_sub(int n, int k, const double* V, int64_t ldv, const double* h,
                             double* w, double* acc, cudaStream_t st) {
  if(k <= 0) return cudaSuccess;
  if(k > 64) return cudaErrorInvalidValue;
  mgemv_sub_kernel<<<kVecBlocks, 256, 0, st>>>(n, k, V, ldv, h, w, acc);
  return cudaGetLastError();
}

cudaError_t launch_axpy(int n, double a, const double* x, double* y, cudaStream_t st) {
  axpy_kernel<<<kVecBlocks, 256, 0, st>>>(n, a, x, y);
  return cudaGetLastError();
}

cudaError_t launch_scal_copy(int n, double a, const double* x, double* y, cudaStream_t st) {
  scal_copy_kernel<<<kVecBlocks, 256, 0, st>>>(n, a, x, y);
  return cudaGetLastError();
}

cudaError_t launch_sub(int n, const double* a, const double* b, double* c, cudaStream_t st) {
  sub_kernel<<<kVecBlocks, 256, 0, st>>>(n, a, b, c);
  return cudaGetLastError();
}

}  // namespace hplb
