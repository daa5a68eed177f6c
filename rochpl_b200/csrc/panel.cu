// Panel factorisation and row-interchange kernels of the single-process solve.
//
//  leaf_kernel      -- right-looking unblocked LU of an M x w leaf with partial
//                      pivoting, one persistent cooperative grid, pivot search by
//                      warp shuffles and one bounded grid barrier per column.
//                      Replaces pdpanrlT<1024> and its per-column host handshake
//                      (src/pfact/HPL_pdpanrlT_device.cpp:23-320, :455-463;
//                      src/pfact/HPL_pdmxswp.cpp:96-121): the pivot row travels
//                      through a device workspace instead of pinned host memory.
//  panel_swap_kernel-- the leaf's interchanges applied to the other columns of
//                      the panel (the reference swaps full panel rows inside the
//                      leaf, :200-214; the result is the same).
//  perm_kernel      -- ipiv -> permU (src/pgesv/HPL_pipid.cpp,
//                      src/panel/HPL_pdpanel_swapids.cpp:22-44) on the device.
//  diag_inv_kernel  -- inverses of the 32 x 32 unit-lower diagonal blocks of L11.
//  laswp_trsm_kernel-- fused row interchange (HPL_dlaswp00N) + unit-lower TRSM
//                      (rocblas_dtrsm, src/pgesv/HPL_pdupdateTT.cpp:95-106)
//                      over a block of columns held in shared memory.
#include <algorithm>
#include <cooperative_groups.h>
#include <cstdlib>
#include <cstring>

#include "common.cuh"
#include "internal.h"

namespace hplb {

namespace {

constexpr int kLeafThreads = 256;
constexpr int kTri         = 32;  // diagonal block size of the blocked TRSM

// (|v|, row) ordering for the pivot search: larger |v| wins, ties go to the
// lower row; row < 0 marks "no candidate".
HPLB_DEV bool better(double av, int ar, double bv, int br) {
  if(br < 0) return ar >= 0;
  if(ar < 0) return false;
  const double fa = fabs(av), fb = fabs(bv);
  if(fa > fb) return true;
  if(fa < fb) return false;
  return ar < br;
}

// Block-wide arg-max in the order of `better`; result valid in every thread.
// Two barriers: the first orders this call's writes of s_v / s_r after the
// previous call's reads.  With `separated` (every warp has passed a
// block-wide barrier -- a grid or cluster barrier counts -- since it last read
// the slots) the first is left out.
HPLB_DEV void block_argmax(double& v, int& r, double* s_v, int* s_r, bool separated = false) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  warp_argmax(v, r);
  if(!separated) __syncthreads();
  if(lane == 0) {
    s_v[warp] = v;
    s_r[warp] = r;
  }
  __syncthreads();
  const int nw = blockDim.x >> 5;
  v = lane < nw ? s_v[lane] : 0.0;
  r = lane < nw ? s_r[lane] : -1;
  warp_argmax(v, r);
}

template <typename T>
struct LeafParams {
  T*      A;
  int64_t ld;
  int     r0, end;  // leaf rows [r0, end)
  int     c0, w;    // leaf columns [c0, c0 + w), w <= kMaxLeaf
  int     rpb;      // rows owned per block
  int*    ipiv;     // ipiv[c] = global pivot row of column c
  double* cand;     // [2][grid][2 + w]  (value, row, leaf row values)
  double* cur;      // [2][w]            (the diagonal row's leaf values)
  int*    bar;      // grid barrier words
  int*    status;
  int     pc, pw;   // the panel [pc, pc + pw) the leaf belongs to (cluster leaf:
                    // it also swaps the panel's other columns)
};

// Publish this block's pivot candidate for leaf column k (its rows >= d) and,
// when it owns row d, the diagonal row itself.
template <typename T>
HPLB_DEV void leaf_publish(const LeafParams<T>& P, int k, int par, double* s_v, int* s_r) {
  const int d   = P.r0 + k;
  const int lo  = P.r0 + blockIdx.x * P.rpb;
  const int hi  = min(P.end, lo + P.rpb);
  const int beg = max(lo, d);
  const T* colk = P.A + (size_t)(P.c0 + k) * P.ld;
  double v = 0.0;
  int    r = -1;
  for(int i = beg + threadIdx.x; i < hi; i += blockDim.x) {
    const double a = colk[i];
    if(better(a, i, v, r)) {
      v = a;
      r = i;
    }
  }
  block_argmax(v, r, s_v, s_r);
  double* slot = P.cand + ((size_t)par * gridDim.x + blockIdx.x) * (2 + P.w);
  if(threadIdx.x == 0) {
    slot[0] = v;
    slot[1] = (double)r;
  }
  if(r >= 0)
    for(int c = threadIdx.x; c < P.w; c += blockDim.x)
      slot[2 + c] = P.A[(size_t)r + (size_t)(P.c0 + c) * P.ld];
  if(d >= lo && d < hi)
    for(int c = threadIdx.x; c < P.w; c += blockDim.x)
      P.cur[par * P.w + c] = P.A[(size_t)d + (size_t)(P.c0 + c) * P.ld];
}

template <typename T>
__global__ void __launch_bounds__(kLeafThreads) leaf_kernel(LeafParams<T> P) {
  __shared__ double s_v[32];
  __shared__ int    s_r[32];
  __shared__ double s_u[kMaxLeaf];    // pivot row (leaf columns)
  __shared__ double s_cur[kMaxLeaf];  // old diagonal row
  __shared__ double s_piv;
  __shared__ int    s_p;

  const int G   = gridDim.x;
  const int lo  = P.r0 + blockIdx.x * P.rpb;
  const int hi  = min(P.end, lo + P.rpb);
  const size_t ld = (size_t)P.ld;

  leaf_publish(P, 0, 0, s_v, s_r);
  if(!grid_sync(P.bar, G, 1, P.status, 11)) return;

  for(int k = 0; k < P.w; ++k) {
    const int par = k & 1;
    const int c   = P.c0 + k;
    const int d   = P.r0 + k;
    // Global pivot: warp 0 scans every block's candidate.
    if(threadIdx.x < 32) {
      double v = 0.0;
      int    r = -1, slot = -1;
      for(int b = threadIdx.x; b < G; b += 32) {
        const double* sl = P.cand + ((size_t)par * G + b) * (2 + P.w);
        const double  sv = __ldcg(sl);
        const int     sr = (int)__ldcg(sl + 1);
        if(better(sv, sr, v, r)) {
          v = sv;
          r = sr;
          slot = b;
        }
      }
#pragma unroll
      for(int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, v, off);
        const int    orow = __shfl_down_sync(0xffffffffu, r, off);
        const int    os = __shfl_down_sync(0xffffffffu, slot, off);
        if(better(ov, orow, v, r)) {
          v = ov;
          r = orow;
          slot = os;
        }
      }
      slot = __shfl_sync(0xffffffffu, slot, 0);
      if(slot < 0) {  // unreachable while the leaf has rows >= d; keeps reads in bounds
        slot = 0;
        v    = 0.0;
        r    = d;
      }
      if(threadIdx.x == 0) {
        s_piv = v;
        s_p   = r;
      }
      const double* sl = P.cand + ((size_t)par * G + slot) * (2 + P.w);
      for(int cc = threadIdx.x; cc < P.w; cc += 32) {
        s_u[cc]   = __ldcg(sl + 2 + cc);
        s_cur[cc] = __ldcg(P.cur + par * P.w + cc);
      }
    }
    __syncthreads();
    const T   piv = (T)s_piv;
    const int p   = s_p;
    if(blockIdx.x == 0 && threadIdx.x == 0) {
      P.ipiv[c] = p;
      if(piv == (T)0) record_info(P.status, c + 1);
    }
    // Interchange rows d and p over the leaf columns.
    if(p != d && p >= lo && p < hi)
      for(int cc = threadIdx.x; cc < P.w; cc += blockDim.x)
        P.A[(size_t)p + (size_t)(P.c0 + cc) * ld] = (T)s_cur[cc];
    if(d >= lo && d < hi)
      for(int cc = threadIdx.x; cc < P.w; cc += blockDim.x)
        P.A[(size_t)d + (size_t)(P.c0 + cc) * ld] = (T)s_u[cc];
    __syncthreads();
    // Scale column c below the diagonal (division, as the reference does at
    // src/pfact/HPL_pdpanrlT_device.cpp:232) and apply the rank-1 update to the
    // remaining leaf columns.
    T* colc = P.A + (size_t)c * ld;
    for(int i = max(lo, d + 1) + threadIdx.x; i < hi; i += blockDim.x) {
      const T l = colc[i] / piv;
      colc[i]   = l;
      for(int cc = k + 1; cc < P.w; ++cc) {
        T* a = P.A + (size_t)i + (size_t)(P.c0 + cc) * ld;
        *a   = *a - l * (T)s_u[cc];
      }
    }
    if(k + 1 == P.w) break;
    __syncthreads();
    leaf_publish(P, k + 1, par ^ 1, s_v, s_r);
    if(!grid_sync(P.bar, G, k + 2, P.status, 12)) return;
  }
}

// Leaf with the block's rows resident in shared memory (w <= kSmemLeafW).
//
// Each block loads its rpb x w slice of the leaf once, runs all w column steps
// on it, and writes it back once; only the pivot candidates, the pivot row and
// the old diagonal row cross global memory (the same exchange and bounded grid
// barrier as leaf_kernel).  The arithmetic is that of leaf_kernel, operation
// for operation (division by the pivot, then a_cc - l * u_cc per entry), so
// the two kernels give identical bits; this one just never waits on L2
// latency inside a column step.  The slice is column-major in shared memory,
// sm[cc * rpb + i], so the pivot search and the update read consecutive words.
constexpr int kSmemLeafW       = 32;
constexpr int kSmemLeafThreads = 256;

template <typename T>
HPLB_DEV void leaf_smem_publish(const LeafParams<T>& P, const T* sm, int lo, int nr, int k,
                                int par, double* s_v, int* s_r) {
  const int d   = P.r0 + k;
  const T*  col = sm + (size_t)k * P.rpb;
  double    v   = 0.0;
  int       r   = -1;
  for(int i = max(0, d - lo) + threadIdx.x; i < nr; i += blockDim.x) {
    const double a = col[i];
    if(better(a, lo + i, v, r)) {
      v = a;
      r = lo + i;
    }
  }
  block_argmax(v, r, s_v, s_r);
  double* slot = P.cand + ((size_t)par * gridDim.x + blockIdx.x) * (2 + P.w);
  if(threadIdx.x == 0) {
    slot[0] = v;
    slot[1] = (double)r;
  }
  if(r >= 0)
    for(int c = threadIdx.x; c < P.w; c += blockDim.x)
      slot[2 + c] = sm[(size_t)c * P.rpb + (r - lo)];
  if(d >= lo && d < lo + nr)
    for(int c = threadIdx.x; c < P.w; c += blockDim.x)
      P.cur[par * P.w + c] = sm[(size_t)c * P.rpb + (d - lo)];
}

template <typename T>
__global__ void __launch_bounds__(kSmemLeafThreads) leaf_smem_kernel(LeafParams<T> P) {
  extern __shared__ __align__(16) unsigned char leaf_raw[];
  T* sm = reinterpret_cast<T*>(leaf_raw);
  __shared__ double s_v[32];
  __shared__ int    s_r[32];
  __shared__ double s_u[kSmemLeafW];
  __shared__ double s_cur[kSmemLeafW];
  __shared__ double s_piv;
  __shared__ int    s_p;

  const int    G  = gridDim.x;
  const int    R  = P.rpb;
  const int    lo = P.r0 + blockIdx.x * R;
  const int    nr = max(0, min(P.end, lo + R) - lo);
  const size_t ld = (size_t)P.ld;

  for(int c = 0; c < P.w; ++c)
    for(int i = threadIdx.x; i < nr; i += blockDim.x)
      sm[(size_t)c * R + i] = P.A[(size_t)(lo + i) + (size_t)(P.c0 + c) * ld];
  __syncthreads();

  leaf_smem_publish(P, sm, lo, nr, 0, 0, s_v, s_r);
  if(!grid_sync(P.bar, G, 1, P.status, 13)) return;

  for(int k = 0; k < P.w; ++k) {
    const int par = k & 1;
    const int d   = P.r0 + k;
    if(threadIdx.x < 32) {
      double v = 0.0;
      int    r = -1, slot = -1;
      for(int b = threadIdx.x; b < G; b += 32) {
        const double* sl = P.cand + ((size_t)par * G + b) * (2 + P.w);
        const double  sv = __ldcg(sl);
        const int     sr = (int)__ldcg(sl + 1);
        if(better(sv, sr, v, r)) {
          v    = sv;
          r    = sr;
          slot = b;
        }
      }
#pragma unroll
      for(int off = 16; off > 0; off >>= 1) {
        const double ov   = __shfl_down_sync(0xffffffffu, v, off);
        const int    orow = __shfl_down_sync(0xffffffffu, r, off);
        const int    os   = __shfl_down_sync(0xffffffffu, slot, off);
        if(better(ov, orow, v, r)) {
          v    = ov;
          r    = orow;
          slot = os;
        }
      }
      slot = __shfl_sync(0xffffffffu, slot, 0);
      if(slot < 0) {  // unreachable while the leaf has rows >= d; keeps reads in bounds
        slot = 0;
        v    = 0.0;
        r    = d;
      }
      if(threadIdx.x == 0) {
        s_piv = v;
        s_p   = r;
      }
      const double* sl = P.cand + ((size_t)par * G + slot) * (2 + P.w);
      if(threadIdx.x < P.w) {
        s_u[threadIdx.x]   = __ldcg(sl + 2 + threadIdx.x);
        s_cur[threadIdx.x] = __ldcg(P.cur + par * P.w + threadIdx.x);
      }
    }
    __syncthreads();
    const T   piv = (T)s_piv;
    const int p   = s_p;
    if(blockIdx.x == 0 && threadIdx.x == 0) {
      P.ipiv[P.c0 + k] = p;
      if(piv == (T)0) record_info(P.status, P.c0 + k + 1);
    }
    if(p != d && p >= lo && p < lo + nr && threadIdx.x < P.w)
      sm[(size_t)threadIdx.x * R + (p - lo)] = (T)s_cur[threadIdx.x];
    if(d >= lo && d < lo + nr && threadIdx.x < P.w)
      sm[(size_t)threadIdx.x * R + (d - lo)] = (T)s_u[threadIdx.x];
    __syncthreads();
    // Scale the column below the diagonal and update the remaining columns.
    // The row's values are loaded before any is stored, so the loads issue
    // back to back.
    for(int i = max(0, d + 1 - lo) + threadIdx.x; i < nr; i += blockDim.x) {
      const T l = sm[(size_t)k * R + i] / piv;
      sm[(size_t)k * R + i] = l;
      T x[kSmemLeafW];
#pragma unroll
      for(int cc = 0; cc < kSmemLeafW; ++cc)
        if(cc > k && cc < P.w) x[cc] = sm[(size_t)cc * R + i];
#pragma unroll
      for(int cc = 0; cc < kSmemLeafW; ++cc)
        if(cc > k && cc < P.w) sm[(size_t)cc * R + i] = x[cc] - l * (T)s_u[cc];
    }
    if(k + 1 == P.w) break;
    __syncthreads();
    leaf_smem_publish(P, sm, lo, nr, k + 1, par ^ 1, s_v, s_r);
    if(!grid_sync(P.bar, G, k + 2, P.status, 14)) return;
  }
  __syncthreads();
  for(int c = 0; c < P.w; ++c)
    for(int i = threadIdx.x; i < nr; i += blockDim.x)
      P.A[(size_t)(lo + i) + (size_t)(P.c0 + c) * ld] = sm[(size_t)c * R + i];
}

// Leaf with every row in registers: thread t of block b owns rows
// r0 + b * rpb + t + q * blockDim.x (q < RPT) across all w <= 32 leaf
// columns.  The column loop is a run-time loop (not unrolled: an unrolled
// 32-step body is about a megabyte of code, fetched from L2 once per column);
// its body reaches column k of the row registers by selects and updates
// columns k+1 .. w-1 by predicated FMAs, so the rows stay in registers.  A
// column step costs the pivot search, one bounded grid barrier and two
// 32-word reads (pivot row, old diagonal row).  Arithmetic identical to
// leaf_kernel (division by the pivot, a_cc - l * u_cc), hence identical bits.
constexpr int kRegLeafW       = 32;
constexpr int kRegLeafThreads = 256;

template <typename T, int N>
HPLB_DEV T pick_col(const T (&x)[N], int c) {
  if constexpr(N == 32) {
    // A select tree on the bits of c: depth 5 instead of a 31-long chain.
    T a[16], b[8], e[4], f[2];
#pragma unroll
    for(int i = 0; i < 16; ++i) a[i] = (c & 1) ? x[2 * i + 1] : x[2 * i];
#pragma unroll
    for(int i = 0; i < 8; ++i) b[i] = (c & 2) ? a[2 * i + 1] : a[2 * i];
#pragma unroll
    for(int i = 0; i < 4; ++i) e[i] = (c & 4) ? b[2 * i + 1] : b[2 * i];
#pragma unroll
    for(int i = 0; i < 2; ++i) f[i] = (c & 8) ? e[2 * i + 1] : e[2 * i];
    return (c & 16) ? f[1] : f[0];
  } else {
    T s = x[0];
#pragma unroll
    for(int q = 1; q < N; ++q) s = (q == c) ? x[q] : s;
    return s;
  }
}

// One column step's work on the rows a thread holds, shared by the register
// leaves.  d = r0 + k is the diagonal row, p the pivot row; s_u holds the
// pivot row's w values, s_uz the same with the entries of columns <= k set
// to zero, s_cur the old diagonal row.
//   * the interchange: only the warps that hold row d or row p take the branch;
//   * below the diagonal: l = a_k / pivot, then a_c -= l u_c for c > k.  With
//     a finite l every column is updated against s_uz (columns <= k see a zero
//     u and keep their value), one select per entry putting l in column k;
//     a non-finite l (a zero pivot) keeps the predicated form, so columns
//     before k stay untouched exactly as in the other leaves.
template <typename T, int RPT>
HPLB_DEV void leaf_rows_step(T (&x)[RPT][kRegLeafW], const int (&row)[RPT], int k, int d, int p,
                             T piv, const double* s_u, const double* s_uz, const double* s_cur) {
  bool touch = false;
#pragma unroll
  for(int q = 0; q < RPT; ++q) touch |= (row[q] == d) | (row[q] == p);
  if(__any_sync(0xffffffffu, touch)) {
#pragma unroll
    for(int q = 0; q < RPT; ++q) {
      if(row[q] == d) {
#pragma unroll
        for(int c = 0; c < kRegLeafW; ++c) x[q][c] = (T)s_u[c];
      } else if(row[q] == p) {
#pragma unroll
        for(int c = 0; c < kRegLeafW; ++c) x[q][c] = (T)s_cur[c];
      }
    }
  }
#pragma unroll
  for(int q = 0; q < RPT; ++q) {
    if(row[q] > d) {
      const T l = pick_col(x[q], k) / piv;
      if(isfinite((double)l)) {
#pragma unroll
        for(int c = 0; c < kRegLeafW; ++c) {
          const T nx = x[q][c] - l * (T)s_uz[c];
          x[q][c]    = (c == k) ? l : nx;
        }
      } else {
#pragma unroll
        for(int c = 0; c < kRegLeafW; ++c) {
          if(c == k)
            x[q][c] = l;
          else if(c > k)
            x[q][c] = x[q][c] - l * (T)s_u[c];
        }
      }
    }
  }
}

// Publish the rows a column step needs from this block: its candidate row
// (to slot, w values) and, on the owner, the diagonal row (to cur).  Only the
// warps holding one of the two take the branch.
template <typename T, int RPT>
HPLB_DEV void leaf_rows_publish(const T (&x)[RPT][kRegLeafW], const int (&row)[RPT], int r, int d,
                                int w, double* slot, double* cur) {
  bool touch = false;
#pragma unroll
  for(int q = 0; q < RPT; ++q) touch |= (r >= 0 && row[q] == r) | (row[q] == d);
  if(!__any_sync(0xffffffffu, touch)) return;
#pragma unroll
  for(int q = 0; q < RPT; ++q) {
    if(r >= 0 && row[q] == r)
#pragma unroll
      for(int c = 0; c < kRegLeafW; ++c)
        if(c < w) slot[c] = (double)x[q][c];
    if(row[q] == d)
#pragma unroll
      for(int c = 0; c < kRegLeafW; ++c)
        if(c < w) cur[c] = (double)x[q][c];
  }
}

template <typename T, int RPT>
__global__ void __launch_bounds__(kRegLeafThreads, 1) leaf_reg_kernel(LeafParams<T> P) {
  __shared__ double s_v[32];
  __shared__ int    s_r[32];
  __shared__ double s_u[kRegLeafW];
  __shared__ double s_uz[kRegLeafW];
  __shared__ double s_cur[kRegLeafW];
  __shared__ double s_piv;
  __shared__ int    s_p;

  const int    G    = gridDim.x;
  const int    lane = threadIdx.x & 31;
  const int    lo   = P.r0 + blockIdx.x * P.rpb;
  const size_t ld   = (size_t)P.ld;
  const int    w    = P.w;
  const int    sw   = (3 + w) & ~1;  // slot stride: 2 + w rounded up to even (16-byte pairs)

  T   x[RPT][kRegLeafW];
  int row[RPT];
#pragma unroll
  for(int q = 0; q < RPT; ++q) {
    row[q]         = lo + threadIdx.x + q * blockDim.x;
    const bool in  = row[q] < P.end && threadIdx.x + q * blockDim.x < P.rpb;
    if(!in) row[q] = -1;
#pragma unroll
    for(int c = 0; c < kRegLeafW; ++c)
      x[q][c] = (in && c < w) ? P.A[(size_t)row[q] + (size_t)(P.c0 + c) * ld] : (T)0;
  }

#pragma unroll 1
  for(int k = 0; k < w; ++k) {
    const int par = k & 1;
    const int d   = P.r0 + k;
    // This block's candidate among its rows >= d, and the rows it must publish.
    double v = 0.0;
    int    r = -1;
#pragma unroll
    for(int q = 0; q < RPT; ++q) {
      const double xk = (double)pick_col(x[q], k);
      if(row[q] >= d && better(xk, row[q], v, r)) {
        v = xk;
        r = row[q];
      }
    }
    block_argmax(v, r, s_v, s_r, true);  // the grid barrier separates the columns
    double* slot = P.cand + ((size_t)par * G + blockIdx.x) * sw;
    if(threadIdx.x == 0) *reinterpret_cast<double2*>(slot) = make_double2(v, (double)r);
    leaf_rows_publish(x, row, r, d, w, slot + 2, P.cur + par * w);
    if(!grid_sync(P.bar, G, k + 1, P.status, 15)) return;

    if(threadIdx.x < 32) {
      // Every block's (value, row) pair, all loads in flight before any
      // comparison; then the lane's best, then the warp's.
      constexpr int kHoist = 8;  // grids up to 256 blocks
      double2       cv[kHoist];
#pragma unroll
      for(int t = 0; t < kHoist; ++t) {
        const int b = lane + 32 * t;
        cv[t] = b < G ? __ldcg(reinterpret_cast<const double2*>(P.cand + ((size_t)par * G + b) * sw))
                      : make_double2(0.0, -1.0);
      }
      double bv = 0.0;
      int    br = -1, bs = -1;
#pragma unroll
      for(int t = 0; t < kHoist; ++t)
        if(better(cv[t].x, (int)cv[t].y, bv, br)) {
          bv = cv[t].x;
          br = (int)cv[t].y;
          bs = lane + 32 * t;
        }
      for(int b = lane + 32 * kHoist; b < G; b += 32) {
        const double2 c2 = __ldcg(reinterpret_cast<const double2*>(P.cand + ((size_t)par * G + b) * sw));
        if(better(c2.x, (int)c2.y, bv, br)) {
          bv = c2.x;
          br = (int)c2.y;
          bs = b;
        }
      }
      const int wl = warp_argmax(bv, br);
      bs           = __shfl_sync(0xffffffffu, bs, wl < 0 ? 0 : wl);
      if(wl < 0 || bs < 0) {  // unreachable while the leaf has rows >= d; keeps reads in bounds
        bs = 0;
        bv = 0.0;
        br = d;
      }
      if(threadIdx.x == 0) {
        s_piv = bv;
        s_p   = br;
      }
      const double* sl = P.cand + ((size_t)par * G + bs) * sw;
      if(threadIdx.x < w) {
        const double u     = __ldcg(sl + 2 + threadIdx.x);
        s_u[threadIdx.x]   = u;
        s_uz[threadIdx.x]  = (int)threadIdx.x > k ? u : 0.0;
        s_cur[threadIdx.x] = __ldcg(P.cur + par * w + threadIdx.x);
      }
    }
    __syncthreads();
    const T   piv = (T)s_piv;
    const int p   = s_p;
    if(blockIdx.x == 0 && threadIdx.x == 0) {
      P.ipiv[P.c0 + k] = p;
      if(piv == (T)0) record_info(P.status, P.c0 + k + 1);
    }
    leaf_rows_step(x, row, k, d, p, piv, s_u, s_uz, s_cur);
  }

#pragma unroll
  for(int q = 0; q < RPT; ++q)
    if(row[q] >= 0)
#pragma unroll
      for(int c = 0; c < kRegLeafW; ++c)
        if(c < w) P.A[(size_t)row[q] + (size_t)(P.c0 + c) * ld] = x[q][c];
}

// The register leaf on ONE thread-block cluster (up to 16 CTAs, one per SM,
// co-scheduled by the hardware): the rows stay in registers exactly as in
// leaf_reg_kernel and every column performs the same operations in the same
// order (hence the same bits), but the exchange per column is on chip:
//   * each CTA's candidate (value, row) and its candidate row's leaf values go
//     to its own shared memory, the diagonal row to its owner's, in one of two
//     buffers by column parity;
//   * one hardware cluster barrier (arrive.release / wait.acquire) replaces
//     the grid-wide atomic barrier;
//   * warp 0 of every CTA reads the G candidates, then the winning row and the
//     diagonal row, from the peers' shared memory (ld.shared::cluster).
// A CTA writes buffer k & 1 only after the barrier of column k - 1, which
// every peer reaches after its last read of buffer (k - 2) & 1, so one barrier
// per column suffices; a last barrier keeps every CTA resident until its
// peers' final reads are done.  No wait here is a spin on memory.
HPLB_DEV unsigned cluster_ctarank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
HPLB_DEV unsigned cluster_nctarank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
HPLB_DEV void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n"
               "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// A double in CTA `rank`'s shared memory at the offset of `local`.
HPLB_DEV double ld_peer(const double* local, unsigned rank) {
  uint32_t a = (uint32_t)__cvta_generic_to_shared(local), r;
  double   v;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(r) : "memory");
  return v;
}

constexpr int kClusterLeafMax = 16;  // CTAs per cluster at most (non-portable above 8)

template <typename T, int RPT>
__global__ void __launch_bounds__(kRegLeafThreads, 1) leaf_cluster_kernel(LeafParams<T> P) {
  __shared__ double s_v[32];
  __shared__ int    s_r[32];
  __shared__ double s_slot[2][2 + kRegLeafW];  // (value, row, candidate row) per parity
  __shared__ double s_diag[2][kRegLeafW];      // the diagonal row, on its owner
  __shared__ double s_u[kRegLeafW];
  __shared__ double s_uz[kRegLeafW];
  __shared__ double s_cur[kRegLeafW];
  __shared__ double s_piv;
  __shared__ int    s_p;
  __shared__ int    s_pv[kRegLeafW];  // the leaf's pivots, relative to r0
  __shared__ int    s_src[kRegLeafW], s_dst[kRegLeafW];

  const unsigned G    = cluster_nctarank();
  const unsigned me   = cluster_ctarank();
  const int      lane = threadIdx.x & 31;
  const int      lo   = P.r0 + (int)me * P.rpb;
  const size_t   ld   = (size_t)P.ld;
  const int      w    = P.w;

  T   x[RPT][kRegLeafW];
  int row[RPT];
#pragma unroll
  for(int q = 0; q < RPT; ++q) {
    row[q]         = lo + threadIdx.x + q * blockDim.x;
    const bool in  = row[q] < P.end && threadIdx.x + q * blockDim.x < P.rpb;
    if(!in) row[q] = -1;
#pragma unroll
    for(int c = 0; c < kRegLeafW; ++c)
      x[q][c] = (in && c < w) ? P.A[(size_t)row[q] + (size_t)(P.c0 + c) * ld] : (T)0;
  }

#pragma unroll 1
  for(int k = 0; k < w; ++k) {
    const int par = k & 1;
    const int d   = P.r0 + k;
    double v = 0.0;
    int    r = -1;
#pragma unroll
    for(int q = 0; q < RPT; ++q) {
      const double xk = (double)pick_col(x[q], k);
      if(row[q] >= d && better(xk, row[q], v, r)) {
        v = xk;
        r = row[q];
      }
    }
    block_argmax(v, r, s_v, s_r, true);  // the cluster barrier separates the columns
    if(threadIdx.x == 0) {
      s_slot[par][0] = v;
      s_slot[par][1] = (double)r;
    }
    leaf_rows_publish(x, row, r, d, w, &s_slot[par][2], &s_diag[par][0]);
    cluster_barrier();

    if(threadIdx.x < 32) {
      double bv = 0.0;
      int    br = -1;
      if(lane < (int)G) {
        bv = ld_peer(&s_slot[par][0], (unsigned)lane);
        br = (int)ld_peer(&s_slot[par][1], (unsigned)lane);
      }
      const int wl = warp_argmax(bv, br);
      int       bs = wl < 0 ? 0 : wl;  // the winning CTA
      if(wl < 0) {  // unreachable while the leaf has rows >= d; keeps reads in bounds
        bv = 0.0;
        br = d;
      }
      if(threadIdx.x == 0) {
        s_piv = bv;
        s_p   = br;
      }
      const unsigned owner = (unsigned)min((int)G - 1, (d - P.r0) / P.rpb);
      if(lane < w) {
        const double u = ld_peer(&s_slot[par][2 + lane], (unsigned)bs);
        s_u[lane]      = u;
        s_uz[lane]     = lane > k ? u : 0.0;
        s_cur[lane]    = ld_peer(&s_diag[par][lane], owner);
      }
    }
    __syncthreads();
    const T   piv = (T)s_piv;
    const int p   = s_p;
    if(me == 0 && threadIdx.x == 0) {
      P.ipiv[P.c0 + k] = p;
      if(piv == (T)0) record_info(P.status, P.c0 + k + 1);
    }
    if(threadIdx.x == 0) s_pv[k] = p - P.r0;
    leaf_rows_step(x, row, k, d, p, piv, s_u, s_uz, s_cur);
  }
  cluster_barrier();

#pragma unroll
  for(int q = 0; q < RPT; ++q)
    if(row[q] >= 0)
#pragma unroll
      for(int c = 0; c < kRegLeafW; ++c)
        if(c < w) P.A[(size_t)row[q] + (size_t)(P.c0 + c) * ld] = x[q][c];

  // The leaf's interchanges on the panel's other columns (the work of
  // panel_swap_kernel, which this leaf replaces): the interchange sequence
  // traced into a row map, then per column all reads before any write.  The
  // leaf's own columns are not touched here, so no ordering with the
  // write-back above is needed.
  const int ncols = P.pw - w;
  if(ncols <= 0) return;
  if(threadIdx.x < w) {
    const int xr = threadIdx.x;
    int       pos = xr;
    for(int i = w - 1; i >= 0; --i) {
      const int pp = s_pv[i];
      pos          = (pos == i) ? pp : (pos == pp ? i : pos);
    }
    s_src[xr] = pos;
    pos       = xr;
    for(int i = 0; i < w; ++i) {
      const int pp = s_pv[i];
      pos          = (pos == i) ? pp : (pos == pp ? i : pos);
    }
    s_dst[xr] = pos >= w ? pos : -1;
  }
  __syncthreads();
  // A warp per column, lane = row of the leaf's top block: the top rows'
  // writes are one contiguous segment, and every warp of the cluster takes
  // columns in turn.
  const int nwarp = (int)G * (int)(blockDim.x >> 5);
  for(int j = (int)me * (int)(blockDim.x >> 5) + (int)(threadIdx.x >> 5); j < ncols; j += nwarp) {
    const int col = (P.pc + j < P.c0) ? P.pc + j : P.pc + j + w;
    T*        a   = P.A + (size_t)col * ld + P.r0;
    T         v = (T)0, o = (T)0;
    const int dst = lane < w ? s_dst[lane] : -1;
    if(lane < w) {
      v = a[s_src[lane]];
      if(dst >= 0) o = a[lane];
    }
    __syncwarp();  // every read of the column before any write to it
    if(dst >= 0) a[dst] = o;
    if(lane < w) a[lane] = v;
    __syncwarp();
  }
}

// Apply the w interchanges of leaf columns [c0, c0+w) to the panel columns
// outside the leaf.  For w <= 32 the interchange sequence is traced once per
// block into a row map (src[x]: the row whose value ends in row r0 + x;
// dst[x]: where the old row r0 + x ends when it leaves the top w rows, else
// -1), and a warp takes each column, lane = row of the top block: every read
// of the column before any write, the top rows written as one contiguous
// segment.  Wider leaves swap in order, a thread per column.
constexpr int kSwapWarps = 8;
template <typename T>
__global__ void __launch_bounds__(kSwapWarps * 32)
panel_swap_kernel(T* A, int64_t ld, const int* ipiv, int r0, int c0, int w, int pc, int pw) {
  constexpr int kMap = 32;
  __shared__ int s_src[kMap], s_dst[kMap];
  const int ncols = pw - w;
  if(w <= kMap) {
    if(threadIdx.x < w) {
      const int x = threadIdx.x;
      int       pos = x;
      for(int i = w - 1; i >= 0; --i) {
        const int p = ipiv[c0 + i] - r0;
        pos         = (pos == i) ? p : (pos == p ? i : pos);
      }
      s_src[x] = pos;
      pos      = x;
      for(int i = 0; i < w; ++i) {
        const int p = ipiv[c0 + i] - r0;
        pos         = (pos == i) ? p : (pos == p ? i : pos);
      }
      s_dst[x] = pos >= w ? pos : -1;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int j    = blockIdx.x * kSwapWarps + (threadIdx.x >> 5);
    if(j >= ncols) return;
    const int col = (pc + j < c0) ? pc + j : pc + j + w;
    T*        a   = A + (size_t)col * ld + r0;
    T         v = (T)0, o = (T)0;
    const int dst = lane < w ? s_dst[lane] : -1;
    if(lane < w) {
      v = a[s_src[lane]];
      if(dst >= 0) o = a[lane];
    }
    __syncwarp();
    if(dst >= 0) a[dst] = o;
    if(lane < w) a[lane] = v;
    return;
  }
  for(int j = blockIdx.x * blockDim.x + threadIdx.x; j < ncols; j += gridDim.x * blockDim.x) {
    const int col = (pc + j < c0) ? pc + j : pc + j + w;
    T*        a   = A + (size_t)col * ld;
    for(int k = 0; k < w; ++k) {
      const int d = r0 + k, p = ipiv[c0 + k];
      if(p != d) {
        const T t = a[d];
        a[d]      = a[p];
        a[p]      = t;
      }
    }
  }
}

// permU from the panel's jb pivots (global rows), relative to row ia:
//   permU[x]      = source row landing in row ia + x, x < jb
//   permU[jb + s] = destination of original top row s when it leaves the top
//                   block, else -1.
// Each thread traces one row through the interchange sequence.
__global__ void perm_kernel(const int* ipiv, int ia, int jb, int* permU) {
  extern __shared__ int s_piv[];
  for(int i = threadIdx.x; i < jb; i += blockDim.x) s_piv[i] = ipiv[i] - ia;
  __syncthreads();
  for(int x = threadIdx.x; x < jb; x += blockDim.x) {
    int pos = x;
    for(int i = jb - 1; i >= 0; --i) {
      const int p = s_piv[i];
      pos         = (pos == i) ? p : (pos == p ? i : pos);
    }
    permU[x] = pos;
    pos      = x;
    for(int i = 0; i < jb; ++i) {
      const int p = s_piv[i];
      pos         = (pos == i) ? p : (pos == p ? i : pos);
    }
    permU[jb + x] = pos >= jb ? pos : -1;
  }
}

// Inverses of the unit-lower kTri x kTri diagonal blocks of L (n x n at
// (r0, c0)); block b's inverse goes to inv[b * kTri * kTri], column-major.
// A partial last block is padded with the identity.
template <typename T>
__global__ void diag_inv_kernel(const T* A, int64_t ld, int r0, int c0, int n, T* inv) {
  __shared__ T L[kTri][kTri + 1];
  const int b = blockIdx.x, lane = threadIdx.x;
  const int base = b * kTri;
  for(int c = 0; c < kTri; ++c) {
    const bool in = (base + lane < n) && (base + c < n);
    L[lane][c] = in ? A[(size_t)(r0 + base + lane) + (size_t)(c0 + base + c) * ld] : (T)0;
  }
  __syncwarp();
  // Column `lane` of L^-1: forward substitution with the unit diagonal.
  T x[kTri];
#pragma unroll
  for(int i = 0; i < kTri; ++i) {
    T s = (i == lane) ? (T)1 : (T)0;
#pragma unroll
    for(int k = 0; k < i; ++k) s -= L[i][k] * x[k];
    x[i] = (i < lane) ? (T)0 : s;
  }
  T* out = inv + (size_t)b * kTri * kTri + (size_t)lane * kTri;
#pragma unroll
  for(int i = 0; i < kTri; ++i) out[i] = x[i];
}

// Fused interchange + TRSM over WCOL columns per CTA.
//   X = rows [ia, ia+jb) of columns [c0 + blockIdx.x*WCOL, ...).
//   permU (optional): apply the panel's interchanges first (dlaswp00N
//   semantics: gather the new top rows, send displaced top rows down).
//   Then X := L^-1 X with L the unit-lower jb x jb block at (ia, lc), blocked
//   by kTri rows: X_b = Dinv_b (X_b - L(b, 0:b) X(0:b)).
//   dinv: the diagonal blocks' inverses (diag_inv_kernel), or null for
//   jb <= kFusedTri: then every CTA inverts them itself into shared memory
//   first (a warp per block, the operations of diag_inv_kernel), which saves
//   the recursion a launch per node.
template <int WCOL, typename T>
__global__ void __launch_bounds__(256)
laswp_trsm_kernel(T* A, int64_t ld, int ia, int jb, const T* L, int64_t ldl,
                  const int* permU, const T* dinv, int c0, int n) {
  extern __shared__ __align__(16) unsigned char sx_raw[];
  T* sx = (T*)sx_raw;  // [WCOL][jb + 1] column-major, padded
  const int ldx = jb + 1;
  const int cb  = c0 + blockIdx.x * WCOL;
  const int nc  = min(WCOL, c0 + n - cb);
  const size_t lds = (size_t)ld;
  constexpr int kSlot = kTri * (kTri + 1);
  T* sD = sx + (size_t)WCOL * ldx;  // [nblk][kTri][kTri + 1] when dinv is null

  if(!dinv) {
    const int lane = threadIdx.x & 31;
    for(int b = threadIdx.x >> 5; b * kTri < jb; b += blockDim.x >> 5) {
      T*        slot = sD + (size_t)b * kSlot;
      const int base = b * kTri;
      for(int c = 0; c < kTri; ++c) {  // row `lane` of the block, row-major
        const bool in = (base + lane < jb) && (base + c < jb);
        slot[lane * (kTri + 1) + c] = in ? L[(size_t)(base + lane) + (size_t)(base + c) * ldl] : (T)0;
      }
      __syncwarp();
      T x[kTri];  // column `lane` of the inverse, by forward substitution
#pragma unroll
      for(int i = 0; i < kTri; ++i) {
        T s = (i == lane) ? (T)1 : (T)0;
#pragma unroll
        for(int k = 0; k < i; ++k) s -= slot[i * (kTri + 1) + k] * x[k];
        x[i] = (i < lane) ? (T)0 : s;
      }
      __syncwarp();
#pragma unroll
      for(int i = 0; i < kTri; ++i) slot[lane * (kTri + 1) + i] = x[i];  // Dinv(i, lane)
    }
  }

  // Load the top block; with permU, gather the new top rows first (the old
  // top rows are still intact in global memory), then send displaced top
  // rows down.  The gathers from rows >= jb read exactly the positions the
  // displaced rows are written to, hence the barrier between the two.
  for(int idx = threadIdx.x; idx < nc * jb; idx += blockDim.x) {
    const int c = idx / jb, x = idx % jb;
    const int src = permU ? permU[x] : x;
    sx[(size_t)c * ldx + x] = A[(size_t)(ia + src) + (size_t)(cb + c) * lds];
  }
  __syncthreads();
  if(permU) {
    for(int idx = threadIdx.x; idx < nc * jb; idx += blockDim.x) {
      const int c = idx / jb, s = idx % jb;
      const int dst = permU[jb + s];
      if(dst >= 0)
        A[(size_t)(ia + dst) + (size_t)(cb + c) * lds] = A[(size_t)(ia + s) + (size_t)(cb + c) * lds];
    }
  }
  __syncthreads();

  // Blocked forward substitution.  Thread layout: row r = tid % 32 of the
  // current 32-row block, column group cg = tid / 32 handles WCOL/8 columns.
  constexpr int CPT = WCOL / 8;
  const int r  = threadIdx.x & 31;
  const int cg = threadIdx.x >> 5;
  const int nblk = (jb + kTri - 1) / kTri;
  for(int b = 0; b < nblk; ++b) {
    const int row0 = b * kTri;
    T acc[CPT];
#pragma unroll
    for(int q = 0; q < CPT; ++q) acc[q] = (T)0;
    const int gr = row0 + r;
    if(gr < jb) {
      // Row gr of L from global memory, 16 loads in flight before their FMAs
      // (the sum still runs over kk in order, so the bits do not change).
      const T* Lrow = L + (size_t)gr;
      int      kk   = 0;
      for(; kk + 16 <= row0; kk += 16) {
        T l[16];
#pragma unroll
        for(int u = 0; u < 16; ++u) l[u] = Lrow[(size_t)(kk + u) * (size_t)ldl];
#pragma unroll
        for(int u = 0; u < 16; ++u)
#pragma unroll
          for(int q = 0; q < CPT; ++q)
            acc[q] += l[u] * sx[(size_t)(cg * CPT + q) * ldx + kk + u];
      }
      for(; kk < row0; ++kk) {
        const T l = Lrow[(size_t)kk * (size_t)ldl];
#pragma unroll
        for(int q = 0; q < CPT; ++q) acc[q] += l * sx[(size_t)(cg * CPT + q) * ldx + kk];
      }
    }
    // R = X_b - acc, kept in registers; then X_b = Dinv_b R via shared memory.
    T rv[CPT];
#pragma unroll
    for(int q = 0; q < CPT; ++q) {
      const int c = cg * CPT + q;
      rv[q] = (gr < jb) ? sx[(size_t)c * ldx + gr] - acc[q] : (T)0;
    }
    __syncthreads();
#pragma unroll
    for(int q = 0; q < CPT; ++q) {
      const int c = cg * CPT + q;
      if(gr < jb) sx[(size_t)c * ldx + gr] = rv[q];
    }
    __syncthreads();
    const T*  D    = dinv ? dinv + (size_t)b * kTri * kTri : sD + (size_t)b * kSlot;
    const int dstr = dinv ? kTri : kTri + 1;
#pragma unroll
    for(int q = 0; q < CPT; ++q) acc[q] = (T)0;
    {
      T dv[kTri];  // row r of Dinv_b, all loads in flight at once
#pragma unroll
      for(int kk = 0; kk < kTri; ++kk) dv[kk] = D[kk * dstr + r];
#pragma unroll
      for(int kk = 0; kk < kTri; ++kk)
        if(row0 + kk < jb)
#pragma unroll
          for(int q = 0; q < CPT; ++q)
            acc[q] += dv[kk] * sx[(size_t)(cg * CPT + q) * ldx + row0 + kk];
    }
    __syncthreads();
#pragma unroll
    for(int q = 0; q < CPT; ++q) {
      const int c = cg * CPT + q;
      if(gr < jb) sx[(size_t)c * ldx + gr] = acc[q];
    }
    __syncthreads();
  }

  for(int idx = threadIdx.x; idx < nc * jb; idx += blockDim.x) {
    const int c = idx / jb, x = idx % jb;
    A[(size_t)(ia + x) + (size_t)(cb + c) * lds] = sx[(size_t)c * ldx + x];
  }
}

// Row interchanges of the panel applied to columns [c0, c0+n), with the new
// top jb rows gathered into W (jb x n, leading dimension ldw) instead of being
// written back: W then feeds U12 = L11^-1 W as a DMMA GEMM that writes the top
// rows of A.  Displaced top rows go straight to their new rows below.  The
// row map sits in shared memory; each warp owns whole columns (lane = row, so
// every W store and every unpermuted read is a 256-byte segment), gathers a
// column's jb rows into registers before any of its displaced writes (which
// overwrite exactly rows the gather may read: the warp's own column only, so a
// __syncwarp orders them), and moves on to its next column.
constexpr int kGatherWarps = 8;
constexpr int kGatherRegs  = 16;  // rows per lane held at once (jb <= 512 in one pass)
template <typename T>
__global__ void __launch_bounds__(kGatherWarps * 32)
laswp_gather_kernel(T* A, int64_t ld, int ia, int jb, const int* __restrict__ permU,
                    T* __restrict__ W, int64_t ldw, int c0, int n) {
  extern __shared__ int s_perm[];  // 2 jb ints
  for(int i = threadIdx.x; i < 2 * jb; i += blockDim.x) s_perm[i] = permU[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * kGatherWarps;
  for(int c = blockIdx.x * kGatherWarps + (threadIdx.x >> 5); c < n; c += warps) {
    T*       col = A + (size_t)ia + (size_t)(c0 + c) * (size_t)ld;
    T*       wc  = W + (size_t)c * (size_t)ldw;
    for(int x0 = 0; x0 < jb; x0 += 32 * kGatherRegs) {
      T v[kGatherRegs];
#pragma unroll
      for(int k = 0; k < kGatherRegs; ++k) {
        const int x = x0 + 32 * k + lane;
        v[k] = x < jb ? col[s_perm[x]] : (T)0;
      }
#pragma unroll
      for(int k = 0; k < kGatherRegs; ++k) {
        const int x = x0 + 32 * k + lane;
        if(x < jb) wc[x] = v[k];
      }
    }
    __syncwarp();
    for(int x = lane; x < jb; x += 32) {
      const int dst = s_perm[jb + x];
      if(dst >= 0) col[dst] = col[x];
    }
    __syncwarp();
  }
}

// Writes the jb x jb identity into X (leading dimension ldx).
template <typename T>
__global__ void identity_kernel(T* X, int64_t ldx, int jb) {
  const int c = blockIdx.x;
  for(int r = threadIdx.x; r < jb; r += blockDim.x)
    X[(size_t)r + (size_t)c * ldx] = (r == c) ? (T)1 : (T)0;
}

}  // namespace

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------

int leaf_grid_size(int num_sms, int rows) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, leaf_kernel<double>, kLeafThreads, 0);
  if(per_sm < 1) per_sm = 1;
  const int max_grid = num_sms * per_sm;
  // At least ~256 rows per block so the barrier count is worth the parallelism.
  int g = (rows + 255) / 256;
  if(g > max_grid) g = max_grid;
  if(g < 1) g = 1;
  return g;
}

// Largest dynamic shared memory the resident-slice leaf may take (bytes), set
// once per element type.
template <typename T>
static int leaf_smem_budget() {
  static int budget = -1;
  if(budget < 0) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, leaf_smem_kernel<T>);
    int b = optin - (int)fa.sharedSizeBytes - 1024;
    if(b < 0 ||
       cudaFuncSetAttribute(leaf_smem_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, b) !=
           cudaSuccess) {
      cudaGetLastError();
      b = 0;
    }
    budget = b;
  }
  return budget;
}

template <typename T, int RPT>
static cudaError_t launch_leaf_reg(LeafParams<T> P, int g, cudaStream_t stream) {
  P.rpb         = RPT * kRegLeafThreads;
  cudaError_t e = cudaMemsetAsync(P.bar, 0, 2 * sizeof(int), stream);
  if(e != cudaSuccess) return e;
  void* args[] = {&P};
  return cudaLaunchCooperativeKernel((const void*)leaf_reg_kernel<T, RPT>, dim3(g),
                                     dim3(kRegLeafThreads), args, 0, stream);
}

// Rows per thread the register leaf is built for: the smallest that puts the
// leaf on at most one block per SM (3 x 32 doubles or 4 x 32 floats per
// thread fill the register file of a 256-thread block without spilling).
template <typename T>
static cudaError_t try_leaf_reg(const LeafParams<T>& P, int rows, int sms, int grid,
                                cudaStream_t stream, bool* done) {
  constexpr int kMaxRpt = sizeof(T) == 8 ? 3 : 4;
  *done                 = false;
  for(int rpt = 1; rpt <= kMaxRpt; ++rpt) {
    const int cap = rpt * kRegLeafThreads;
    const int g   = (rows + cap - 1) / cap;
    if(g > sms || g > grid) continue;
    *done = true;
    switch(rpt) {
      case 1: return launch_leaf_reg<T, 1>(P, g, stream);
      case 2: return launch_leaf_reg<T, 2>(P, g, stream);
      case 3: return launch_leaf_reg<T, 3>(P, g, stream);
      default: return launch_leaf_reg<T, kMaxRpt>(P, g, stream);
    }
  }
  return cudaSuccess;
}

// The cluster leaf with RPT rows per thread on g CTAs.  Whether a cluster of g
// such CTAs can be placed at all is asked once per (type, RPT, g); a launch
// that cannot be placed, or fails, falls through to the next leaf kind.
template <typename T, int RPT>
static cudaError_t launch_leaf_cluster(LeafParams<T> P, int g, cudaStream_t stream, bool* done) {
  static signed char placeable[kClusterLeafMax + 1] = {};  // 0 unknown, 1 yes, -1 no
  *done = false;
  if(g < 1 || g > kClusterLeafMax) return cudaSuccess;
  P.rpb = RPT * kRegLeafThreads;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim  = dim3((unsigned)g);
  cfg.blockDim = dim3(kRegLeafThreads);
  cfg.stream   = stream;
  cudaLaunchAttribute at[1];
  at[0].id               = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)g;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs              = at;
  cfg.numAttrs           = 1;
  if(placeable[g] == 0) {
    int n = 0;
    if(g > 8 && cudaFuncSetAttribute((const void*)leaf_cluster_kernel<T, RPT>,
                                     cudaFuncAttributeNonPortableClusterSizeAllowed,
                                     1) != cudaSuccess) {
      cudaGetLastError();
      placeable[g] = -1;
    } else if(cudaOccupancyMaxActiveClusters(&n, (const void*)leaf_cluster_kernel<T, RPT>, &cfg) !=
                  cudaSuccess ||
              n < 1) {
      cudaGetLastError();
      placeable[g] = -1;
    } else {
      placeable[g] = 1;
    }
  }
  if(placeable[g] < 0) return cudaSuccess;
  cudaError_t e = cudaLaunchKernelEx(&cfg, leaf_cluster_kernel<T, RPT>, P);
  if(e != cudaSuccess) {
    cudaGetLastError();
    placeable[g] = -1;
    return cudaSuccess;
  }
  *done = true;
  return cudaSuccess;
}

// Rows per thread: the smaller of two forms whose cluster (at most 16 CTAs)
// holds the rows; the smaller form keeps its rows in registers without
// spilling (FP64: 2 rows of 32 doubles per thread; FP32: 3 of 32 floats), the
// larger reaches further (FP64: 3 rows, 12288 in all; FP32: 4 rows, 16384).
template <typename T>
static cudaError_t try_leaf_cluster(const LeafParams<T>& P, int rows, cudaStream_t stream,
                                    bool* done) {
  constexpr int kLo = sizeof(T) == 8 ? 2 : 3, kHi = kLo + 1;
  *done = false;
  const int glo = (rows + kLo * kRegLeafThreads - 1) / (kLo * kRegLeafThreads);
  if(glo <= kClusterLeafMax) return launch_leaf_cluster<T, kLo>(P, glo, stream, done);
  const int ghi = (rows + kHi * kRegLeafThreads - 1) / (kHi * kRegLeafThreads);
  if(ghi <= kClusterLeafMax) return launch_leaf_cluster<T, kHi>(P, ghi, stream, done);
  return cudaSuccess;
}

template <typename T>
cudaError_t launch_leaf(T* A, int64_t ld, int r0, int end, int c0, int w, int pc, int pw,
                        int* ipiv, double* cand, double* cur, int* bar, int* status, int grid,
                        int leaf_kind, cudaStream_t stream, bool* swapped) {
  *swapped = false;
  // 0: cluster, then registers; 3: registers (grid-wide); 1: shared memory
  // first; 2: global memory.
  const int mode = leaf_kind == HPLB_LEAF_SHARED      ? 1
                   : leaf_kind == HPLB_LEAF_GLOBAL    ? 2
                   : leaf_kind == HPLB_LEAF_REGISTERS ? 3
                                                      : 0;
  const int rows = end - r0;
  int       dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if(w <= kRegLeafW && rows > 0 && mode == 0) {
    LeafParams<T> P;
    P.A      = A;
    P.ld     = ld;
    P.r0     = r0;
    P.end    = end;
    P.c0     = c0;
    P.w      = w;
    P.rpb    = 0;
    P.ipiv   = ipiv;
    P.cand   = cand;
    P.cur    = cur;
    P.bar    = bar;
    P.status = status;
    P.pc     = pc;
    P.pw     = pw;
    bool              done = false;
    const cudaError_t e    = try_leaf_cluster<T>(P, rows, stream, &done);
    *swapped               = done;
    if(done || e != cudaSuccess) return e;
  }
  if(w <= kRegLeafW && rows > 0 && (mode == 0 || mode == 3)) {
    LeafParams<T> P;
    P.A      = A;
    P.ld     = ld;
    P.r0     = r0;
    P.end    = end;
    P.c0     = c0;
    P.w      = w;
    P.rpb    = 0;
    P.ipiv   = ipiv;
    P.cand   = cand;
    P.cur    = cur;
    P.bar    = bar;
    P.status = status;
    bool              done = false;
    const cudaError_t e    = try_leaf_reg<T>(P, rows, sms, grid, stream, &done);
    if(done) return e;
  }
  // Resident-slice leaf: as few blocks as hold the leaf in shared memory (one
  // per SM at most).
  if(w <= kSmemLeafW && rows > 0 && mode <= 1) {
    const int budget = leaf_smem_budget<T>();
    const int rmax   = budget / (w * (int)sizeof(T));
    if(rmax >= 32) {
      const int g = (rows + rmax - 1) / rmax;
      if(g <= sms && g <= grid) {
        LeafParams<T> P;
        P.A      = A;
        P.ld     = ld;
        P.r0     = r0;
        P.end    = end;
        P.c0     = c0;
        P.w      = w;
        P.rpb    = (rows + g - 1) / g;
        P.ipiv   = ipiv;
        P.cand   = cand;
        P.cur    = cur;
        P.bar    = bar;
        P.status = status;
        cudaError_t e = cudaMemsetAsync(bar, 0, 2 * sizeof(int), stream);
        if(e != cudaSuccess) return e;
        void* args[] = {&P};
        return cudaLaunchCooperativeKernel((const void*)leaf_smem_kernel<T>, dim3(g),
                                           dim3(kSmemLeafThreads), args,
                                           (size_t)P.rpb * w * sizeof(T), stream);
      }
    }
  }
  LeafParams<T> P;
  P.A = A;
  P.ld = ld;
  P.r0 = r0;
  P.end = end;
  P.c0 = c0;
  P.w = w;
  P.rpb = (end - r0 + grid - 1) / grid;
  P.ipiv = ipiv;
  P.cand = cand;
  P.cur = cur;
  P.bar = bar;
  P.status = status;
  cudaError_t e = cudaMemsetAsync(bar, 0, 2 * sizeof(int), stream);
  if(e != cudaSuccess) return e;
  void* args[] = {&P};
  return cudaLaunchCooperativeKernel((const void*)leaf_kernel<T>, dim3(grid),
                                     dim3(kLeafThreads), args, 0, stream);
}

template <typename T>
cudaError_t launch_panel_swap(T* A, int64_t ld, const int* ipiv, int r0, int c0, int w, int pc,
                              int pw, cudaStream_t stream) {
  const int ncols = pw - w;
  if(ncols <= 0) return cudaSuccess;
  const int grid = w <= 32 ? (ncols + kSwapWarps - 1) / kSwapWarps
                            : (ncols + kSwapWarps * 32 - 1) / (kSwapWarps * 32);
  panel_swap_kernel<T><<<grid, kSwapWarps * 32, 0, stream>>>(A, ld, ipiv, r0, c0, w, pc, pw);
  return cudaGetLastError();
}

cudaError_t launch_perm(const int* ipiv, int ia, int jb, int* permU, cudaStream_t stream) {
  if(jb <= 0) return cudaSuccess;
  perm_kernel<<<1, 1024, jb * sizeof(int), stream>>>(ipiv, ia, jb, permU);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_diag_inv(const T* A, int64_t ld, int r0, int c0, int n, T* inv,
                            cudaStream_t stream) {
  if(n <= 0) return cudaSuccess;
  diag_inv_kernel<T><<<(n + kTri - 1) / kTri, kTri, 0, stream>>>(A, ld, r0, c0, n, inv);
  return cudaGetLastError();
}

int trsm_wcol(int jb) { return jb <= 512 ? 32 : (jb <= 1024 ? 16 : 8); }

// Shared memory of laswp_trsm_kernel (sized for double; ample for float):
// the X block, plus the diagonal inverses when the kernel makes them.
size_t trsm_smem_bytes(int jb, bool own_dinv) {
  const int w = trsm_wcol(jb);
  size_t    b = (size_t)w * (jb + 1) * 8;
  if(own_dinv) b += (size_t)((jb + kTri - 1) / kTri) * kTri * (kTri + 1) * 8;
  return b;
}

template <int W, typename T>
static cudaError_t launch_trsm_w(int grid, size_t smem, T* X, int64_t ldx, int ia, int jb,
                                 const T* L, int64_t ldl, const int* permU, const T* dinv,
                                 int c0, int n, cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(laswp_trsm_kernel<W, T>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if(e != cudaSuccess) return e;
  laswp_trsm_kernel<W, T><<<grid, 256, smem, stream>>>(X, ldx, ia, jb, L, ldl, permU, dinv, c0,
                                                       n);
  return cudaGetLastError();
}

template <typename T>
static cudaError_t launch_trsm_any(T* X, int64_t ldx, int ia, int jb, const T* L, int64_t ldl,
                                   const int* permU, const T* dinv, int c0, int n,
                                   cudaStream_t stream) {
  if(n <= 0 || jb <= 0) return cudaSuccess;
  if(!dinv && jb > kFusedTri) return cudaErrorInvalidValue;
  const int    w    = trsm_wcol(jb);
  const size_t smem = trsm_smem_bytes(jb, !dinv);
  const int    grid = (n + w - 1) / w;
  switch(w) {
    case 32:
      return launch_trsm_w<32, T>(grid, smem, X, ldx, ia, jb, L, ldl, permU, dinv, c0, n, stream);
    case 16:
      return launch_trsm_w<16, T>(grid, smem, X, ldx, ia, jb, L, ldl, permU, dinv, c0, n, stream);
    default:
      return launch_trsm_w<8, T>(grid, smem, X, ldx, ia, jb, L, ldl, permU, dinv, c0, n, stream);
  }
}

template <typename T>
cudaError_t launch_laswp_trsm(T* A, int64_t ld, int ia, int jb, int lc, const int* permU,
                              const T* dinv, int c0, int n, cudaStream_t stream) {
  return launch_trsm_any<T>(A, ld, ia, jb, A + (size_t)ia + (size_t)lc * ld, ld, permU, dinv, c0,
                            n, stream);
}

template <typename T>
cudaError_t launch_trsm_node(T* A, int64_t ld, int ia, int jb, int lc, T* dinv_scratch, int c0,
                             int n, cudaStream_t stream, int* launches) {
  if(n <= 0 || jb <= 0) return cudaSuccess;
  if(jb <= kFusedTri) {
    *launches += 1;
    return launch_laswp_trsm<T>(A, ld, ia, jb, lc, nullptr, nullptr, c0, n, stream);
  }
  cudaError_t e = launch_diag_inv<T>(A, ld, ia, lc, jb, dinv_scratch, stream);
  if(e != cudaSuccess) return e;
  *launches += 2;
  return launch_laswp_trsm<T>(A, ld, ia, jb, lc, nullptr, dinv_scratch, c0, n, stream);
}

// X (jb x n, leading dimension ldx) <- L^-1 X for the unit-lower jb x jb L at
// L (leading dimension ldl), dinv its 32 x 32 diagonal inverses (diag_inv).
cudaError_t launch_trsm_unit_lower(double* X, int64_t ldx, int jb, const double* L, int64_t ldl,
                                   const double* dinv, int n, cudaStream_t stream) {
  return launch_trsm_any<double>(X, ldx, 0, jb, L, ldl, nullptr, dinv, 0, n, stream);
}

template <typename T>
cudaError_t launch_unit_lower_inverse(const T* L, int64_t ldl, int jb, const T* dinv, T* Linv,
                                      int64_t ldinv, cudaStream_t stream) {
  if(jb <= 0) return cudaSuccess;
  identity_kernel<T><<<jb, 128, 0, stream>>>(Linv, ldinv, jb);
  cudaError_t e = cudaGetLastError();
  if(e != cudaSuccess) return e;
  return launch_trsm_any<T>(Linv, ldinv, 0, jb, L, ldl, nullptr, dinv, 0, jb, stream);
}

template <typename T>
cudaError_t launch_laswp_gather(T* A, int64_t ld, int ia, int jb, const int* permU, T* W,
                                int64_t ldw, int c0, int n, cudaStream_t stream) {
  if(n <= 0 || jb <= 0) return cudaSuccess;
  // One column per warp, capped at 8 CTAs per SM (wide updates then give each
  // warp several columns instead of re-staging the row map per column).
  int sms = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int want = (n + kGatherWarps - 1) / kGatherWarps;
  const int grid = std::max(1, std::min(want, 8 * std::max(sms, 1)));
  laswp_gather_kernel<T><<<grid, kGatherWarps * 32, 2 * jb * sizeof(int), stream>>>(
      A, ld, ia, jb, permU, W, ldw, c0, n);
  return cudaGetLastError();
}

#define HPLB_PANEL_INSTANTIATE(T)                                                              \
  template cudaError_t launch_leaf<T>(T*, int64_t, int, int, int, int, int, int, int*, double*,  \
                                      double*, int*, int*, int, int, cudaStream_t, bool*);     \
  template cudaError_t launch_panel_swap<T>(T*, int64_t, const int*, int, int, int, int, int,  \
                                            cudaStream_t);                                     \
  template cudaError_t launch_diag_inv<T>(const T*, int64_t, int, int, int, T*, cudaStream_t); \
  template cudaError_t launch_laswp_trsm<T>(T*, int64_t, int, int, int, const int*, const T*,  \
                                            int, int, cudaStream_t);                           \
  template cudaError_t launch_trsm_node<T>(T*, int64_t, int, int, int, T*, int, int,            \
                                           cudaStream_t, int*);                                \
  template cudaError_t launch_unit_lower_inverse<T>(const T*, int64_t, int, const T*, T*,      \
                                                    int64_t, cudaStream_t);                    \
  template cudaError_t launch_laswp_gather<T>(T*, int64_t, int, int, const int*, T*, int64_t,  \
                                              int, int, cudaStream_t);
HPLB_PANEL_INSTANTIATE(double)
HPLB_PANEL_INSTANTIATE(float)

}  // namespace hplb
