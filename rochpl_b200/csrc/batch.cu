// Batched FP64 LU + solve of many independent systems of uneven size in one
// persistent launch (no counterpart in the reference, whose solve is a single
// system; the per-system algorithm is the right-looking blocked LU with
// partial pivoting of HPL_pdgesv, with LAPACK's full-row interchanges so that
// the right-hand sides ride along as extra columns).
//
// One CTA (kBT threads) owns one system at a time and takes the next one from
// a work counter; the plan orders systems by descending cost so the large ones
// start first.  Per panel of nb columns (nb from the plan's size class):
//   panel      the m x kb panel is factored in shared memory (pivot search by
//              warp shuffles and a block reduction, division by the pivot, rank-1
//              updates inside the panel), then written back;
//   swaps      the panel's interchanges applied to the other columns of A and to B;
//   trsm       U12 = L11^-1 A12 (and B's rows), one column per thread;
//   update     A22 -= L21 U12 and B2 -= L21 U12_B on the FP64 tensor cores
//              (DMMA m16n8k8) from 64 x 64 tiles staged in shared memory.
// Then U X = B by blocks (substitution on the diagonal blocks, DMMA updates).
// The stored-factor solves (plain and transposed), the batched rank-k product
// of the adjoint, the per-system LCG generator and the per-system HPL residual
// use the same CTA-per-system loop.
#include <algorithm>

#include "common.cuh"
#include "internal.h"
#include "lcg.cuh"

namespace hplb {

namespace {

constexpr int kBT    = 512;  // threads per CTA
constexpr int kBW    = kBT / 32;
constexpr int kNbMax = 32;   // widest panel
constexpr int kTile  = 64;   // output tile of the block updates
constexpr int kLdT   = kTile + 4;
constexpr int kRegPanelW = 16;  // widest panel held in registers
constexpr int kRecMode   = 64;  // Sys::nb value selecting the recursive factorisation

// Leading dimension of the panel copy in shared memory: >= n rows and = 4
// (mod 16), so the DMMA A-fragment loads (rows g, columns t) hit distinct banks.
__host__ __device__ inline int panel_ld(int n) { return (n + 15) / 16 * 16 + 4; }

struct Sys {
  int       n, nrhs, nb, pad;
  long long a_off, b_off, p_off;
};

struct Args {
  double*       A;      // A pool (factored in place), or null
  const double* LU;     // stored factors (solve-only modes)
  double*       B;      // B pool (overwritten by X)
  int*          ipiv;   // pivot pool (global row within the system, 0-based)
  const int*    ipivc;  // stored pivots (solve-only modes)
  int*          info;   // per system: first zero pivot (1-based) or 0
  const Sys*    sys;    // descriptors
  const int*    order;  // work order
  int           count;
  int*          counter;
  double        alpha;  // rank-k scale
  const double* X;      // rank-k operands (B-pool layout)
  const double* Y;
  double*       C;      // rank-k output (A-pool layout)
  const unsigned long long* seeds;  // generator / residual
  double*       resid;  // per system HPL scaled residual (max over its RHS)
};

// Shared scratch of every mode.  The panel P is [kb][ldp] column-major.
struct Smem {
  double red_v[kBW];
  int    red_r[kBW];
  int    piv[kNbMax];
  int    src[kNbMax];  // new top row x came from row src[x] (panel-local)
  int    dst[kNbMax];  // old top row x went to row dst[x], or -1 if it stayed on top
  int    next;
  int    info;
  // The A tile of the staged GEMMs and the register panel's exchange slots are
  // never live at once.
  union {
    double As[kNbMax][kLdT];  // A tile: k x rows
    // Register panel: per warp, its pivot candidate and that row's values,
    // and the diagonal row; double-buffered by column parity.
    struct {
      double cv[2][kBW];
      int    cr[2][kBW];
      double crow[2][kBW][kRegPanelW];
      double cur[2][kRegPanelW];
    } pr;
  };
  double Bs[kTile][kNbMax + 4];  // B tile: cols x k (row length = 4 mod 16: conflict free)
  double D[kNbMax][kNbMax + 1];  // a diagonal block
};

HPLB_DEV bool better_b(double av, int ar, double bv, int br) {
  if(br < 0) return ar >= 0;
  if(ar < 0) return false;
  const double fa = fabs(av), fb = fabs(bv);
  if(fa > fb) return true;
  if(fa < fb) return false;
  return ar < br;
}

HPLB_DEV void argmax_block(double& v, int& r, Smem& S) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  warp_argmax(v, r);
  __syncthreads();
  if(lane == 0) {
    S.red_v[warp] = v;
    S.red_r[warp] = r;
  }
  __syncthreads();
  v = lane < kBW ? S.red_v[lane] : 0.0;
  r = lane < kBW ? S.red_r[lane] : -1;
  warp_argmax(v, r);
}

HPLB_DEV void dmma(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// C (m x n) -= A (m x k) B (k x n), k <= kNbMax, all column-major in global
// memory, by 64 x 64 tiles: A and B slices staged in shared memory (zero
// padded to a multiple of 8 in k), C accumulated in DMMA fragments.  16 warps:
// 4 x 4, each 16 rows x 16 columns (two m16n8 tiles).  Fragment layout
// (g = lane / 4, t = lane % 4): A a0 (g, t) a1 (g+8, t) a2 (g, t+4)
// a3 (g+8, t+4); B b0 (t, g) b1 (t+4, g); C c0 (g, 2t) c1 (g, 2t+1)
// c2 (g+8, 2t) c3 (g+8, 2t+1).
HPLB_DEV void tile_gemm_sub(int m, int n, int k, const double* A, int64_t lda, const double* B,
                            int64_t ldb, double* C, int64_t ldc, Smem& S) {
  if(m <= 0 || n <= 0 || k <= 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp & 3) * 16, wn = (warp >> 2) * 16;
  const int k8 = (k + 7) & ~7;
  const int tm = (m + kTile - 1) / kTile, tn = (n + kTile - 1) / kTile;
  for(int tile = 0; tile < tm * tn; ++tile) {
    const int m0 = (tile % tm) * kTile, n0 = (tile / tm) * kTile;
    __syncthreads();
    for(int idx = threadIdx.x; idx < k8 * kTile; idx += kBT) {
      const int r = idx % kTile, kk = idx / kTile;
      S.As[kk][r] = (kk < k && m0 + r < m) ? A[(size_t)(m0 + r) + (size_t)kk * lda] : 0.0;
      const int c = idx / k8, k2 = idx % k8;
      S.Bs[c][k2] = (k2 < k && n0 + c < n) ? B[(size_t)k2 + (size_t)(n0 + c) * ldb] : 0.0;
    }
    __syncthreads();
    double acc[2][4];
#pragma unroll
    for(int j = 0; j < 2; ++j)
#pragma unroll
      for(int q = 0; q < 4; ++q) acc[j][q] = 0.0;
    for(int kk = 0; kk < k8; kk += 8) {
      double af[4], bf[2][2];
      af[0] = S.As[kk + t][wm + g];
      af[1] = S.As[kk + t][wm + g + 8];
      af[2] = S.As[kk + t + 4][wm + g];
      af[3] = S.As[kk + t + 4][wm + g + 8];
#pragma unroll
      for(int j = 0; j < 2; ++j) {
        bf[j][0] = S.Bs[wn + j * 8 + g][kk + t];
        bf[j][1] = S.Bs[wn + j * 8 + g][kk + t + 4];
      }
#pragma unroll
      for(int j = 0; j < 2; ++j) dmma(acc[j], af, bf[j]);
    }
#pragma unroll
    for(int j = 0; j < 2; ++j)
#pragma unroll
      for(int q = 0; q < 4; ++q) {
        const int r = m0 + wm + g + (q >> 1) * 8;
        const int c = n0 + wn + j * 8 + 2 * t + (q & 1);
        if(r < m && c < n) {
          double* p = C + (size_t)r + (size_t)c * ldc;
          *p -= acc[j][q];
        }
      }
  }
  __syncthreads();
}

// C (m x n) -= A^T B with A (k x m), B (k x n), m <= kNbMax, n arbitrary:
// k-chunks of 64 of A and of B staged in shared memory; thread (i, c) keeps its
// outputs in registers across the chunks.  For the transposed solves.
HPLB_DEV void tile_gemm_tn_sub(int m, int n, int k, const double* A, int64_t lda,
                               const double* B, int64_t ldb, double* C, int64_t ldc, Smem& S) {
  if(m <= 0 || n <= 0 || k <= 0) return;
  for(int n0 = 0; n0 < n; n0 += kTile) {
    const int nc = min(kTile, n - n0);
    // thread -> (i = idx % m, c = idx / m) for idx = threadIdx.x + s * kBT
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for(int k0 = 0; k0 < k; k0 += kTile) {
      const int kc = min(kTile, k - k0);
      __syncthreads();
      // As[i][kk] (i < m <= 32, kk < 64) reuses As as [kNbMax][kLdT]
      for(int idx = threadIdx.x; idx < kNbMax * kTile; idx += kBT) {
        const int i = idx / kTile, kk = idx % kTile;
        S.As[i][kk] = (i < m && kk < kc) ? A[(size_t)(k0 + kk) + (size_t)i * lda] : 0.0;
      }
      // Bs[c][kk] for c < 64, kk < 32: two halves of the 64-long chunk
      for(int half = 0; half < 2; ++half) {
        __syncthreads();
        for(int idx = threadIdx.x; idx < kTile * kNbMax; idx += kBT) {
          const int c = idx / kNbMax, kk = idx % kNbMax;
          const int kg = half * kNbMax + kk;
          S.Bs[c][kk] = (c < nc && kg < kc) ? B[(size_t)(k0 + kg) + (size_t)(n0 + c) * ldb] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for(int s = 0; s < 4; ++s) {
          const int idx = threadIdx.x + s * kBT;
          const int i = idx % kNbMax, c = idx / kNbMax;
          if(i < m && c < nc) {
            double a = acc[s];
            for(int kk = 0; kk < kNbMax; ++kk) a += S.As[i][half * kNbMax + kk] * S.Bs[c][kk];
            acc[s] = a;
          }
        }
      }
    }
#pragma unroll
    for(int s = 0; s < 4; ++s) {
      const int idx = threadIdx.x + s * kBT;
      const int i = idx % kNbMax, c = idx / kNbMax;
      if(i < m && c < nc) C[(size_t)i + (size_t)(n0 + c) * ldc] -= acc[s];
    }
  }
  __syncthreads();
}

// S.D <- the kb x kb diagonal block at A (leading dimension lda).
HPLB_DEV void load_diag(const double* A, int64_t lda, int kb, Smem& S) {
  __syncthreads();
  for(int idx = threadIdx.x; idx < kb * kb; idx += kBT) {
    const int r = idx % kb, c = idx / kb;
    S.D[r][c] = A[(size_t)r + (size_t)c * lda];
  }
  __syncthreads();
}

// Substitution with S.D on n columns of X (kb rows, leading dimension ldx),
// one warp per column, lane = row, a run-time loop over the kb steps (each
// solved entry broadcast by a shuffle and eliminated from the other lanes):
//   LOWER_UNIT:      X <- L^-1 X     (unit lower, forward)
//   UPPER:           X <- U^-1 X     (backward)
//   UPPER_T:         X <- U^-T X     (U^T lower, forward)
//   LOWER_UNIT_T:    X <- L^-T X     (L^T unit upper, backward)
enum { LOWER_UNIT = 0, UPPER = 1, UPPER_T = 2, LOWER_UNIT_T = 3 };
template <int KIND>
__device__ __noinline__ void diag_solve(int kb, double* X, int64_t ldx, int n, const Smem& S) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for(int c = warp; c < n; c += kBW) {
    double* col = X + (size_t)c * ldx;
    double  x   = lane < kb ? col[lane] : 0.0;
    if(KIND == LOWER_UNIT || KIND == UPPER_T) {
#pragma unroll 4
      for(int r = 0; r < kb; ++r) {
        if(KIND == UPPER_T && lane == r) x = x / S.D[r][r];
        const double xr = __shfl_sync(0xffffffffu, x, r);
        if(lane > r && lane < kb) x -= (KIND == LOWER_UNIT ? S.D[lane][r] : S.D[r][lane]) * xr;
      }
    } else {
#pragma unroll 4
      for(int r = kb - 1; r >= 0; --r) {
        if(KIND == UPPER && lane == r) x = x / S.D[r][r];
        const double xr = __shfl_sync(0xffffffffu, x, r);
        if(lane < r) x -= (KIND == UPPER ? S.D[lane][r] : S.D[r][lane]) * xr;
      }
    }
    if(lane < kb) col[lane] = x;
  }
  __syncthreads();
}

// Take the next system index (or -1), in the plan's order.
HPLB_DEV int next_system(const Args& a, Smem& S) {
  __syncthreads();
  if(threadIdx.x == 0) {
    const int s = atomicAdd(a.counter, 1);
    S.next      = s < a.count ? a.order[s] : -1;
  }
  __syncthreads();
  return S.next;
}

// x[c] for a column index c < KB known only at run time, by a tree of
// selects on the bits of c (log2 KB deep; the row stays in registers).
template <int KB>
HPLB_DEV double pick(const double (&x)[KB], int c) {
  static_assert((KB & (KB - 1)) == 0, "pick: KB must be a power of two");
  double t[KB];
#pragma unroll
  for(int q = 0; q < KB; ++q) t[q] = x[q];
#pragma unroll
  for(int h = KB / 2; h >= 1; h /= 2)
#pragma unroll
    for(int q = 0; q < h; ++q) t[q] = (c & h) ? t[q + h] : t[q];
  return t[0];
}

// The m x kb panel at A (leading dimension lda; rows k0.. of the system),
// kb <= KB, with each thread's rows t + q * kBT (q < RPT) in registers.  The
// column loop is a run-time loop whose body touches every register of the row
// (selects and FMAs), so the code stays a few KB and is fetched once, not once
// per column.  Per column: each warp finds its candidate by shuffles and
// publishes it with the row's values, the owner of the diagonal row publishes
// that row, one barrier, then every thread picks the winner and applies the
// interchange, the scaling by the pivot's reciprocal (as LAPACK's dgetf2) and
// the update to its own rows.  The update runs against the pivot row with its
// entries of columns <= j selected to zero, so each entry costs one FMA and two
// selects, no branch; a non-finite multiplier keeps the predicated form, which
// leaves the columns before j untouched.  The factored
// panel goes back to A and, if P is given, to the shared copy P (leading
// dimension ldp) that the trailing update reads L21 from.
template <int RPT, int KB>
__device__ __noinline__ void panel_reg(double* Ag, int lda, int m, int kb, int k0, int* ip, double* P, int ldp,
                        Smem& S) {
  static_assert(KB <= kRegPanelW, "panel wider than the exchange slots");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double    x[RPT][KB];
  int       row[RPT];
#pragma unroll
  for(int q = 0; q < RPT; ++q) {
    row[q]        = threadIdx.x + q * kBT;
    const bool in = row[q] < m;
    if(!in) row[q] = -1;
#pragma unroll
    for(int c = 0; c < KB; ++c) x[q][c] = (in && c < kb) ? Ag[(size_t)row[q] + (size_t)c * lda] : 0.0;
  }
#pragma unroll 1
  for(int j = 0; j < kb; ++j) {
    const int par = j & 1;
    double    v   = 0.0;
    int       r   = -1;
#pragma unroll
    for(int q = 0; q < RPT; ++q) {
      const double xj = pick(x[q], j);
      if(row[q] >= j && better_b(xj, row[q], v, r)) {
        v = xj;
        r = row[q];
      }
    }
    warp_argmax(v, r);
    if(lane == 0) {
      S.pr.cv[par][warp] = v;
      S.pr.cr[par][warp] = r;
    }
#pragma unroll
    for(int q = 0; q < RPT; ++q) {
      if(r >= 0 && row[q] == r)
#pragma unroll
        for(int c = 0; c < KB; ++c) S.pr.crow[par][warp][c] = x[q][c];
      if(row[q] == j)
#pragma unroll
        for(int c = 0; c < KB; ++c) S.pr.cur[par][c] = x[q][c];
    }
    __syncthreads();
    // The winner among the warps' candidates (lanes 0..15 read one each).
    double bv = lane < kBW ? S.pr.cv[par][lane] : 0.0;
    int    br = lane < kBW ? S.pr.cr[par][lane] : -1;
    int    bw = warp_argmax(bv, br);
    if(bw < 0) {  // no candidate: only when the panel has no rows >= j, which cannot happen
      bw = 0;
      bv = 0.0;
      br = j;
    }
    const double* u = S.pr.crow[par][bw];
    if(threadIdx.x == 0) {
      S.piv[j]   = br;
      ip[k0 + j] = k0 + br;
      if(bv == 0.0 && S.info == 0) S.info = k0 + j + 1;
    }
    const double rcp = bv != 0.0 ? 1.0 / bv : 0.0;
#pragma unroll
    for(int q = 0; q < RPT; ++q) {
      if(row[q] == j) {
#pragma unroll
        for(int c = 0; c < KB; ++c) x[q][c] = u[c];
      } else if(row[q] == br) {
#pragma unroll
        for(int c = 0; c < KB; ++c) x[q][c] = S.pr.cur[par][c];
      }
      if(bv != 0.0 && row[q] > j) {
        const double l = pick(x[q], j) * rcp;
        if(isfinite(l)) {
#pragma unroll
          for(int c = 0; c < KB; ++c) {
            const double uc = u[c];
            const double nx = fma(-l, c > j ? uc : 0.0, x[q][c]);
            x[q][c]         = (c == j) ? l : nx;
          }
        } else {
#pragma unroll
          for(int c = 0; c < KB; ++c) {
            if(c == j) x[q][c] = l;
            else if(c > j) x[q][c] = fma(-l, u[c], x[q][c]);
          }
        }
      }
    }
  }
#pragma unroll
  for(int q = 0; q < RPT; ++q)
    if(row[q] >= 0)
#pragma unroll
      for(int c = 0; c < KB; ++c)
        if(c < kb) {
          Ag[(size_t)row[q] + (size_t)c * lda] = x[q][c];
          if(P) P[(size_t)c * ldp + row[q]] = x[q][c];
        }
  __syncthreads();
}

// C (m2 x ncols, leading dimension ldc) -= L21 U with L21 = rows kb .. kb+m2 of
// the panel copy P (leading dimension ldp, kb columns) and U (kb x ncols,
// leading dimension ldu) in global memory.  U is staged 64 columns at a time;
// within a column block every warp streams its own 16-row strips of C through
// DMMA (A fragments straight from P, B fragments from the staged block, C
// fragments from and back to global memory) with no block barrier between
// strips.
__device__ __noinline__ void update_strips(const double* P, int ldp, int kb, int m2, const double* U, int ldu,
                            double* C, int ldc, int ncols, Smem& S) {
  if(m2 <= 0 || ncols <= 0 || kb <= 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int k8 = (kb + 7) & ~7;
  for(int cb = 0; cb < ncols; cb += kTile) {
    const int nc = min(kTile, ncols - cb);
    __syncthreads();
    for(int idx = threadIdx.x; idx < kTile * k8; idx += kBT) {
      const int c = idx / k8, k = idx % k8;
      S.Bs[c][k] = (k < kb && c < nc) ? U[(size_t)k + (size_t)(cb + c) * ldu] : 0.0;
    }
    __syncthreads();
    for(int r0 = warp * 16; r0 < m2; r0 += kBW * 16) {
      double acc[8][4];
#pragma unroll
      for(int j = 0; j < 8; ++j)
#pragma unroll
        for(int q = 0; q < 4; ++q) {
          const int r = r0 + g + (q >> 1) * 8, c = j * 8 + 2 * t + (q & 1);
          acc[j][q] = (r < m2 && c < nc) ? C[(size_t)r + (size_t)(cb + c) * ldc] : 0.0;
        }
      for(int kk = 0; kk < k8; kk += 8) {
        double af[4];
        const double* pa = P + (size_t)kb + r0 + g;
        af[0] = kk + t < kb ? -pa[(size_t)(kk + t) * ldp] : 0.0;
        af[1] = kk + t < kb ? -pa[(size_t)(kk + t) * ldp + 8] : 0.0;
        af[2] = kk + t + 4 < kb ? -pa[(size_t)(kk + t + 4) * ldp] : 0.0;
        af[3] = kk + t + 4 < kb ? -pa[(size_t)(kk + t + 4) * ldp + 8] : 0.0;
#pragma unroll
        for(int j = 0; j < 8; ++j) {
          double bf[2];
          bf[0] = S.Bs[j * 8 + g][kk + t];
          bf[1] = S.Bs[j * 8 + g][kk + t + 4];
          dmma(acc[j], af, bf);
        }
      }
#pragma unroll
      for(int j = 0; j < 8; ++j)
#pragma unroll
        for(int q = 0; q < 4; ++q) {
          const int r = r0 + g + (q >> 1) * 8, c = j * 8 + 2 * t + (q & 1);
          if(r < m2 && c < nc) C[(size_t)r + (size_t)(cb + c) * ldc] = acc[j][q];
        }
    }
  }
  __syncthreads();
}

// Factor one system (A n x n, lda = n) and solve for its B (n x nrhs, ldb = n).
HPLB_DEV void solve_system(const Args& a, const Sys& y, double* P, Smem& S) {
  const int n = y.n, nrhs = y.nrhs, nb = y.nb;
  const int ldp = panel_ld(n);
  double*   A  = a.A + y.a_off;
  double*   B  = a.B + y.b_off;
  int*      ip = a.ipiv + y.p_off;
  if(threadIdx.x == 0) S.info = 0;
  for(int k0 = 0; k0 < n; k0 += nb) {
    const int kb = min(nb, n - k0), m = n - k0;
    double*   Ap = A + k0 + (size_t)k0 * n;
    __syncthreads();
    if(kb <= kRegPanelW && m <= 2 * kBT) {
      if(m <= kBT) {
        panel_reg<1, kRegPanelW>(Ap, n, m, kb, k0, ip, P, ldp, S);
      } else {
        panel_reg<2, kRegPanelW>(Ap, n, m, kb, k0, ip, P, ldp, S);
      }
    } else {
    // Panel to shared memory.
    for(int idx = threadIdx.x; idx < kb * m; idx += kBT) {
      const int c = idx / m, i = idx % m;
      P[(size_t)c * ldp + i] = A[(size_t)(k0 + i) + (size_t)(k0 + c) * n];
    }
    __syncthreads();
    for(int j = 0; j < kb; ++j) {
      double* col = P + (size_t)j * ldp;
      double  v   = 0.0;
      int     r   = -1;
      for(int i = j + threadIdx.x; i < m; i += kBT)
        if(better_b(col[i], i, v, r)) {
          v = col[i];
          r = i;
        }
      argmax_block(v, r, S);
      if(threadIdx.x == 0) {
        S.piv[j] = r;
        ip[k0 + j] = k0 + r;
        if(v == 0.0 && S.info == 0) S.info = k0 + j + 1;
      }
      if(r != j && threadIdx.x < kb) {
        double* pc = P + (size_t)threadIdx.x * ldp;
        const double tmp = pc[j];
        pc[j]            = pc[r];
        pc[r]            = tmp;
      }
      __syncthreads();
      if(v != 0.0)
        for(int i = j + 1 + threadIdx.x; i < m; i += kBT) {
          const double l = col[i] / v;
          col[i]         = l;
          for(int c = j + 1; c < kb; ++c) {
            double* pc = P + (size_t)c * ldp;
            pc[i]      = pc[i] - l * pc[j];
          }
        }
      __syncthreads();
    }
    for(int idx = threadIdx.x; idx < kb * m; idx += kBT) {
      const int c = idx / m, i = idx % m;
      A[(size_t)(k0 + i) + (size_t)(k0 + c) * n] = P[(size_t)c * ldp + i];
    }
    }  // shared-memory panel
    // The panel's interchanges as a row map (each thread x < kb traces one
    // position through the kb swaps).
    if(threadIdx.x < kb) {
      const int x = threadIdx.x;
      int       pos = x;
      for(int i = kb - 1; i >= 0; --i) {
        const int p = S.piv[i];
        pos         = (pos == i) ? p : (pos == p ? i : pos);
      }
      S.src[x] = pos;
      pos      = x;
      for(int i = 0; i < kb; ++i) {
        const int p = S.piv[i];
        pos         = (pos == i) ? p : (pos == p ? i : pos);
      }
      S.dst[x] = pos >= kb ? pos : -1;
    }
    load_diag(A + k0 + (size_t)k0 * n, n, kb, S);
    // Interchanges on every other column of A and on B: each thread gathers
    // its column's new top rows into registers before it stores anything.
    const int rest = n - k0 - kb;
    const int ncol = k0 + rest + nrhs;
    for(int q = threadIdx.x; q < ncol; q += kBT) {
      double* col = q < k0 ? A + (size_t)q * n
                           : (q < k0 + rest ? A + (size_t)(q + kb) * n : B + (size_t)(q - k0 - rest) * n);
      col += k0;
      double x[kNbMax];
#pragma unroll
      for(int r = 0; r < kNbMax; ++r)
        if(r < kb) x[r] = col[S.src[r]];
      // The displaced old top rows go below the block (dst >= kb), which no
      // later access of this column reads; 8 loads in flight at a time.
#pragma unroll
      for(int h = 0; h < kNbMax; h += 8) {
        double o[8];
#pragma unroll
        for(int r = 0; r < 8; ++r)
          o[r] = (h + r < kb && S.dst[h + r] >= 0) ? col[h + r] : 0.0;
#pragma unroll
        for(int r = 0; r < 8; ++r)
          if(h + r < kb && S.dst[h + r] >= 0) col[S.dst[h + r]] = o[r];
      }
#pragma unroll
      for(int r = 0; r < kNbMax; ++r)
        if(r < kb) col[r] = x[r];
    }
    __syncthreads();
    // U12 = L11^-1 A12 and the same for B's rows.
    diag_solve<LOWER_UNIT>(kb, A + k0 + (size_t)(k0 + kb) * n, n, rest, S);
    diag_solve<LOWER_UNIT>(kb, B + k0, n, nrhs, S);
    if(rest + nrhs > 0) {
      // A22 -= L21 U12, B2 -= L21 B1 (L21 from the panel copy in shared memory).
      update_strips(P, ldp, kb, rest, A + k0 + (size_t)(k0 + kb) * n, n,
                    A + (k0 + kb) + (size_t)(k0 + kb) * n, n, rest, S);
      update_strips(P, ldp, kb, rest, B + k0, n, B + (k0 + kb), n, nrhs, S);
    }
  }
  // U X = B.
  for(int k0 = (n - 1) / nb * nb; k0 >= 0; k0 -= nb) {
    const int kb = min(nb, n - k0);
    load_diag(A + k0 + (size_t)k0 * n, n, kb, S);
    diag_solve<UPPER>(kb, B + k0, n, nrhs, S);
    tile_gemm_sub(k0, nrhs, kb, A + (size_t)k0 * n, n, B + k0, n, B, n, S);
  }
  if(threadIdx.x == 0) a.info[&y - a.sys] = S.info;
}

// ---- recursive per-system factorisation ----

constexpr int kRecLeaf = 16;  // leaf width of the recursive factorisation
constexpr int kGk      = 32;  // k depth of one staged chunk of gemm_nn_sub

constexpr int kGkStages = 4;  // chunks of gemm_nn_sub in flight

// 8-byte asynchronous global -> shared copy; src_bytes = 0 writes zeros and
// reads nothing (src must still be a valid address).
HPLB_DEV void cp_async8(double* dst, const double* src, int src_bytes) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes)
               : "memory");
}
HPLB_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
HPLB_DEV void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// C (m x n) -= A (m x k) B (k x n), all column-major in global memory, any k:
// 64 x 64 C tiles, each accumulated in DMMA fragments over the whole k (C is
// read and written once per call), operands staged 32 deep in shared memory
// (G: kGkStages buffers of A 32 x 64 and B 64 x 32) by asynchronous copies
// issued kGkStages - 1 chunks ahead of the one being multiplied, so that
// several chunks' global loads are in flight behind the DMMAs.  16 warps in
// 4 x 4, each 16 rows x 16 columns.
__device__ __noinline__ void gemm_nn_sub(int m, int n, int k, const double* A, int64_t lda,
                                         const double* B, int64_t ldb, double* C, int64_t ldc,
                                         double* G) {
  if(m <= 0 || n <= 0 || k <= 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp & 3) * 16, wn = (warp >> 2) * 16;
  constexpr int LDA_S = kTile + 4;  // A stage: [k][row], rows padded
  constexpr int LDB_S = kGk + 4;    // B stage: [col][k], k padded (= 4 mod 16)
  constexpr int STAGE = kGk * LDA_S + kTile * LDB_S;
  const int tm = (m + kTile - 1) / kTile, tn = (n + kTile - 1) / kTile;
  const int nck = (k + kGk - 1) / kGk;
  for(int tile = 0; tile < tm * tn; ++tile) {
    const int m0 = (tile % tm) * kTile, n0 = (tile / tm) * kTile;
    // Chunk ck into buffer ck % kGkStages: each thread copies 4 A and 4 B
    // elements (zeros outside the matrices).
    auto issue = [&](int ck) {
      double* As = G + (ck % kGkStages) * STAGE;
      double* Bs = As + kGk * LDA_S;
#pragma unroll
      for(int q = 0; q < 4; ++q) {
        const int  e  = threadIdx.x + q * kBT;  // 0 .. 2047
        const int  r  = e & (kTile - 1), kk = e >> 6;  // A: 64 rows x 32 k
        const int  gk = ck * kGk + kk;
        const bool ia = m0 + r < m && gk < k;
        cp_async8(As + kk * LDA_S + r, ia ? A + (size_t)(m0 + r) + (size_t)gk * lda : A, ia ? 8 : 0);
        const int  k2  = e & (kGk - 1), c = e >> 5;  // B: 32 k x 64 cols
        const int  gk2 = ck * kGk + k2;
        const bool ib  = n0 + c < n && gk2 < k;
        cp_async8(Bs + c * LDB_S + k2, ib ? B + (size_t)gk2 + (size_t)(n0 + c) * ldb : B,
                  ib ? 8 : 0);
      }
    };
    double acc[2][4];
#pragma unroll
    for(int j = 0; j < 2; ++j)
#pragma unroll
      for(int q = 0; q < 4; ++q) {
        const int r = m0 + wm + g + (q >> 1) * 8, c = n0 + wn + j * 8 + 2 * t + (q & 1);
        acc[j][q] = (r < m && c < n) ? C[(size_t)r + (size_t)c * ldc] : 0.0;
      }
    __syncthreads();  // the previous tile's readers of G are done
#pragma unroll
    for(int s = 0; s < kGkStages - 1; ++s) {
      if(s < nck) issue(s);
      cp_async_commit();
    }
    for(int ck = 0; ck < nck; ++ck) {
      cp_async_wait<kGkStages - 2>();  // this thread's copies of chunk ck have landed
      __syncthreads();  // everyone's have; and chunk ck - 1's buffer is no longer read
      if(ck + kGkStages - 1 < nck) issue(ck + kGkStages - 1);
      cp_async_commit();
      const double* As = G + (ck % kGkStages) * STAGE;
      const double* Bs = As + kGk * LDA_S;
#pragma unroll
      for(int kk = 0; kk < kGk; kk += 8) {
        double af[4];
        af[0] = -As[(kk + t) * LDA_S + wm + g];
        af[1] = -As[(kk + t) * LDA_S + wm + g + 8];
        af[2] = -As[(kk + t + 4) * LDA_S + wm + g];
        af[3] = -As[(kk + t + 4) * LDA_S + wm + g + 8];
#pragma unroll
        for(int j = 0; j < 2; ++j) {
          double bf[2];
          bf[0] = Bs[(wn + j * 8 + g) * LDB_S + kk + t];
          bf[1] = Bs[(wn + j * 8 + g) * LDB_S + kk + t + 4];
          dmma(acc[j], af, bf);
        }
      }
    }
#pragma unroll
    for(int j = 0; j < 2; ++j)
#pragma unroll
      for(int q = 0; q < 4; ++q) {
        const int r = m0 + wm + g + (q >> 1) * 8, c = n0 + wn + j * 8 + 2 * t + (q & 1);
        if(r < m && c < n) C[(size_t)r + (size_t)c * ldc] = acc[j][q];
      }
  }
  cp_async_wait<0>();
  __syncthreads();
}

// One leaf of the recursive factorisation: columns [c0, c0 + w) (w <= 16) of
// rows [c0, n), in registers, then its interchanges on every other column of
// A and of B (full rows, as LAPACK's getrf).
HPLB_DEV void rec_leaf(double* A, double* B, int n, int nrhs, int* ip, int c0, int w, double* P,
                       Smem& S) {
  const int m = n - c0;
  double*   Ap = A + c0 + (size_t)c0 * n;
  const int ldp = panel_ld(n);
  __syncthreads();
  if(m <= kBT)
    panel_reg<1, kRecLeaf>(Ap, n, m, w, c0, ip, P, ldp, S);
  else
    panel_reg<2, kRecLeaf>(Ap, n, m, w, c0, ip, P, ldp, S);
  if(threadIdx.x < w) {
    const int x = threadIdx.x;
    int       pos = x;
    for(int i = w - 1; i >= 0; --i) {
      const int p = S.piv[i];
      pos         = (pos == i) ? p : (pos == p ? i : pos);
    }
    S.src[x] = pos;
    pos      = x;
    for(int i = 0; i < w; ++i) {
      const int p = S.piv[i];
      pos         = (pos == i) ? p : (pos == p ? i : pos);
    }
    S.dst[x] = pos >= w ? pos : -1;
  }
  __syncthreads();
  // Half a warp per column, lane = row of the leaf's top block (w <= 16): the
  // top rows are written as one contiguous segment, and each column's reads
  // all happen before any of its writes (the half-warp's own columns only).
  // A half-warp takes kSwapCols columns per trip, so that many columns' loads
  // are in flight at once.
  constexpr int kSwapCols = 4;
  const int ncol = n - w + nrhs;
  const int hl   = threadIdx.x & 15;
  const int src  = hl < w ? S.src[hl] : 0;
  const int dst  = hl < w ? S.dst[hl] : -1;
  const int half = (threadIdx.x >> 4) & 1;
  // The whole warp iterates together (2 kSwapCols columns per trip), so every
  // lane reaches each __syncwarp; a half-warp past the last column idles.
  for(int q0 = (threadIdx.x >> 5) * 2 * kSwapCols; q0 < ncol; q0 += (kBT / 16) * kSwapCols) {
    double* col[kSwapCols];
    double  v[kSwapCols], o[kSwapCols];
    bool    on[kSwapCols];
#pragma unroll
    for(int i = 0; i < kSwapCols; ++i) {
      const int q = q0 + half + 2 * i;
      on[i]       = q < ncol && hl < w;
      col[i]      = nullptr;
      v[i] = o[i] = 0.0;
      if(on[i]) {
        col[i] = (q < c0 ? A + (size_t)q * n
                         : (q < n - w ? A + (size_t)(q + w) * n : B + (size_t)(q - (n - w)) * n)) +
                 c0;
        v[i] = col[i][src];
        if(dst >= 0) o[i] = col[i][hl];
      }
    }
    __syncwarp();
#pragma unroll
    for(int i = 0; i < kSwapCols; ++i)
      if(on[i]) {
        // The displaced old top rows go below the block (dst >= w).
        if(dst >= 0) col[i][dst] = o[i];
        col[i][hl] = v[i];
      }
    __syncwarp();
  }
  __syncthreads();
}

// Width of the upper half of a node of the recursive triangular solve (w > 32):
// about half, rounded up to whole 32-row diagonal blocks.
HPLB_DEV int trsm_split(int w) {
  const int h = ((w / 2 + kNbMax - 1) / kNbMax) * kNbMax;
  return h < w ? h : w - kNbMax;
}

// X (w1 x ncols, leading dimension ldx) <- L^-1 X for the unit-lower w1 x w1 L
// at L (leading dimension ldl), recursively: the rows split in halves down to
// diagonal blocks of at most 32 rows, each solved by substitution; after a
// node's upper half is solved, its lower half takes X2 -= L21 X1 in one DMMA
// GEMM with k = the upper half's height.  The recursion is walked without a
// stack, as in solve_system_rec: blocks top to bottom, and after the block
// that ends at row pos the one node whose upper half ends at pos updates.
// Each row of X is rewritten once per level (log2(w1 / 32) times) instead of
// once per 32-row block.
HPLB_DEV void trsm_lower_unit(int w1, int ncols, const double* L, int64_t ldl, double* X,
                              int64_t ldx, double* G, Smem& S) {
  if(w1 <= 0 || ncols <= 0) return;
  int pos = 0;
  while(pos < w1) {
    int r0 = 0, h = w1;
    while(h > kNbMax) {  // the diagonal block that starts at pos
      const int h1 = trsm_split(h);
      if(pos < r0 + h1) {
        h = h1;
      } else {
        r0 += h1;
        h -= h1;
      }
    }
    load_diag(L + r0 + (size_t)r0 * ldl, ldl, h, S);
    diag_solve<LOWER_UNIT>(h, X + r0, ldx, ncols, S);
    pos = r0 + h;
    r0 = 0, h = w1;
    while(pos < w1 && h > kNbMax) {  // the node whose upper half ends at pos
      const int h1 = trsm_split(h);
      if(pos == r0 + h1) {
        gemm_nn_sub(h - h1, ncols, h1, L + (r0 + h1) + (size_t)r0 * ldl, ldl, X + r0, ldx,
                    X + r0 + h1, ldx, G);
        break;
      }
      if(pos < r0 + h1) {
        h = h1;
      } else {
        r0 += h1;
        h -= h1;
      }
    }
  }
}

// X (w1 x ncols, leading dimension ldx) <- U^-1 X for the upper-triangular
// w1 x w1 U at U (leading dimension ldu), recursively, the mirror of
// trsm_lower_unit: diagonal blocks bottom to top, and after the block that
// starts at row pos the one node whose lower half starts at pos takes
// X1 -= U12 X2 in one DMMA GEMM.
HPLB_DEV void trsm_upper(int w1, int ncols, const double* U, int64_t ldu, double* X, int64_t ldx,
                         double* G, Smem& S) {
  if(w1 <= 0 || ncols <= 0) return;
  int pos = w1;
  while(pos > 0) {
    int r0 = 0, h = w1;
    while(h > kNbMax) {  // the diagonal block that ends at pos
      const int h1 = trsm_split(h);
      if(pos > r0 + h1) {
        r0 += h1;
        h -= h1;
      } else {
        h = h1;
      }
    }
    load_diag(U + r0 + (size_t)r0 * ldu, ldu, h, S);
    diag_solve<UPPER>(h, X + r0, ldx, ncols, S);
    pos = r0;
    r0 = 0, h = w1;
    while(pos > 0 && h > kNbMax) {  // the node whose lower half starts at pos
      const int h1 = trsm_split(h);
      if(pos == r0 + h1) {
        gemm_nn_sub(h1, ncols, h - h1, U + r0 + (size_t)(r0 + h1) * ldu, ldu, X + r0 + h1, ldx,
                    X + r0, ldx, G);
        break;
      }
      if(pos > r0 + h1) {
        r0 += h1;
        h -= h1;
      } else {
        h = h1;
      }
    }
  }
}

// Width of the left half of a node of the recursive factorisation (w > 16):
// about half, rounded up to a whole number of leaves.
HPLB_DEV int rec_split(int w) {
  const int w1 = ((w / 2 + kRecLeaf - 1) / kRecLeaf) * kRecLeaf;
  return w1 < w ? w1 : w - kRecLeaf;
}

// Recursive factorisation of one system (the columns split in halves down to
// 16-wide leaves), then X = U^-1 L^-1 B by blocks (B took every interchange
// as it happened).  The recursion is walked without a stack: the leaves are
// factored left to right, and after the leaf that ends at column pos the one
// node whose left half ends at pos does its update (U12 = L11^-1 A12, then
// A22 -= L21 U12) -- the order of the recursive algorithm.  Both are found
// by a descent from the root, so the walk lives in a few registers.
HPLB_DEV void solve_system_rec(const Args& a, const Sys& y, double* P, double* G, Smem& S) {
  const int n = y.n, nrhs = y.nrhs;
  double*   A  = a.A + y.a_off;
  double*   B  = a.B + y.b_off;
  int*      ip = a.ipiv + y.p_off;
  if(threadIdx.x == 0) S.info = 0;
  int pos = 0;
  while(pos < n) {
    int c0 = 0, w = n;
    while(w > kRecLeaf) {  // the leaf that starts at pos
      const int w1 = rec_split(w);
      if(pos < c0 + w1) {
        w = w1;
      } else {
        c0 += w1;
        w -= w1;
      }
    }
    rec_leaf(A, B, n, nrhs, ip, c0, w, P, S);
    pos = c0 + w;
    c0 = 0, w = n;
    while(pos < n && w > kRecLeaf) {  // the node whose left half ends at pos
      const int w1 = rec_split(w);
      if(pos == c0 + w1) {
        const int w2 = w - w1;
        trsm_lower_unit(w1, w2, A + c0 + (size_t)c0 * n, n, A + c0 + (size_t)(c0 + w1) * n, n,
                        G, S);
        gemm_nn_sub(n - c0 - w1, w2, w1, A + (c0 + w1) + (size_t)c0 * n, n,
                    A + c0 + (size_t)(c0 + w1) * n, n, A + (c0 + w1) + (size_t)(c0 + w1) * n, n,
                    G);
        break;
      }
      if(pos < c0 + w1) {
        w = w1;
      } else {
        c0 += w1;
        w -= w1;
      }
    }
  }
  // L Y = B, then U X = Y, both recursive.
  trsm_lower_unit(n, nrhs, A, n, B, n, G, S);
  trsm_upper(n, nrhs, A, n, B, n, G, S);
  if(threadIdx.x == 0) a.info[&y - a.sys] = S.info;
}

// Dynamic shared memory of the recursive mode: the GEMM's two stages (the
// leaves keep no panel copy).
__host__ __device__ constexpr int rec_stage_doubles() {
  return kGkStages * (kGk * (kTile + 4) + kTile * (kGk + 4));
}

__global__ void __launch_bounds__(kBT, 1) batch_gesv_kernel(const Args* pa) {
  extern __shared__ __align__(16) double panel_smem[];
  __shared__ Smem S;
  const Args a = *pa;
  for(;;) {
    const int s = next_system(a, S);
    if(s < 0) break;
    const Sys& y = a.sys[s];
    if(y.nb == kRecMode)
      solve_system_rec(a, y, nullptr, panel_smem, S);
    else
      solve_system(a, y, panel_smem, S);
  }
}

// ---- solves with stored factors ----

// Rows of B (n x nrhs, leading dimension n) permuted by the pivots: forward,
// B <- P B (the swaps j = 0 .. n-1 in order), or inverse, B <- P^T B.  The
// permutation is traced once on an index array in shared memory (idx[i] =
// original row now at position i), then applied as a gather through shared
// memory, kPermCols columns at a time.
constexpr int kPermCols = 8;
HPLB_DEV void permute_rows(const int* ip, int n, double* B, int nrhs, bool inverse, int* idx,
                           double* T) {
  for(int i = threadIdx.x; i < n; i += kBT) idx[i] = ip[i];
  __syncthreads();
  if(threadIdx.x == 0) {
    // idx[] holds the pivots; trace positions in place with a second pass.
    int* pv = idx;
    // positions are rebuilt into the upper half of the same buffer
    int* pos = idx + n;
    for(int i = 0; i < n; ++i) pos[i] = i;
    for(int j = 0; j < n; ++j) {
      const int r = pv[j];
      if(r != j && r >= 0 && r < n) {
        const int t = pos[j];
        pos[j]      = pos[r];
        pos[r]      = t;
      }
    }
  }
  __syncthreads();
  const int* pos = idx + n;
  for(int c0 = 0; c0 < nrhs; c0 += kPermCols) {
    const int nc = min(kPermCols, nrhs - c0);
    for(int e = threadIdx.x; e < nc * n; e += kBT) {
      const int c = e / n, i = e % n;
      const double* col = B + (size_t)(c0 + c) * n;
      if(!inverse)
        T[(size_t)c * n + i] = col[pos[i]];
      else
        T[(size_t)c * n + pos[i]] = col[i];
    }
    __syncthreads();
    for(int e = threadIdx.x; e < nc * n; e += kBT) {
      const int c = e / n, i = e % n;
      B[(size_t)i + (size_t)(c0 + c) * n] = T[(size_t)c * n + i];
    }
    __syncthreads();
  }
}

template <bool TRANS>
__global__ void __launch_bounds__(kBT, 1) batch_getrs_kernel(const Args* pa) {
  extern __shared__ __align__(16) double perm_smem[];
  __shared__ Smem S;
  const Args a = *pa;
  for(;;) {
    const int s = next_system(a, S);
    if(s < 0) break;
    const Sys&    y = a.sys[s];
    const int     n = y.n, nrhs = y.nrhs, nb = y.nb;
    const double* L = a.LU + y.a_off;
    double*       B = a.B + y.b_off;
    const int*    ip = a.ipivc + y.p_off;
    int*          idx = reinterpret_cast<int*>(perm_smem);
    double*       T   = perm_smem + n;  // after 2n ints
    if(!TRANS) {
      // x = U^-1 L^-1 P b
      permute_rows(ip, n, B, nrhs, false, idx, T);
      for(int k0 = 0; k0 < n; k0 += nb) {
        const int kb = min(nb, n - k0);
        load_diag(L + k0 + (size_t)k0 * n, n, kb, S);
        diag_solve<LOWER_UNIT>(kb, B + k0, n, nrhs, S);
        tile_gemm_sub(n - k0 - kb, nrhs, kb, L + (k0 + kb) + (size_t)k0 * n, n, B + k0, n,
                      B + k0 + kb, n, S);
      }
      for(int k0 = (n - 1) / nb * nb; k0 >= 0; k0 -= nb) {
        const int kb = min(nb, n - k0);
        load_diag(L + k0 + (size_t)k0 * n, n, kb, S);
        diag_solve<UPPER>(kb, B + k0, n, nrhs, S);
        tile_gemm_sub(k0, nrhs, kb, L + (size_t)k0 * n, n, B + k0, n, B, n, S);
      }
    } else {
      // x = P^T L^-T U^-T b
      for(int k0 = 0; k0 < n; k0 += nb) {
        const int kb = min(nb, n - k0);
        tile_gemm_tn_sub(kb, nrhs, k0, L + (size_t)k0 * n, n, B, n, B + k0, n, S);
        load_diag(L + k0 + (size_t)k0 * n, n, kb, S);
        diag_solve<UPPER_T>(kb, B + k0, n, nrhs, S);
      }
      for(int k0 = (n - 1) / nb * nb; k0 >= 0; k0 -= nb) {
        const int kb = min(nb, n - k0);
        tile_gemm_tn_sub(kb, nrhs, n - k0 - kb, L + (k0 + kb) + (size_t)k0 * n, n, B + k0 + kb,
                         n, B + k0, n, S);
        load_diag(L + k0 + (size_t)k0 * n, n, kb, S);
        diag_solve<LOWER_UNIT_T>(kb, B + k0, n, nrhs, S);
      }
      permute_rows(ip, n, B, nrhs, true, idx, T);
    }
  }
}


// C_i = alpha X_i Y_i^T for every system (X_i, Y_i n_i x nrhs_i in the B-pool
// layout, C_i n_i x n_i in the A-pool layout): 64 x 64 output tiles, the
// nrhs-long slices of X and Y staged in shared memory (k <= 64 in two halves),
// each thread 2 x 4 outputs, streaming stores.
__global__ void __launch_bounds__(kBT, 1) batch_rank_k_kernel(const Args* pa) {
  __shared__ Smem S;
  const Args a = *pa;
  const int  tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // rows tx + 32 i, cols ty + 16 j
  for(;;) {
    const int s = next_system(a, S);
    if(s < 0) break;
    const Sys&    y = a.sys[s];
    const int     n = y.n, k = y.nrhs;
    const double* X = a.X + y.b_off;
    const double* Yp = a.Y + y.b_off;
    double*       C = a.C + y.a_off;
    const int     tn = (n + kTile - 1) / kTile;
    for(int tile = 0; tile < tn * tn; ++tile) {
      const int m0 = (tile % tn) * kTile, n0 = (tile / tn) * kTile;
      double acc[2][4] = {};
      for(int k0 = 0; k0 < k; k0 += kNbMax) {
        const int kc = min(kNbMax, k - k0);
        __syncthreads();
        for(int idx = threadIdx.x; idx < kNbMax * kTile; idx += kBT) {
          const int r = idx % kTile, kk = idx / kTile;
          S.As[kk][r] = (kk < kc && m0 + r < n) ? X[(size_t)(m0 + r) + (size_t)(k0 + kk) * n] : 0.0;
          S.Bs[r][kk] = (kk < kc && n0 + r < n) ? Yp[(size_t)(n0 + r) + (size_t)(k0 + kk) * n] : 0.0;
        }
        __syncthreads();
        for(int kk = 0; kk < kc; ++kk) {
          double xa[2], yb[4];
#pragma unroll
          for(int i = 0; i < 2; ++i) xa[i] = S.As[kk][tx + 32 * i];
#pragma unroll
          for(int j = 0; j < 4; ++j) yb[j] = S.Bs[ty + 16 * j][kk];
#pragma unroll
          for(int i = 0; i < 2; ++i)
#pragma unroll
            for(int j = 0; j < 4; ++j) acc[i][j] = fma(xa[i], yb[j], acc[i][j]);
        }
      }
#pragma unroll
      for(int j = 0; j < 4; ++j) {
        const int c = n0 + ty + 16 * j;
#pragma unroll
        for(int i = 0; i < 2; ++i) {
          const int r = m0 + tx + 32 * i;
          if(r < n && c < n) __stcs(C + (size_t)r + (size_t)c * n, a.alpha * acc[i][j]);
        }
      }
    }
  }
}

// LCG of one system: [A_i | B_i] = HPL_pdrandmat(n_i, n_i + nrhs_i, seed_i)
// with m = n_i rows, i.e. entry (r, c) is X(1 + r + c n_i); columns >= n_i are
// B_i.  Thread per row: the row's first state by the binary jump table, then a
// jump of n_i per column.
HPLB_DEV uint64_t state_of(uint64_t x1, uint64_t k, const Jump* pow2) {
  Jump acc{1, 0};
  for(int b = 0; k; ++b, k >>= 1)
    if(k & 1) acc = compose(acc, pow2[b]);
  return apply(acc, x1);
}

__global__ void __launch_bounds__(kBT, 1) batch_matgen_kernel(const Args* pa) {
  __shared__ Smem S;
  __shared__ Jump pow2[64];
  __shared__ Jump jn;
  const Args a = *pa;
  if(threadIdx.x == 0) {
    Jump p{kLcgMult, kLcgAdd};
    for(int b = 0; b < 64; ++b) {
      pow2[b] = p;
      p       = compose(p, p);
    }
  }
  for(;;) {
    const int s = next_system(a, S);
    if(s < 0) break;
    const Sys& y = a.sys[s];
    const int  n = y.n;
    if(threadIdx.x == 0) jn = jump_by((uint64_t)n);
    __syncthreads();
    const uint64_t x1 = kLcgMult * a.seeds[s] + kLcgAdd;
    double*        A  = a.A + y.a_off;
    double*        B  = a.B + y.b_off;
    for(int r = threadIdx.x; r < n; r += kBT) {
      uint64_t st = state_of(x1, (uint64_t)r, pow2);
      for(int c = 0; c < n + y.nrhs; ++c) {
        const double v = lcg_value(st);
        if(c < n)
          A[(size_t)r + (size_t)c * n] = v;
        else
          B[(size_t)r + (size_t)(c - n) * n] = v;
        st = apply(jn, st);
      }
    }
  }
}

// HPL scaled residual of every system against its regenerated [A_i | B_i]:
// per right-hand side c, ||B_c - A X_c||oo / (eps (||A||oo ||X_c||oo +
// ||B_c||oo) n) with eps = 2^-53 (src/HPL_pdtest.cpp:330-438); resid[i] is the
// largest over the system's right-hand sides.  X_c is staged in shared memory
// kPermCols columns at a time; A is regenerated for each group.
__global__ void __launch_bounds__(kBT, 1) batch_residual_kernel(const Args* pa) {
  extern __shared__ __align__(16) double xs[];
  __shared__ Smem S;
  __shared__ Jump pow2[64];
  __shared__ Jump jn;
  __shared__ double s_worst;
  const Args a = *pa;
  if(threadIdx.x == 0) {
    Jump p{kLcgMult, kLcgAdd};
    for(int b = 0; b < 64; ++b) {
      pow2[b] = p;
      p       = compose(p, p);
    }
  }
  for(;;) {
    const int s = next_system(a, S);
    if(s < 0) break;
    const Sys&    y = a.sys[s];
    const int     n = y.n, nrhs = y.nrhs;
    const double* X = a.X + y.b_off;
    if(threadIdx.x == 0) {
      jn      = jump_by((uint64_t)n);
      s_worst = 0.0;
    }
    __syncthreads();
    const uint64_t x1 = kLcgMult * a.seeds[s] + kLcgAdd;
    for(int c0 = 0; c0 < nrhs; c0 += kPermCols) {
      const int nc = min(kPermCols, nrhs - c0);
      for(int e = threadIdx.x; e < nc * n; e += kBT) xs[e] = X[(size_t)c0 * n + e];
      __syncthreads();
      double rmax[kPermCols], bmax[kPermCols], xmax[kPermCols], amax = 0.0;
#pragma unroll
      for(int c = 0; c < kPermCols; ++c) rmax[c] = bmax[c] = xmax[c] = 0.0;
      for(int r = threadIdx.x; r < n; r += kBT) {
        uint64_t st = state_of(x1, (uint64_t)r, pow2);
        double   dot[kPermCols], rs = 0.0;
#pragma unroll
        for(int c = 0; c < kPermCols; ++c) dot[c] = 0.0;
        for(int j = 0; j < n; ++j) {
          const double v = lcg_value(st);
          rs += fabs(v);
#pragma unroll
          for(int c = 0; c < kPermCols; ++c)
            if(c < nc) dot[c] = fma(v, xs[(size_t)c * n + j], dot[c]);
          st = apply(jn, st);
        }
        amax = fmax(amax, rs);
        // skip to the right-hand side columns c0 ..
        uint64_t sb = state_of(x1, (uint64_t)r + (uint64_t)(n + c0) * (uint64_t)n, pow2);
#pragma unroll
        for(int c = 0; c < kPermCols; ++c)
          if(c < nc) {
            const double b = lcg_value(sb);
            rmax[c]        = fmax(rmax[c], fabs(b - dot[c]));
            bmax[c]        = fmax(bmax[c], fabs(b));
            xmax[c]        = fmax(xmax[c], fabs(xs[(size_t)c * n + r]));
            sb             = apply(jn, sb);
          }
      }
      // Block maxima (row sums, then per column r, b, x).
      double v = amax;
      for(int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
      __syncthreads();
      if((threadIdx.x & 31) == 0) S.red_v[threadIdx.x >> 5] = v;
      __syncthreads();
      double an = 0.0;
      for(int w = 0; w < kBW; ++w) an = fmax(an, S.red_v[w]);
      for(int c = 0; c < nc; ++c) {
        double m3[3] = {rmax[c], bmax[c], xmax[c]};
        double out[3];
        for(int q = 0; q < 3; ++q) {
          double t = m3[q];
          for(int off = 16; off > 0; off >>= 1) t = fmax(t, __shfl_down_sync(0xffffffffu, t, off));
          __syncthreads();
          if((threadIdx.x & 31) == 0) S.red_v[threadIdx.x >> 5] = t;
          __syncthreads();
          double u = 0.0;
          for(int w = 0; w < kBW; ++w) u = fmax(u, S.red_v[w]);
          out[q] = u;
        }
        if(threadIdx.x == 0) {
          const double eps = 0x1p-53;
          const double res = out[0] / (eps * (an * out[2] + out[1]) * (double)n);
          s_worst          = fmax(s_worst, res);
        }
      }
      __syncthreads();
    }
    if(threadIdx.x == 0) a.resid[s] = s_worst;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Launchers (the plan in batch_api.cu sizes the shared memory and the grid).
// ---------------------------------------------------------------------------

size_t batch_static_smem() { return sizeof(Smem); }
size_t batch_rec_stage_bytes() { return (size_t)rec_stage_doubles() * sizeof(double); }
int    batch_threads() { return kBT; }
int    batch_nb_max() { return kNbMax; }

// Raise every dynamic-shared-memory kernel's limit to what its own static
// shared memory leaves of the per-block opt-in maximum; *budget = the
// smallest of those limits (what a plan may use in every mode).
cudaError_t batch_set_smem(size_t* budget) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if(e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if(e != cudaSuccess) return e;
  const void* fns[4] = {(const void*)batch_gesv_kernel, (const void*)batch_getrs_kernel<false>,
                        (const void*)batch_getrs_kernel<true>, (const void*)batch_residual_kernel};
  size_t lowest = (size_t)optin;
  for(const void* f : fns) {
    cudaFuncAttributes fa{};
    if((e = cudaFuncGetAttributes(&fa, f)) != cudaSuccess) return e;
    const int lim = optin - (int)fa.sharedSizeBytes;
    if(lim <= 0) return cudaErrorInvalidValue;
    if((e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, lim)) !=
       cudaSuccess)
      return e;
    lowest = std::min(lowest, (size_t)lim);
  }
  *budget = lowest;
  return cudaSuccess;
}

// mode: 0 gesv, 1 getrs, 2 getrs transposed, 3 rank-k, 4 matgen, 5 residual.
cudaError_t launch_batch(int mode, const void* d_args, int grid, size_t dyn_bytes,
                         cudaStream_t st) {
  const Args* pa = static_cast<const Args*>(d_args);
  switch(mode) {
    case 0: batch_gesv_kernel<<<grid, kBT, dyn_bytes, st>>>(pa); break;
    case 1: batch_getrs_kernel<false><<<grid, kBT, dyn_bytes, st>>>(pa); break;
    case 2: batch_getrs_kernel<true><<<grid, kBT, dyn_bytes, st>>>(pa); break;
    case 3: batch_rank_k_kernel<<<grid, kBT, 0, st>>>(pa); break;
    case 4: batch_matgen_kernel<<<grid, kBT, 0, st>>>(pa); break;
    case 5: batch_residual_kernel<<<grid, kBT, dyn_bytes, st>>>(pa); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

size_t batch_args_bytes() { return sizeof(Args); }

void batch_fill_args(void* host_args, double* A, const double* LU, double* B, int* ipiv,
                     const int* ipivc, int* info, const void* sys, const int* order, int count,
                     int* counter, double alpha, const double* X, const double* Y, double* C,
                     const unsigned long long* seeds, double* resid) {
  Args* a    = static_cast<Args*>(host_args);
  a->A       = A;
  a->LU      = LU;
  a->B       = B;
  a->ipiv    = ipiv;
  a->ipivc   = ipivc;
  a->info    = info;
  a->sys     = static_cast<const Sys*>(sys);
  a->order   = order;
  a->count   = count;
  a->counter = counter;
  a->alpha   = alpha;
  a->X       = X;
  a->Y       = Y;
  a->C       = C;
  a->seeds   = seeds;
  a->resid   = resid;
}

size_t batch_sys_bytes() { return sizeof(Sys); }
void   batch_fill_sys(void* dst, int i, int n, int nrhs, int nb, long long a_off, long long b_off,
                      long long p_off) {
  Sys* y   = static_cast<Sys*>(dst) + i;
  y->n     = n;
  y->nrhs  = nrhs;
  y->nb    = nb;
  y->pad   = 0;
  y->a_off = a_off;
  y->b_off = b_off;
  y->p_off = p_off;
}

}  // namespace hplb
