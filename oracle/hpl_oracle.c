/*
 * hpl_oracle.c -- CPU restatement of rocHPL's single-process (P = Q = 1) solve
 * path: LCG matrix generation, blocked right-looking LU with recursive panel
 * factorisation and partial pivoting, the back-solve, and the HPL scaled
 * residual.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA path is compared
 * against (pytest, the smoke check and the CPU-baseline leg of bench.py); the
 * product library never links it and has no CPU fallback.
 *
 * Pinning: the LCG is checked bit-for-bit against rocHPL's own hpl_randmat
 * kernel and HPL_xjumpm (built from the reference sources by build_ref.sh), and
 * the permutation map against rocHPL's own HPL_pipid.  The LU itself relies on
 * rocBLAS in the reference and cannot be built here; its parity is anchored on
 * the HPL scaled residual (< 16) plus exact pivot agreement with this file.
 *
 * Level-3 work can be routed to an external BLAS (hplo_use_blas) so the same
 * restatement doubles as the timed host-BLAS baseline; the scalar loops are
 * used otherwise.  Build with -ffp-contract=off: the LCG value expression is
 * evaluated in source order with no fused multiply-add.
 */
#include <dlfcn.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define HPLO_MULT 6364136223846793005ULL /* include/hpl_pmatgen.hpp:35 */
#define HPLO_IADD 1ULL                   /* include/hpl_pmatgen.hpp:36 */
#define HPLO_DIVFAC 2147483648.0         /* include/hpl_pmatgen.hpp:37 */
#define HPLO_POW16 65536.0               /* include/hpl_pmatgen.hpp:38 */
#define HPLO_HALF 0.5                    /* include/hpl_pmatgen.hpp:39 */

#define A_(i, j) A[(size_t)(i) + (size_t)(j) * (size_t)ld]

/* ------------------------------------------------------------------------ */
/* LCG                                                                        */
/* ------------------------------------------------------------------------ */

/* Constants (a, c) with X(n+k) = a X(n) + c, by repeated squaring.  Same values
 * as the O(k) loop of src/matgen/HPL_xjumpm.cpp:81-91 (mod 2^64). */
void hplo_jump(uint64_t k, uint64_t* a_out, uint64_t* c_out) {
  uint64_t a = 1, c = 0;          /* accumulated jump */
  uint64_t pa = HPLO_MULT, pc = HPLO_IADD; /* jump by 2^bit */
  while(k) {
    if(k & 1) {
      a = pa * a;
      c = pa * c + pc;
    }
    pc = pa * pc + pc;
    pa = pa * pa;
    k >>= 1;
  }
  *a_out = a;
  *c_out = c;
}

/* One matrix entry from an LCG state, in the operation order of
 * src/matgen/HPL_pdrandmat_device.cpp:65-73. */
double hplo_lcg_value(uint64_t r) {
  const double p1 = (double)((r >> 0) & 65535ULL);
  const double p2 = (double)((r >> 16) & 65535ULL);
  const double p3 = (double)((r >> 32) & 65535ULL);
  const double p4 = (double)((r >> 48) & 65535ULL);
  double t = p1 + p2 * HPLO_POW16;
  t        = t / HPLO_DIVFAC * HPLO_HALF;
  t        = t + p3;
  t        = t + p4 * HPLO_POW16;
  return HPLO_HALF - t / HPLO_DIVFAC * HPLO_HALF;
}

/* State index of entry (i, j) of an M-row matrix at P = Q = 1: the generator
 * starts one step after the seed and walks down columns
 * (src/matgen/HPL_pdrandmat_device.cpp:138-175). */
uint64_t hplo_lcg_state(uint64_t seed, int64_t M, int64_t i, int64_t j) {
  uint64_t a, c;
  hplo_jump((uint64_t)(1 + i + j * M), &a, &c);
  return a * seed + c;
}

/* HPL_pdrandmat at P = Q = 1: the M x N matrix, column-major, leading dim ld. */
void hplo_matgen(int M, int N, uint64_t seed, double* A, int64_t ld) {
  uint64_t ac, cc; /* one column */
  hplo_jump((uint64_t)M, &ac, &cc);
  uint64_t col = HPLO_MULT * seed + HPLO_IADD;
  for(int j = 0; j < N; ++j) {
    uint64_t r = col;
    for(int i = 0; i < M; ++i) {
      A_(i, j) = hplo_lcg_value(r);
      r        = HPLO_MULT * r + HPLO_IADD;
    }
    col = ac * col + cc;
  }
}

/* Rows [i0, i0 + m) x columns [j0, j0 + n) of the M-row matrix of hplo_matgen:
 * the local block a process of a P x Q grid generates in HPL_pdrandmat
 * (src/matgen/HPL_pdrandmat_device.cpp:136-175), entry (i, j) being state
 * X(1 + (i0 + i) + (j0 + j) M). */
void hplo_matgen_block(int64_t M, int64_t i0, int64_t j0, int m, int n, uint64_t seed,
                       double* A, int64_t ld) {
  uint64_t ac, cc; /* one column */
  hplo_jump((uint64_t)M, &ac, &cc);
  uint64_t col = hplo_lcg_state(seed, M, i0, j0);
  for(int j = 0; j < n; ++j) {
    uint64_t r = col;
    for(int i = 0; i < m; ++i) {
      A_(i, j) = hplo_lcg_value(r);
      r        = HPLO_MULT * r + HPLO_IADD;
    }
    col = ac * col + cc;
  }
}

/* FNV-1a over the bit patterns of the M x N block, column by column: a cheap
 * fingerprint for the golden files. */
uint64_t hplo_hash(int M, int N, const double* A, int64_t ld) {
  uint64_t h = 1469598103934665603ULL;
  for(int j = 0; j < N; ++j)
    for(int i = 0; i < M; ++i) {
      uint64_t b;
      memcpy(&b, &A_(i, j), 8);
      for(int k = 0; k < 8; ++k) {
        h ^= (b >> (8 * k)) & 0xff;
        h *= 1099511628211ULL;
      }
    }
  return h;
}

/* ------------------------------------------------------------------------ */
/* Optional host BLAS (for the timed baseline)                                */
/* ------------------------------------------------------------------------ */

typedef void (*dgemm_fn)(const char*, const char*, const int*, const int*,
                         const int*, const double*, const double*, const int*,
                         const double*, const int*, const double*, double*,
                         const int*);
typedef void (*dtrsm_fn)(const char*, const char*, const char*, const char*,
                         const int*, const int*, const double*, const double*,
                         const int*, double*, const int*);
typedef void (*setthreads_fn)(int);

static dgemm_fn g_dgemm = NULL;
static dtrsm_fn g_dtrsm = NULL;

/* Load an LP64 Fortran-convention BLAS (dgemm/dtrsm symbols, optionally with
 * a prefix such as "scipy_") and set its thread count.  Returns 0 on success. */
int hplo_use_blas(const char* path, const char* prefix, int nthreads) {
  if(!path) {
    g_dgemm = NULL;
    g_dtrsm = NULL;
    return 0;
  }
  void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if(!h) return 1;
  char name[128];
  snprintf(name, sizeof name, "%sdgemm_", prefix ? prefix : "");
  g_dgemm = (dgemm_fn)dlsym(h, name);
  snprintf(name, sizeof name, "%sdtrsm_", prefix ? prefix : "");
  g_dtrsm = (dtrsm_fn)dlsym(h, name);
  snprintf(name, sizeof name, "%sopenblas_set_num_threads", prefix ? prefix : "");
  setthreads_fn st = (setthreads_fn)dlsym(h, name);
  if(st && nthreads > 0) st(nthreads);
  if(!g_dgemm || !g_dtrsm) {
    g_dgemm = NULL;
    g_dtrsm = NULL;
    return 2;
  }
  return 0;
}

/* C(m x n) -= A(m x k) * B(k x n), all column-major. */
static void gemm_sub(int m, int n, int k, const double* A, int64_t lda,
                     const double* B, int64_t ldb, double* C, int64_t ldc) {
  if(m <= 0 || n <= 0 || k <= 0) return;
  if(g_dgemm) {
    const double mone = -1.0, one = 1.0;
    int ilda = (int)lda, ildb = (int)ldb, ildc = (int)ldc;
    g_dgemm("N", "N", &m, &n, &k, &mone, A, &ilda, B, &ildb, &one, C, &ildc);
    return;
  }
  for(int j = 0; j < n; ++j)
    for(int l = 0; l < k; ++l) {
      const double b = B[(size_t)l + (size_t)j * ldb];
      if(b == 0.0) continue;
      const double* a = A + (size_t)l * lda;
      double*       c = C + (size_t)j * ldc;
      for(int i = 0; i < m; ++i) c[i] -= a[i] * b;
    }
}

/* B(m x n) := L^-1 B, L unit lower triangular m x m (left side). */
static void trsm_llu(int m, int n, const double* L, int64_t ldl, double* B,
                     int64_t ldb) {
  if(m <= 0 || n <= 0) return;
  if(g_dtrsm) {
    const double one = 1.0;
    int il = (int)ldl, ib = (int)ldb;
    g_dtrsm("L", "L", "N", "U", &m, &n, &one, L, &il, B, &ib);
    return;
  }
  for(int j = 0; j < n; ++j) {
    double* b = B + (size_t)j * ldb;
    for(int k = 0; k < m; ++k) {
      const double bk = b[k];
      if(bk == 0.0) continue;
      const double* l = L + (size_t)k * ldl;
      for(int i = k + 1; i < m; ++i) b[i] -= l[i] * bk;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* LU                                                                         */
/* ------------------------------------------------------------------------ */

typedef struct {
  double* A;
  int64_t ld;
  int     pr, pc, pw; /* panel: first row, first column, width */
  int     nbmin, ndiv, pfact, rfact;
  int*    ipiv;  /* global pivot rows, indexed by global column */
  int     info;  /* first zero-pivot column (1-based), 0 if none */
} panel_t;

/* Swap global rows r1, r2 over the panel's columns. */
static void panel_swap(panel_t* P, int r1, int r2) {
  if(r1 == r2) return;
  double* A  = P->A;
  int64_t ld = P->ld;
  for(int c = P->pc; c < P->pc + P->pw; ++c) {
    double t  = A_(r1, c);
    A_(r1, c) = A_(r2, c);
    A_(r2, c) = t;
  }
}

/* Pivot search: the first row of largest |a| in column c over rows [r, end).
 * The reference's scans use a strict '>' (src/pfact/HPL_pdpanrlT_device.cpp:
 * 164-171, include/hpl_hip_ex.hpp:689-820), so the lowest row wins ties here. */
static int pivot_row(panel_t* P, int c, int r, int end) {
  double* A   = P->A;
  int64_t ld  = P->ld;
  int     loc = r;
  double  mx  = 0.0;
  for(int i = r; i < end; ++i) {
    const double v = A_(i, c);
    if(fabs(v) > fabs(mx)) {
      mx  = v;
      loc = i;
    }
  }
  return loc;
}

/* Record the pivot, swap, and scale column c below the diagonal row d (the
 * per-column core of every leaf; src/pfact/HPL_pdmxswp.cpp:121 and
 * src/pfact/HPL_pdpanrlT_device.cpp:221-232). */
static void pivot_scale(panel_t* P, int c, int d, int end) {
  double* A  = P->A;
  int64_t ld = P->ld;
  int     p  = pivot_row(P, c, d, end);
  P->ipiv[c] = p;
  panel_swap(P, d, p);
  const double piv = A_(d, c);
  if(piv == 0.0 && P->info == 0) P->info = c + 1;
  for(int i = d + 1; i < end; ++i) A_(i, c) = A_(i, c) / piv;
}

/* Leaf, right-looking: rows [r0, end), columns [c0, c0+n).
 * src/pfact/HPL_pdpanrlT_device.cpp:147-319. */
static void leaf_right(panel_t* P, int r0, int end, int c0, int n) {
  double* A  = P->A;
  int64_t ld = P->ld;
  for(int k = 0; k < n; ++k) {
    const int c = c0 + k, d = r0 + k;
    pivot_scale(P, c, d, end);
    for(int cc = c + 1; cc < c0 + n; ++cc) {
      const double u = A_(d, cc);
      for(int i = d + 1; i < end; ++i) A_(i, cc) -= A_(i, c) * u;
    }
  }
}

/* Leaf, left-looking: column k is brought up to date by all previous leaf
 * columns just before its pivot search.  src/pfact/HPL_pdpanllT_device.cpp. */
static void leaf_left(panel_t* P, int r0, int end, int c0, int n) {
  double* A  = P->A;
  int64_t ld = P->ld;
  for(int k = 0; k < n; ++k) {
    const int c = c0 + k, d = r0 + k;
    /* U part of column c: forward substitution with the leaf's unit L. */
    for(int kk = 0; kk < k; ++kk) {
      const double u = A_(r0 + kk, c);
      for(int i = r0 + kk + 1; i < r0 + k; ++i) A_(i, c) -= A_(i, c0 + kk) * u;
    }
    /* Rest of column c. */
    for(int kk = 0; kk < k; ++kk) {
      const double u = A_(r0 + kk, c);
      for(int i = d; i < end; ++i) A_(i, c) -= A_(i, c0 + kk) * u;
    }
    pivot_scale(P, c, d, end);
  }
}

/* Leaf, Crout: row d of U and column c of L are both brought up to date at
 * step k (src/pfact/HPL_pdpancrT_device.cpp). */
static void leaf_crout(panel_t* P, int r0, int end, int c0, int n) {
  double* A  = P->A;
  int64_t ld = P->ld;
  for(int k = 0; k < n; ++k) {
    const int c = c0 + k, d = r0 + k;
    for(int kk = 0; kk < k; ++kk) {
      const double u = A_(r0 + kk, c);
      for(int i = d; i < end; ++i) A_(i, c) -= A_(i, c0 + kk) * u;
    }
    pivot_scale(P, c, d, end);
    /* Row d of U over the remaining leaf columns. */
    for(int cc = c + 1; cc < c0 + n; ++cc)
      for(int kk = 0; kk < k; ++kk) A_(d, cc) -= A_(d, c0 + kk) * A_(r0 + kk, cc);
  }
}

static void leaf(panel_t* P, int r0, int end, int c0, int n) {
  if(P->pfact == 0)
    leaf_left(P, r0, end, c0, n);
  else if(P->pfact == 1)
    leaf_crout(P, r0, end, c0, n);
  else
    leaf_right(P, r0, end, c0, n);
}

/* Recursive panel factorisation of rows [r0, end) x columns [c0, c0+N).
 * Right-looking split: src/pfact/HPL_pdrpanrlT.cpp:74-160; the piece width
 * is jb = ceil(ceil(N/NBMIN)/NDIV)*NBMIN (:93).  The left-looking and Crout
 * recursions (HPL_pdrpanllT.cpp:116-159, HPL_pdrpancrT.cpp:116-175) bring each
 * piece up to date just before factoring it instead of right after the
 * previous one; in exact arithmetic all three give the same factors. */
static void rpanel(panel_t* P, int r0, int end, int c0, int N) {
  if(N <= P->nbmin) {
    leaf(P, r0, end, c0, N);
    return;
  }
  double* A  = P->A;
  int64_t ld = P->ld;
  const int nbs = (((N + P->nbmin - 1) / P->nbmin + P->ndiv - 1) / P->ndiv) * P->nbmin;
  if(P->rfact == 2) { /* right-looking */
    int jj = 0, n = N, jb = nbs;
    do {
      n -= jb;
      rpanel(P, r0 + jj, end, c0 + jj, jb);
      /* U of the trailing panel columns, then the panel-local update. */
      trsm_llu(jb, n, &A_(r0 + jj, c0 + jj), ld, &A_(r0 + jj, c0 + jj + jb), ld);
      gemm_sub(end - (r0 + jj + jb), n, jb, &A_(r0 + jj + jb, c0 + jj), ld,
               &A_(r0 + jj, c0 + jj + jb), ld, &A_(r0 + jj + jb, c0 + jj + jb), ld);
      jj += jb;
      jb = n < nbs ? n : nbs;
    } while(n > 0);
  } else { /* left-looking (0) and Crout (1): update piece, then factor */
    int jj = 0, n = N, jb = nbs;
    do {
      n -= jb;
      const int cj = c0 + jj;
      if(jj > 0) {
        /* U rows of the piece from all previous pieces, then the rest. */
        trsm_llu(jj, jb, &A_(r0, c0), ld, &A_(r0, cj), ld);
        gemm_sub(end - (r0 + jj), jb, jj, &A_(r0 + jj, c0), ld, &A_(r0, cj), ld,
                 &A_(r0 + jj, cj), ld);
      }
      rpanel(P, r0 + jj, end, cj, jb);
      jj += jb;
      jb = n < nbs ? n : nbs;
    } while(n > 0);
    (void)A;
  }
}

/* HPL_pdfact for one process of a 1 x Q grid (P = 1: the process holds every
 * row of its columns): factor the panel of global rows [j, N) held in local
 * columns [lc, lc + jb) of A, with the recursion and leaf of rpanel.  ipiv[k]
 * (k < jb) receives the global row swapped into row j + k.  Returns the first
 * zero-pivot global column (1-based), or 0.  src/pfact/HPL_pdfact.cpp:20-110. */
int hplo_panel_factor(int N, int j, int jb, int nbmin, int ndiv, int pfact, int rfact,
                      double* A, int64_t ld, int lc, int* ipiv) {
  panel_t P;
  memset(&P, 0, sizeof P);
  int* piv = (int*)calloc((size_t)(lc + jb > 0 ? lc + jb : 1), sizeof(int));
  P.A     = A;
  P.ld    = ld;
  P.nbmin = nbmin < 1 ? 1 : nbmin;
  P.ndiv  = ndiv < 2 ? 2 : ndiv;
  P.pfact = pfact;
  P.rfact = rfact;
  P.ipiv  = piv; /* indexed by local column */
  P.pr    = j;
  P.pc    = lc;
  P.pw    = jb;
  rpanel(&P, j, N, lc, jb);
  for(int k = 0; k < jb; ++k) ipiv[k] = piv[lc + k];
  free(piv);
  return P.info ? j + (P.info - 1 - lc) + 1 : 0;
}

/* HPL_pdupdateTT for one process of a 1 x Q grid: the panel of global rows
 * [j, N) (jb columns; L(i, k) is global row j + i, leading dimension ldl, unit
 * lower L11 in its top jb rows, L21 below) with pivots ipiv (global rows),
 * applied to local columns [c0, c0 + ncols) of A: the row interchanges in
 * order, U12 = L11^-1 A12, A22 -= L21 U12.  The same operations, per column,
 * as the single-process loop of hplo_pdgesv.  src/pgesv/HPL_pdupdateTT.cpp:91-163,
 * src/pgesv/HPL_pdlaswp.cpp:300-389. */
void hplo_panel_update(int N, int j, int jb, const double* L, int64_t ldl, const int* ipiv,
                       double* A, int64_t ld, int c0, int ncols) {
  for(int k = 0; k < jb; ++k) {
    const int r = j + k, p = ipiv[k];
    if(p == r) continue;
    for(int c = c0; c < c0 + ncols; ++c) {
      double t = A_(r, c);
      A_(r, c) = A_(p, c);
      A_(p, c) = t;
    }
  }
  trsm_llu(jb, ncols, L, ldl, &A_(j, c0), ld);
  gemm_sub(N - (j + jb), ncols, jb, L + jb, ldl, &A_(j, c0), ld, &A_(j + jb, c0), ld);
}

/* Single-process HPL_pdgesv: factor the N x (N+1) [A|b] in place (b in column
 * N), then back-solve U x = y into x.  ipiv[j] receives the global row that
 * was swapped into row j.  Returns info (first zero-pivot column, 1-based).
 * Loop structure: src/pgesv/HPL_pdgesv.cpp:168-362; the look-ahead only
 * reorders independent work, so the panel order here is the same math. */
int hplo_pdgesv(int N, int nb, int nbmin, int ndiv, int pfact, int rfact,
                double* A, int64_t ld, double* x, int* ipiv) {
  panel_t P;
  memset(&P, 0, sizeof P);
  P.A     = A;
  P.ld    = ld;
  P.nbmin = nbmin < 1 ? 1 : nbmin;
  P.ndiv  = ndiv < 2 ? 2 : ndiv;
  P.pfact = pfact;
  P.rfact = rfact;
  P.ipiv  = ipiv;
  for(int j = 0; j < N; j += nb) {
    const int jb = (N - j) < nb ? (N - j) : nb;
    P.pr = j;
    P.pc = j;
    P.pw = jb;
    rpanel(&P, j, N, j, jb);
    /* Row interchanges on the trailing columns, b included
     * (src/pgesv/HPL_pdlaswp.cpp:300-389, HPL_dlaswp00N_device.cpp). */
    for(int k = j; k < j + jb; ++k) {
      const int p = ipiv[k];
      if(p == k) continue;
      for(int c = j + jb; c <= N; ++c) {
        double t = A_(k, c);
        A_(k, c) = A_(p, c);
        A_(p, c) = t;
      }
    }
    /* U12 and the trailing update (src/pgesv/HPL_pdupdateTT.cpp:95-163). */
    const int nt = N + 1 - (j + jb);
    trsm_llu(jb, nt, &A_(j, j), ld, &A_(j, j + jb), ld);
    gemm_sub(N - (j + jb), nt, jb, &A_(j + jb, j), ld, &A_(j, j + jb), ld,
             &A_(j + jb, j + jb), ld);
  }
  /* Back-solve U x = y, y in column N (src/pgesv/HPL_pdtrsv_device.cpp). */
  for(int i = 0; i < N; ++i) x[i] = A_(i, N);
  for(int i = N - 1; i >= 0; --i) {
    x[i] = x[i] / A_(i, i);
    const double xi = x[i];
    for(int r = 0; r < i; ++r) x[r] -= A_(r, i) * xi;
  }
  return P.info;
}

/* ------------------------------------------------------------------------ */
/* Permutation map                                                            */
/* ------------------------------------------------------------------------ */

/* Net row movement of jb sequential interchanges (ia+i <-> ipiv[i]):
 * permU[i] (i < jb) = source row, relative to ia, that lands in row ia+i;
 * permU[jb+s] = destination (relative) of original top row s when it leaves
 * the top block, else -1.  Same map as HPL_pipid + HPL_pdpanel_swapids
 * (src/pgesv/HPL_pipid.cpp:90-163, src/panel/HPL_pdpanel_swapids.cpp:22-44). */
void hplo_swapids(int ia, int jb, const int* ipiv, int* permU) {
  for(int x = 0; x < jb; ++x) {
    int pos = x; /* trace backwards: which original row ends at x */
    for(int i = jb - 1; i >= 0; --i) {
      const int p = ipiv[i] - ia;
      if(pos == i)
        pos = p;
      else if(pos == p)
        pos = i;
    }
    permU[x] = pos;
  }
  for(int s = 0; s < jb; ++s) {
    int pos = s; /* trace forwards: where original top row s ends */
    for(int i = 0; i < jb; ++i) {
      const int p = ipiv[i] - ia;
      if(pos == i)
        pos = p;
      else if(pos == p)
        pos = i;
    }
    permU[jb + s] = pos >= jb ? pos : -1;
  }
}

/* ------------------------------------------------------------------------ */
/* Residual                                                                   */
/* ------------------------------------------------------------------------ */

/* HPL scaled residual on the regenerated [A|b] (src/HPL_pdtest.cpp:307-438):
 * out = {resid, ||b-Ax||oo, ||A||1, ||A||oo, ||x||1, ||x||oo, ||b||oo, eps}.
 * Norms follow src/pauxil/HPL_pdlange_device.cpp:76-116; eps = 2^-53 is
 * HPL_dlamch's relative machine precision under rounding
 * (src/auxil/HPL_dlamch.cpp:104-111).  The residual vector is accumulated in
 * long double to serve as the reference for the device kernel's r. */
void hplo_residual(int N, const double* A, int64_t ld, const double* x,
                   double* out, double* r_out) {
  double anorm1 = 0, anormi = 0, xnorm1 = 0, xnormi = 0, bnormi = 0, rnorm = 0;
  long double* r  = (long double*)calloc((size_t)(N > 0 ? N : 1), sizeof(long double));
  double*      rs = (double*)calloc((size_t)(N > 0 ? N : 1), sizeof(double));
  for(int i = 0; i < N; ++i) r[i] = A_(i, N);
  for(int j = 0; j < N; ++j) {
    double cs = 0;
    const long double xj = x[j];
    for(int i = 0; i < N; ++i) {
      const double a = A_(i, j);
      cs += fabs(a);
      rs[i] += fabs(a);
      r[i] -= (long double)a * xj;
    }
    if(cs > anorm1) anorm1 = cs;
  }
  for(int i = 0; i < N; ++i) {
    if(rs[i] > anormi) anormi = rs[i];
    const double ri = (double)r[i];
    if(r_out) r_out[i] = ri;
    if(fabs(ri) > rnorm) rnorm = fabs(ri);
    if(fabs(A_(i, N)) > bnormi) bnormi = fabs(A_(i, N));
    xnorm1 += fabs(x[i]);
    if(fabs(x[i]) > xnormi) xnormi = fabs(x[i]);
  }
  const double eps = ldexp(1.0, -53);
  out[0] = N > 0 ? rnorm / (eps * (anormi * xnormi + bnormi) * (double)N) : 0.0;
  out[1] = rnorm;
  out[2] = anorm1;
  out[3] = anormi;
  out[4] = xnorm1;
  out[5] = xnormi;
  out[6] = bnormi;
  out[7] = eps;
  free(r);
  free(rs);
}

/* Whole HPL test at P = Q = 1: generate, solve, regenerate, check.  Used by
 * the CPU baseline.  res must hold 8 doubles (see hplo_residual). */
int hplo_hpl_test(int N, int nb, int nbmin, int ndiv, int pfact, int rfact,
                  uint64_t seed, double* A, int64_t ld, double* x, int* ipiv,
                  double* res) {
  hplo_matgen(N, N + 1, seed, A, ld);
  int info = hplo_pdgesv(N, nb, nbmin, ndiv, pfact, rfact, A, ld, x, ipiv);
  hplo_matgen(N, N + 1, seed, A, ld);
  hplo_residual(N, A, ld, x, res, NULL);
  return info;
}
