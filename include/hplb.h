/*
 * hplb.h -- C ABI of the B200-native HPL solve path: the single-process
 * (P = Q = 1) solve, and the per-process building blocks of the process-grid
 * drivers (rochpl_b200/grid.py for 1 x Q, rochpl_b200/grid2d.py for P x Q).
 *
 * Drop-in boundary for rocHPL's solve path.  Each entry point names the
 * reference interface it replaces (paths are within the rocHPL tree):
 *
 *   hplb_matgen   <- HPL_pdrandmat / hpl_randmat   src/matgen/HPL_pdrandmat_device.cpp:84-201
 *   hplb_matgen_block <- the local block of HPL_pdrandmat on a P x Q grid (same lines)
 *   hplb_pdgesv   <- HPL_pdgesv                     include/hpl_pgesv.hpp:162,
 *                                                   src/pgesv/HPL_pdgesv.cpp:19-368
 *   hplb_residual <- the check in HPL_pdtest        src/HPL_pdtest.cpp:307-438
 *                    with HPL_pdlange               src/pauxil/HPL_pdlange_device.cpp:118-302
 *   hplb_default_ld <- the ld padding of HPL_pdmatgen src/matgen/HPL_pdmatgen.cpp:109-110
 *
 * Conventions
 *  - Matrices are column-major FP64 in device memory owned by the caller;
 *    [A|b] is N x (N+1) with b in column N, exactly as HPL_pdmatgen lays it out.
 *  - The context owns its streams, events and workspaces; one context per host
 *    thread.  Calls return once the device work they queued has finished.
 *  - Every call returns an hplb_status; nothing calls exit().  Device-side waits
 *    are bounded and surface as HPLB_ERR_TIMEOUT.
 */
#ifndef HPLB_H
#define HPLB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum hplb_status {
  HPLB_OK              = 0,
  HPLB_ERR_ARG         = 1, /* invalid argument (message in hplb_last_error) */
  HPLB_ERR_OOM         = 2, /* workspace allocation failed */
  HPLB_ERR_SINGULAR    = 3, /* exact zero pivot; the solve still completed */
  HPLB_ERR_TIMEOUT     = 4, /* a bounded device-side wait expired */
  HPLB_ERR_CUDA        = 5, /* CUDA runtime error (message in hplb_last_error) */
  HPLB_ERR_UNSUPPORTED = 6  /* parameter combination rocHPL also rejects */
} hplb_status;

typedef struct hplb_ctx hplb_ctx;

/* Algorithm parameters: the HPL.dat fields of HPL_T_palg that reach the solve
 * (include/hpl_pgesv.hpp:63-81).  pfact / rfact use the HPL.dat encoding:
 * 0 = left-looking, 1 = Crout, 2 = right-looking. */
typedef struct hplb_algo {
  int nb;       /* panel width NB (>= 1) */
  int nbmin;    /* recursion stopping width NBMIN (>= 1) */
  int ndiv;     /* panels per recursion level NDIV (>= 2) */
  int pfact;    /* leaf factorisation PFACT */
  int rfact;    /* recursive factorisation RFACT */
  int depth;    /* look-ahead depth; rocHPL accepts 1 only (src/HPL_pdinfo.cpp:931-935) */
  int l1notran; /* L1 form; 0 (transposed) or 1; no effect on results */
} hplb_algo;

/* Residual check results (src/HPL_pdtest.cpp:330-438). */
typedef struct hplb_resid {
  double resid;     /* ||b-Ax||oo / (eps (||A||oo ||x||oo + ||b||oo) N) */
  double rnorm_inf; /* ||b-Ax||oo */
  double anorm_1;   /* ||A||1 */
  double anorm_inf; /* ||A||oo */
  double xnorm_1;   /* ||x||1 */
  double xnorm_inf; /* ||x||oo */
  double bnorm_inf; /* ||b||oo */
  double eps;       /* 2^-53, HPL_dlamch's eps (src/auxil/HPL_dlamch.cpp:104-111) */
} hplb_resid;

/* Per-call timings of the last hplb_pdgesv, from CUDA events (ms). */
typedef struct hplb_timing {
  double total_ms;  /* whole solve, LU + back-solve */
  double lu_ms;     /* factorisation incl. trailing updates */
  double trsv_ms;   /* back-solve */
  double gemm_ms;   /* sum of trailing-update DGEMM kernel time */
  double gemm_flops; /* algorithmic DGEMM flops of those kernels */
  double panel_ms;  /* sum of panel factorisation time (concurrent with updates) */
  int    gemm_launches;
  int    kernel_launches; /* every kernel this library queued during the call */
} hplb_timing;

/* Create a context on CUDA device `device`.  Returns NULL on failure, with the
 * reason in *status when status is not NULL.  A process may hold several
 * contexts (one per host thread, say), all on one device: some kernels' shared
 * memory limits are raised once per process, so drive each GPU from its own
 * process, as rocHPL's one MPI rank per GPU does.  A context on a second
 * device is refused with HPLB_ERR_UNSUPPORTED (and a message on stderr). */
hplb_ctx* hplb_create(int device, hplb_status* status);
void      hplb_destroy(hplb_ctx* ctx);

/* Inputs of every later call on ctx are read only after the work queued on
 * `stream` (a cudaStream_t) before that call has finished; NULL (the default)
 * means the legacy default stream.  Calls still return with their own work
 * complete.  (The reference is synchronous per call, with no stream
 * parameter.) */
hplb_status hplb_set_stream(hplb_ctx* ctx, void* stream);

/* Per-context options (no counterpart in the reference).
 *   HPLB_OPT_LEAF: where the panel leaf keeps the rows of its NBMIN-wide slice
 *   while it factors it -- HPLB_LEAF_AUTO (default: in the registers of one
 *   thread-block cluster of up to 16 SMs when the slice fits there, else in
 *   registers across the GPU, else shared memory, else global memory),
 *   HPLB_LEAF_REGISTERS (registers across the GPU first, never the cluster),
 *   HPLB_LEAF_SHARED (shared memory first) or HPLB_LEAF_GLOBAL.  All perform
 *   the same operations in the same order and give identical results; the
 *   choice only moves time.  The rocHPL leaf keeps its slice in global memory
 *   (src/pfact/HPL_pdpanrlT_device.cpp:23-320). */
#define HPLB_OPT_LEAF 1
#define HPLB_LEAF_AUTO 0
#define HPLB_LEAF_SHARED 1
#define HPLB_LEAF_GLOBAL 2
#define HPLB_LEAF_REGISTERS 3
/*   HPLB_OPT_PANEL_SMS: SMs that the trailing-update DGEMM leaves to the panel
 *   factorisation while the next panel is being factored beside it: 0 (the
 *   DGEMM may take every SM; the high-priority panel kernels take SMs as its
 *   CTAs retire), or k > 0 in every step (the DGEMM's grid is capped at
 *   SMs - k CTAs, each walking a longer run of tiles).  HPLB_PANEL_SMS_AUTO
 *   (-1, the default) keeps 32 SMs only in the steps whose update is at most 4
 *   waves of tiles, where the panel is the longer chain; a cap in every step
 *   slows the solve, because the panel's own GEMMs and triangular solves then
 *   run on the few SMs left to them.  Results do not depend on it. */
#define HPLB_OPT_PANEL_SMS 2
#define HPLB_PANEL_SMS_AUTO (-1)
hplb_status hplb_set_option(hplb_ctx* ctx, int option, int value);

const char* hplb_status_string(hplb_status s);
/* Message of the last failing call on this context (never NULL). */
const char* hplb_last_error(const hplb_ctx* ctx);

/* rocHPL's padded leading dimension for an n-row local matrix:
 * ((max(1,n)+95)/128)*128 + 32 (src/matgen/HPL_pdmatgen.cpp:109-110). */
int64_t hplb_default_ld(int n);

/* HPL_pdrandmat at P = Q = 1: fill the m x n column-major device matrix dA
 * (leading dimension ld >= m) from the 64-bit LCG with seed `seed`; entry
 * (i, j) is the value of state X(1 + i + j*m).  Bit-exact with rocHPL.
 * nb is accepted for interface parity and does not change the values. */
hplb_status hplb_matgen(hplb_ctx* ctx, int m, int n, int nb, uint64_t seed,
                        double* dA, int64_t ld);

/* A block of the same LCG matrix: rows [i0, i0 + m) and columns [j0, j0 + n)
 * of the global mg x ng matrix of `seed`, into the m x n column-major dA
 * (leading dimension ld >= m).  Local entry (i, j) is the value of state
 * X(1 + (i0 + i) + (j0 + j) mg), bit-identical to the same entry of
 * hplb_matgen(mg, ng).  This is the local part a process of a P x Q grid
 * generates in HPL_pdrandmat (src/matgen/HPL_pdrandmat_device.cpp:136-175,
 * one block-cyclic block per call here). */
hplb_status hplb_matgen_block(hplb_ctx* ctx, int64_t mg, int64_t ng, int64_t i0, int64_t j0,
                              int m, int n, uint64_t seed, double* dA, int64_t ld);

/* HPL_pdgesv at P = Q = 1: LU-factor the n x (n+1) [A|b] in dA (ld >= n) with
 * row partial pivoting and look-ahead depth 1, then back-solve U x = y into
 * dX (n doubles, device).  On exit dA holds U in its upper triangle, the panel
 * multipliers below it (unpivoted across panels, as in rocHPL) and y in
 * column n.  ipiv_out (device, n ints, may be NULL) receives, for each column
 * j, the global row swapped into row j.  *info (host, may be NULL) receives
 * the first zero-pivot column (1-based) or 0; a zero pivot also returns
 * HPLB_ERR_SINGULAR after the solve completes. */
hplb_status hplb_pdgesv(hplb_ctx* ctx, const hplb_algo* algo, int n, double* dA,
                        int64_t ld, double* dX, int* ipiv_out, int* info);

/* hplb_pdgesv for nrhs >= 1 right-hand sides at once: B occupies columns
 * n .. n + nrhs - 1 of the same column-major array (A | B, leading dimension
 * ld >= n, n + nrhs columns) and takes every interchange and trailing update
 * as HPL_pdgesv's column n does, so no separate forward solve is needed; then
 * X = U^-1 B (device, n x nrhs, leading dimension ldx >= n) by a persistent
 * back-solve of 32 right-hand sides per launch.  dA, ipiv_out and info as in
 * hplb_pdgesv; nrhs = 1 gives the same result as hplb_pdgesv.  The reference
 * carries exactly one right-hand side (include/hpl_pgesv.hpp:162). */
hplb_status hplb_gesv(hplb_ctx* ctx, const hplb_algo* algo, int n, int nrhs, double* dA,
                      int64_t ld, double* dX, int64_t ldx, int* ipiv_out, int* info);

/* The factorisation of hplb_pdgesv on the n x n A alone (no right-hand side
 * column, no back-solve): the same panels, pivots and layout, for use with
 * hplb_getrs.  No counterpart in the reference (HPL_pdgesv always carries b). */
hplb_status hplb_getrf(hplb_ctx* ctx, const hplb_algo* algo, int n, double* dA, int64_t ld,
                       int* ipiv_out, int* info);

/* Solve op(A) X = B with the factors hplb_pdgesv / hplb_getrf left in dLU
 * (leading dimension ld) and their pivots d_ipiv (device, n ints, each
 * ipiv[i] in [i, n)); nb must be the NB of that factorisation.  trans = 0:
 * A X = B; trans = 1: A^T X = B (this form also takes an n x n workspace).  B
 * (device, n x nrhs, leading dimension ldb) is overwritten by X.  The
 * solve-side building block of the differentiable solve; no counterpart in the
 * reference. */
hplb_status hplb_getrs(hplb_ctx* ctx, int trans, int n, int nb, int nrhs, const double* dLU,
                       int64_t ld, const int* d_ipiv, double* dB, int64_t ldb);

/* C = alpha A B^T (accumulate = 0) or C += alpha A B^T (accumulate != 0) in one
 * fused kernel: A m x k, B n x k, C m x n, all column-major FP64 on the device,
 * k <= 64.  The adjoint's Abar = -Bbar X^T. */
hplb_status hplb_rank_k(hplb_ctx* ctx, int m, int n, int k, double alpha, const double* dA,
                        int64_t lda, const double* dB, int64_t ldb, double* dC, int64_t ldc,
                        int accumulate);

/* ---------------------------------------------------------------------------
 * Batched form (no counterpart in the reference, which solves one system per
 * run).  Many independent systems of uneven size, system i being n[i] x n[i]
 * with nrhs[i] right-hand sides, solved in one persistent, graph-captured
 * launch: one CTA per system at a time, largest first, right-looking blocked
 * LU with partial pivoting (full-row interchanges, as LAPACK's getrf, so P A =
 * L U), the panel width from the system's size class.
 *
 * Layout (device pools, all column-major, packed in system order): A_i at
 * a_off[i] with leading dimension n[i]; B_i (n[i] x nrhs[i]) at b_off[i] with
 * leading dimension n[i]; pivots at p_off[i] (n[i] ints, 0-based row swapped
 * into each row, as LAPACK's ipiv minus one).
 * ------------------------------------------------------------------------ */
#define HPLB_BATCH_CLASSES 6   /* size classes: n < 48, < 96, < 192, < 384, < 768, >= 768 */
#define HPLB_BATCH_MAX_N 2048
/* Class entry selecting the recursive factorisation (columns halved down to
 * 16-wide leaves, GEMM updates with k up to n/2) for systems with n <=
 * HPLB_BATCH_RECURSIVE_MAX_N; larger systems of the class use 16-wide panels. */
#define HPLB_BATCH_RECURSIVE 64
#define HPLB_BATCH_RECURSIVE_MAX_N 1024

typedef struct hplb_batch hplb_batch;

/* Plan a batch (host arrays n, nrhs of length count).  nb_by_class: per size
 * class, a right-looking panel width (8, 16 or 32) or HPLB_BATCH_RECURSIVE,
 * e.g. from hplb_batch_tune; NULL for the built-in table.  Widths are lowered
 * where a panel would not fit in shared memory. */
hplb_status hplb_batch_create(hplb_ctx* ctx, int count, const int* n, const int* nrhs,
                              const int* nb_by_class, hplb_batch** out);
void        hplb_batch_destroy(hplb_batch* b);
/* Pool sizes (elements) and, when the arrays are not NULL, every system's
 * offsets and panel width (host arrays of length count). */
hplb_status hplb_batch_layout(const hplb_batch* b, int64_t* a_elems, int64_t* b_elems,
                              int64_t* p_elems, int64_t* a_off, int64_t* b_off, int64_t* p_off,
                              int* nb);
/* [A_i | B_i] = the HPL LCG matrix of seeds[i] (host array), n[i] x (n[i] +
 * nrhs[i]) with n[i] rows: the first n[i] columns go to A_i, the rest to B_i. */
hplb_status hplb_batch_matgen(hplb_batch* b, const uint64_t* seeds, double* dA, double* dB);
/* Factor every A_i in place (L and U), overwrite B_i with X_i = A_i^-1 B_i,
 * pivots to dipiv, first zero pivot (1-based, 0 if none) to dinfo[i]. */
hplb_status hplb_batch_gesv(hplb_batch* b, double* dA, double* dB, int* dipiv, int* dinfo);
/* With the factors and pivots of hplb_batch_gesv: B_i <- A_i^-1 B_i (trans = 0)
 * or A_i^-T B_i (trans = 1). */
hplb_status hplb_batch_getrs(hplb_batch* b, int trans, const double* dLU, const int* dipiv,
                             double* dB);
/* C_i = alpha X_i Y_i^T (X_i, Y_i in the B layout, C_i in the A layout). */
hplb_status hplb_batch_rank_k(hplb_batch* b, double alpha, const double* dX, const double* dY,
                              double* dC);
/* dresid[i] (device) = the HPL scaled residual of X_i against the regenerated
 * LCG system of seeds[i], the largest over its right-hand sides. */
hplb_status hplb_batch_residual(hplb_batch* b, const uint64_t* seeds, const double* dX,
                                double* dresid);
/* Device time of the last batch call (ms). */
hplb_status hplb_batch_last_ms(const hplb_batch* b, double* ms);
/* The autotuner: times panel widths 8 / 16 / 32 and the recursive
 * factorisation on a batch of each size class (2 x SM-count systems, nrhs
 * right-hand sides) and writes the fastest to nb_by_class; ms_table (6 x 4,
 * may be NULL) receives every timing, -1 where a candidate does not fit. */
hplb_status hplb_batch_tune(hplb_ctx* ctx, int nrhs, int* nb_by_class, double* ms_table);

/* ---------------------------------------------------------------------------
 * Building blocks of HPL_pdgesv on a 1 x Q process grid (P = 1, Q > 1; one
 * process per GPU).  [A|b] is distributed in NB-wide column blocks, block c
 * on process c mod Q (the block-cyclic layout of HPL_pdmatgen,
 * src/matgen/HPL_pdmatgen.cpp:85-383, at P = 1); each process holds all n rows
 * of its blocks in a local column-major array (local column lc of a block =
 * its position among the process's blocks times NB).  Global row indices
 * throughout.  The per-panel driver (factor on the owner, broadcast, update
 * everywhere, then the distributed back-solve) is rochpl_b200/grid.py.
 * ------------------------------------------------------------------------ */

/* HPL_pdfact on the process that owns the panel (src/pfact/HPL_pdfact.cpp:20-110;
 * at P = 1 the pivot search needs no other process): factor global rows
 * [j, n) of local columns [lc, lc + jb) in place with the recursion and leaf
 * of algo; d_ipiv (device, jb ints) receives the global rows swapped into rows
 * j .. j + jb - 1.  A zero pivot sets *info to its global column (1-based) and
 * returns HPLB_ERR_SINGULAR. */
hplb_status hplb_panel_factor(hplb_ctx* ctx, const hplb_algo* algo, int n, int j, int jb,
                              double* dA, int64_t ld, int lc, int* d_ipiv, int* info);

/* HPL_pdupdateTT on one process's columns (src/pgesv/HPL_pdupdateTT.cpp:19-168,
 * with the P = 1 row interchanges of src/pgesv/HPL_pdlaswp.cpp:300-389): the
 * factored panel of global rows [j, n) in dL (leading dimension ldl >= n - j;
 * row 0 of dL is global row j: unit lower L11 in its top jb rows, L21 below)
 * with its pivots d_ipiv (device, jb global rows, each checked to lie in
 * [j + k, n)), applied to local columns [c0, c0 + ncols) of dA: the
 * interchanges, U12 = L11^-1 A12 in the top rows, A22 -= L21 U12. */
hplb_status hplb_panel_update(hplb_ctx* ctx, int n, int j, int jb, const double* dL,
                              int64_t ldl, const int* d_ipiv, double* dA, int64_t ld, int c0,
                              int ncols);

/* One block step of the distributed back-solve (HPL_pdtrsv,
 * src/pgesv/HPL_pdtrsv_device.cpp:29-346) on the process owning the column
 * block [j, j + jb) at local column lc: x[j : j+jb] = U_jj^-1 (y[j : j+jb] -
 * s), then z[0 : j] += U[0 : j, block] x[j : j+jb].  dy, dx, dz: n doubles
 * (device, global indexing); ds: jb doubles, the sum over all processes of
 * their z[j : j+jb]. */
hplb_status hplb_trsv_block(hplb_ctx* ctx, int n, int j, int jb, const double* dA, int64_t ld,
                            int lc, const double* dy, const double* ds, double* dx, double* dz);

/* Building blocks of the solve on a P x Q process grid (rows block-cyclic as
 * well; the driver is rochpl_b200/grid2d.py), where a panel column's rows are
 * spread over the processes of a process column.
 *
 * hplb_col_argmax: the local part of one column's pivot search
 * (HPL_pdmxswp, src/pfact/HPL_pdmxswp.cpp:19-126, combines these across the
 * process column): the value of largest magnitude in rows [r0, r1) of column
 * col of dA, and its row (the lowest among equal magnitudes), to host
 * *v_out / *row_out; -1 for an empty range. */
hplb_status hplb_col_argmax(hplb_ctx* ctx, const double* dA, int64_t ld, int r0, int r1, int col,
                            double* v_out, int* row_out);

/* The leaf's column step on local rows [r0, r1) (the scale and rank-1 update
 * of src/pfact/HPL_pdpanrlT_device.cpp:225-240): l = A[r, c0+k] / piv into
 * column c0 + k, then A[r, c0+c] -= l du[c] for k < c < kend (du: the pivot
 * row's panel values, device). */
hplb_status hplb_col_rank1(hplb_ctx* ctx, double* dA, int64_t ld, int r0, int r1, int c0, int k,
                           int kend, double piv, const double* du);

/* Largest n hplb_trsm_lower_unit accepts: a panel's width (NB) at most; each
 * CTA keeps a slice of X's columns, n rows deep, in shared memory. */
#define HPLB_TRSM_LOWER_MAX_N 2048

/* X <- L^-1 X for the unit-lower n x n L (leading dimension ldl) and X
 * (n x nrhs, leading dimension ldx), device (the rocblas_dtrsm of
 * src/pgesv/HPL_pdupdateTT.cpp:95-106 and of the recursive panel,
 * src/pfact/HPL_pdrpanrlT.cpp:124-140); n <= HPLB_TRSM_LOWER_MAX_N. */
hplb_status hplb_trsm_lower_unit(hplb_ctx* ctx, int n, int nrhs, const double* dL, int64_t ldl,
                                 double* dX, int64_t ldx);

/* X = U^-1 Y for the upper triangle of the n x n U (leading dimension ldu)
 * and Y, X (n x nrhs), device; X may be Y.  The persistent multi-RHS
 * back-solve of hplb_gesv (the diagonal-block solve of HPL_pdtrsv,
 * src/pgesv/HPL_pdtrsv_device.cpp:170-307, for any number of columns). */
hplb_status hplb_trsm_upper(hplb_ctx* ctx, int n, int nrhs, const double* dU, int64_t ldu,
                            const double* dY, int64_t ldy, double* dX, int64_t ldx);

/* The HPL residual check: dA must hold the regenerated [A|b] (hplb_matgen with
 * the seed of the solve), dX the solution.  Results go to *out (host). */
hplb_status hplb_residual(hplb_ctx* ctx, int n, const double* dA, int64_t ld,
                          const double* dX, hplb_resid* out);

/* Same check without a stored matrix: [A|b] is regenerated from the LCG inside
 * the kernel (bit-identical values), so no N x N buffer is read or written. */
hplb_status hplb_residual_lcg(hplb_ctx* ctx, int n, uint64_t seed,
                              const double* dX, hplb_resid* out);

/* Timings of the last hplb_pdgesv on this context. */
hplb_status hplb_last_timing(const hplb_ctx* ctx, hplb_timing* out);

/* Per-step times of the last hplb_pdgesv / hplb_getrf on this context, for
 * the progress report of src/pgesv/HPL_pdgesv.cpp:136-341 (HPL_PROGRESS_REPORT):
 * step i factors columns [col[i], col[i] + NB); ms[i] runs from the end of
 * step i-1 (the start of the call for i = 0) to the end of step i's trailing
 * update, CUDA events on the update stream.  *count = the number of steps;
 * min(cap, *count) entries are written. */
hplb_status hplb_last_steps(const hplb_ctx* ctx, int cap, int* count, int* col, double* ms);

/* Building blocks, exposed for tests and tools (device pointers, synchronous).
 *   hplb_dgemm_sub : C(m x n) -= A(m x k) B(k x n), column-major; the trailing
 *                    update kernel of hplb_pdgesv (rocblas_dgemm call in
 *                    src/pgesv/HPL_pdupdateTT.cpp:131-163).
 *   hplb_laswp_trsm: apply the row interchanges ipiv (jb global rows, first row
 *                    ia) to columns [c0, c0+n) of dA and replace the top jb rows
 *                    by L11^-1 times them, L11 the unit lower triangle at
 *                    (ia, lc) (HPL_dlaswp00N + rocblas_dtrsm,
 *                    src/pgesv/HPL_pdupdateTT.cpp:95-106). */
hplb_status hplb_dgemm_sub(hplb_ctx* ctx, int m, int n, int k, const double* dA,
                           int64_t lda, const double* dB, int64_t ldb, double* dC,
                           int64_t ldc);
hplb_status hplb_laswp_trsm(hplb_ctx* ctx, double* dA, int64_t ld, int ia, int jb,
                            int lc, const int* ipiv_host, int c0, int n);

/* ------------------------------------------------------------------------
 * Mixed-precision form (no counterpart in the reference, which is FP64 only).
 * LU in FP32 storage with the panel in FP32 and the trailing update on the
 * tensor cores in BF16 or FP16 (per-tile power-of-two scaling, FP32
 * accumulation), then flexible GMRES iterative refinement in FP64,
 * preconditioned by the low-precision factors, until the HPL scaled residual
 * is below target_resid.  FP64 is used only for r = b - A x against the FP64
 * A, the solution update and the norms.
 * ------------------------------------------------------------------------ */
typedef struct hplb_mixed_opts {
  int    precision;    /* trailing update: 0 = BF16 (default), 1 = FP16, 2 = BF16 x3 and
                          3 = FP16 x3 (each operand split into high and low 16-bit parts,
                          three products accumulated in FP32: FP32-accurate factors) */
  int    restart;      /* GMRES restart length (<= 0: 20) */
  int    max_outer;    /* refinement steps (<= 0: 20) */
  double target_resid; /* stop below this HPL scaled residual (<= 0: 16.0) */
  double gmres_tol;    /* relative residual reduction per GMRES cycle (<= 0: 1e-6) */
} hplb_mixed_opts;

typedef struct hplb_mixed_report {
  double resid;        /* final HPL scaled residual */
  double resid_lu;     /* scaled residual of x = M^-1 b with the low-precision LU alone */
  int    outer_iters;  /* refinement steps taken */
  int    gmres_iters;  /* GMRES iterations in total (one preconditioned A-product each) */
  int    converged;    /* resid < target_resid */
  int    info;         /* first zero pivot of the FP32 panel (1-based), 0 if none */
  double lu_ms;        /* low-precision factorisation */
  double ir_ms;        /* refinement (initial solve included) */
  double total_ms;     /* time to solution (device events, first to last) */
  double gemm_ms;      /* tensor-core trailing-update kernel time within lu_ms */
  double gemm_flops;   /* tensor-core flops of those kernels (x3 counted for the split forms) */
  double panel_ms;     /* FP32 panel factorisation time (concurrent with the updates) */
} hplb_mixed_report;

/* Solve the n x n system of [A|b].  dA: the FP64 [A|b] (n x (n+1), leading
 * dimension ld, not modified), or NULL to use the HPL LCG matrix of `seed`
 * regenerated on the fly (bit-identical to hplb_matgen; no n x n FP64 buffer
 * is needed, which is what lets n = 131072 fit beside the FP32 factors).
 * dX receives x (n doubles, device); ipiv_out (device, may be NULL) the pivots
 * of the low-precision LU. */
hplb_status hplb_pdgesv_mixed(hplb_ctx* ctx, const hplb_algo* algo, const hplb_mixed_opts* opts,
                              int n, const double* dA, int64_t ld, uint64_t seed, double* dX,
                              int* ipiv_out, hplb_mixed_report* report);

/* Mixed-precision trailing update (tensor cores, tcgen05): C -= sA[i] sB[j]
 * A16 B16^T on 128 x 256 tiles, FP32 accumulation.  C is m x n FP32
 * column-major; A16 (m x k) and B16 (n x k) are row-major 16-bit (bf16 != 0:
 * BF16, else FP16) with leading dimensions that are multiples of 8; sA holds
 * ceil(m/128) and sB ceil(n/256) FP32 tile scale factors.  The building block of
 * hplb_pdgesv_mixed; no counterpart in the reference (rocHPL is FP64 only). */
hplb_status hplb_gemm_lp_sub(hplb_ctx* ctx, int bf16, int m, int n, int k, const void* dA16,
                             int64_t lda, const void* dB16, int64_t ldb, const float* dsA,
                             const float* dsB, float* dC, int64_t ldc);

/* Measurement and self-test utilities (no counterpart in the reference).
 *   hplb_fp64_peak          : FP64 tensor-core (DMMA m16n8k8) and FP64 FMA issue
 *                             rates of this GPU in TFLOP/s, the roofline
 *                             denominators for the trailing-update DGEMM.
 *   hplb_selftest_wait_timeout : runs one bounded device wait on a flag nothing
 *                             sets, with a budget of budget_ns nanoseconds; returns
 *                             HPLB_ERR_TIMEOUT and leaves the context usable. */
hplb_status hplb_fp64_peak(hplb_ctx* ctx, int iters, double* dmma_tflops, double* dfma_tflops);
hplb_status hplb_selftest_wait_timeout(hplb_ctx* ctx, uint64_t budget_ns);

/* Largest n hplb_residual_lcg_noalloc accepts (its static scratch is sized for it). */
#define HPLB_NOALLOC_MAX_N 16384

/* Allocation-free variant of hplb_residual_lcg.  No counterpart in the
 * reference: it exists for callers that must not allocate device memory, such
 * as a program whose device memory is all handed to its own pool allocator, or
 * a check run between solves where cudaMalloc's implicit synchronisation is not
 * allowed.  It needs no context and calls no allocating routine; its scratch is
 * a fixed array in the library's device image (about 2.1 MB, held by every GPU
 * that loads the library until exit), so n is limited to HPLB_NOALLOC_MAX_N
 * (larger n returns HPLB_ERR_ARG with a message on stderr).
 *   dX     : the solution, n doubles in device memory of the current device
 *   stream : a cudaStream_t (NULL = the default stream); the call waits for it
 *   out    : host results, as hplb_residual_lcg
 * The first call on each device looks up the scratch address on that device
 * (make it with that device current and before any stream capture).  That
 * address is kept for the life of the process and does not survive a
 * cudaDeviceReset.  Under CUDA's default lazy module loading the library's
 * device image, array included, is loaded by the first kernel launch or
 * symbol lookup on a device: make the first call on each device before the
 * device memory is handed to the caller's own pool, or run with
 * CUDA_MODULE_LOADING=EAGER so the image loads when the context is made.  All calls
 * on a device share the one scratch array: calls that overlap on the GPU (two
 * host threads, or two streams) race and must be serialised by the caller. */
hplb_status hplb_residual_lcg_noalloc(int n, uint64_t seed, const double* dX, void* stream,
                                      hplb_resid* out);

#ifdef __cplusplus
}
#endif

#endif /* HPLB_H */
