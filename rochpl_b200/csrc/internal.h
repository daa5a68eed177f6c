// Internal launcher interface shared by the .cu files of libhplb200.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace hplb {

constexpr int kMaxLeaf = 128;  // widest leaf (NBMIN) the leaf kernel holds

cudaError_t launch_matgen(int m, int n, uint64_t seed, double* A, int64_t ld,
                          cudaStream_t stream);
// Rows [i0, i0 + m) x columns [j0, j0 + n) of the global mg-row LCG matrix.
cudaError_t launch_matgen_block(int64_t mg, int64_t i0, int64_t j0, int m, int n, uint64_t seed,
                                double* A, int64_t ld, cudaStream_t stream);

// C -= A B.  Uses the TMA-fed warp-specialised kernel when the operands
// qualify (dgemm_tma_eligible), the cp.async kernel otherwise.  status may be
// null (then only the cp.async kernel, which has no waits, is used).
// max_ctas > 0 caps the TMA kernel's grid (each CTA then walks a longer run of
// tiles), leaving the other SMs free for concurrent work.
cudaError_t launch_dgemm_sub(int m, int n, int k, const double* A, int64_t lda,
                             const double* B, int64_t ldb, double* C, int64_t ldc,
                             int* status, cudaStream_t stream, int max_ctas = 0);
// C = A B (store form of the same kernels; C is not read).
cudaError_t launch_dgemm_set(int m, int n, int k, const double* A, int64_t lda,
                             const double* B, int64_t ldb, double* C, int64_t ldc,
                             int* status, cudaStream_t stream);
bool        dgemm_tma_eligible(int m, int n, int k, const double* A, int64_t lda,
                               const double* B, int64_t ldb);
cudaError_t launch_dgemm_tma(int m, int n, int k, const double* A, int64_t lda,
                             const double* B, int64_t ldb, double* C, int64_t ldc,
                             int* status, bool accumulate, cudaStream_t stream,
                             int max_ctas = 0);
cudaError_t launch_dgemm_cpasync(int m, int n, int k, const double* A, int64_t lda,
                                 const double* B, int64_t ldb, double* C, int64_t ldc,
                                 bool accumulate, cudaStream_t stream);

int         leaf_grid_size(int num_sms, int rows);
// The panel kernels exist for double (the FP64 solve) and float (the FP32
// panel of the mixed-precision solve).
// leaf_kind: where the leaf's rows live, HPLB_LEAF_* of include/hplb.h
// (auto = registers, then shared memory, then global memory, the first that
// holds the leaf; a forced kind falls through the same way when it does not).
// pc, pw: the panel the leaf belongs to.  *swapped is set when the leaf also
// applied its interchanges to the panel's other columns (the cluster leaf
// does; otherwise the caller runs launch_panel_swap).
template <typename T>
cudaError_t launch_leaf(T* A, int64_t ld, int r0, int end, int c0, int w, int pc, int pw,
                        int* ipiv, double* cand, double* cur, int* bar, int* status, int grid,
                        int leaf_kind, cudaStream_t stream, bool* swapped);
template <typename T>
cudaError_t launch_panel_swap(T* A, int64_t ld, const int* ipiv, int r0, int c0, int w, int pc,
                              int pw, cudaStream_t stream);
cudaError_t launch_perm(const int* ipiv, int ia, int jb, int* permU, cudaStream_t stream);
template <typename T>
cudaError_t launch_diag_inv(const T* A, int64_t ld, int r0, int c0, int n, T* inv,
                            cudaStream_t stream);
int         trsm_wcol(int jb);
size_t      trsm_smem_bytes(int jb, bool own_dinv);
// Largest jb for which launch_laswp_trsm may be given dinv = null (the kernel
// then inverts the diagonal blocks itself).
constexpr int kFusedTri = 256;
template <typename T>
cudaError_t launch_laswp_trsm(T* A, int64_t ld, int ia, int jb, int lc, const int* permU,
                              const T* dinv, int c0, int n, cudaStream_t stream);
// U12 = L11^-1 A12 of one node of the recursive panel (L11 the unit-lower
// jb x jb block at (ia, lc), A12 rows [ia, ia+jb) of columns [c0, c0+n)): one
// launch for jb <= kFusedTri, else diag_inv into dinv_scratch and the TRSM.
// Adds the kernels it launched to *launches.
template <typename T>
cudaError_t launch_trsm_node(T* A, int64_t ld, int ia, int jb, int lc, T* dinv_scratch, int c0,
                             int n, cudaStream_t stream, int* launches);
// Linv (jb x jb, leading dimension ldinv) = L^-1 for the unit-lower L at L
// (leading dimension ldl), by the blocked substitution applied to the identity.
template <typename T>
cudaError_t launch_unit_lower_inverse(const T* L, int64_t ldl, int jb, const T* dinv, T* Linv,
                                      int64_t ldinv, cudaStream_t stream);
// X (jb x n) <- L^-1 X for the unit-lower L at L (leading dimension ldl) with
// its 32 x 32 diagonal inverses dinv (launch_diag_inv), FP64.
cudaError_t launch_trsm_unit_lower(double* X, int64_t ldx, int jb, const double* L, int64_t ldl,
                                   const double* dinv, int n, cudaStream_t stream);
// Panel interchanges on columns [c0, c0+n): new top rows gathered into W
// (jb x n, leading dimension ldw), displaced rows written in place.
template <typename T>
cudaError_t launch_laswp_gather(T* A, int64_t ld, int ia, int jb, const int* permU, T* W,
                                int64_t ldw, int c0, int n, cudaStream_t stream);

// Back-solve U x = y, y = column n of A, x written to X.
// The back-solve's flags: one per 64-row block plus the ticket counter.
size_t      trsv_flag_ints(int n);
cudaError_t launch_trsv(const double* A, int64_t ld, int n, double* X, int* flags, int* status,
                        cudaStream_t stream, int* launches);
// The same back-solve with the right-hand side y in its own vector (n doubles).
cudaError_t launch_trsv_y(const double* A, int64_t ld, int n, const double* Y, double* X,
                          int* flags, int* status, cudaStream_t stream, int* launches);
// z[0:m] += U[0:m, 0:k] x (U column-major, leading dimension ld); r = y - s.
// The P x Q grid's local column steps (grid2d.cu): the arg-max of |A[r, c]|
// over rows [r0, r1) into out[0] (value) and out[1] (row, -1 if none), and the
// leaf step on rows [r0, r1) of columns c0 + k .. c0 + kend - 1.
cudaError_t launch_col_argmax(const double* A, int64_t ld, int r0, int r1, int c, double* out,
                              cudaStream_t stream);
cudaError_t launch_col_rank1(double* A, int64_t ld, int r0, int r1, int c0, int k, int kend,
                             double piv, const double* u, int num_sms, cudaStream_t stream);
// X (n x nrhs, leading dimension ldx) = U^-1 Y for the upper triangle of A
// (n x n, leading dimension ld); Y (leading dimension ldy) may be X itself.
// Persistent, one launch per 32 right-hand sides; flags: trsv_flag_ints(n).
cudaError_t launch_trsm_upper(const double* A, int64_t ld, int n, int nrhs, const double* Y,
                              int64_t ldy, double* X, int64_t ldx, int* flags, int* status,
                              cudaStream_t stream, int* launches);
cudaError_t launch_gemv_acc(int m, int k, const double* U, int64_t ld, const double* x,
                            double* z, cudaStream_t stream);
cudaError_t launch_vsub(int n, const double* y, const double* s, double* r, cudaStream_t stream);

// Residual check.  ws must hold residual_ws_doubles(n) doubles.
size_t      residual_ws_doubles(int n);
cudaError_t launch_residual(int n, const double* A, int64_t ld, bool lcg, uint64_t seed,
                            const double* X, double* ws, double* out8, cudaStream_t stream);

// y = A x (FP64) and column extraction for [A|b], stored or regenerated from
// the LCG; ws as for launch_residual.
cudaError_t launch_gemv_hpl(int n, const double* A, int64_t ld, bool lcg, uint64_t seed,
                            const double* x, double* y, double* ws, cudaStream_t stream);
cudaError_t launch_column_hpl(int n, int col, const double* A, int64_t ld, bool lcg,
                              uint64_t seed, double* out, double* ws, cudaStream_t stream);

// Mixed-precision helpers (mixed.cu, sgemm.cu, matgen.cu).
cudaError_t launch_sgemm(int m, int n, int k, const float* A, int64_t lda, const float* B,
                         int64_t ldb, float* C, int64_t ldc, bool accumulate, cudaStream_t stream);
cudaError_t launch_f64_to_f32(int m, int n, const double* A, int64_t lda, float* W, int64_t ldw,
                              cudaStream_t st);
// split: three jb-wide segments per packed row (hi/lo parts, K = 3 jb).  The
// values are multiplied by sign (1 or -1) along with the tile scale.
cudaError_t launch_pack_l(bool bf16, bool split, int m, int jb, const float* L, int64_t ld,
                          void* out, int64_t ldo, float* sL, cudaStream_t st, float sign = 1.f);
cudaError_t launch_pack_u(bool bf16, bool split, int jb, int n, const float* U, int64_t ld,
                          void* out, int64_t ldo, float* sU, cudaStream_t st, float sign = 1.f);
// Uinv = U^-1 for the upper-triangular U (jb x jb at U, leading dimension
// ld); work: 2 jb^2 + jb elements, dinv_work: (jb/32 + 1) * 1024.
template <typename T>
cudaError_t launch_upper_inverse(int jb, const T* U, int64_t ld, T* Uinv, T* work, T* dinv_work,
                                 cudaStream_t st);
cudaError_t launch_perm_vec(double* z, int ia, int jb, const int* permU, cudaStream_t st);
// y -= M x / y = M x with FP32 M (rows x cols, column-major), FP64 x and y
// (not overlapping).
cudaError_t launch_gemv_sub(int rows, int cols, const float* M, int64_t ld, const double* x,
                            double* y, cudaStream_t st);
cudaError_t launch_gemv_set(int rows, int cols, const float* M, int64_t ld, const double* x,
                            double* y, cudaStream_t st);
int         vec_partials();
cudaError_t launch_dot(int n, const double* a, const double* b, double* part, double* out,
                       cudaStream_t st);
cudaError_t launch_amax(int n, const double* a, double* part, double* out, cudaStream_t st);
// Gram-Schmidt over k <= 64 columns of V (leading dimension ldv):
// out[i] = V_i . w (part: mdot_partials(k) doubles) and w -= V h (acc += h
// when acc is not null).
size_t      mdot_partials(int k);
cudaError_t launch_mdot(int n, int k, const double* V, int64_t ldv, const double* w,
                        double* part, double* out, cudaStream_t st);
cudaError_t launch_mgemv_sub(int n, int k, const double* V, int64_t ldv, const double* h,
                             double* w, double* acc, cudaStream_t st);
cudaError_t launch_axpy(int n, double a, const double* x, double* y, cudaStream_t st);
cudaError_t launch_scal_copy(int n, double a, const double* x, double* y, cudaStream_t st);
cudaError_t launch_sub(int n, const double* a, const double* b, double* c, cudaStream_t st);
cudaError_t launch_matgen_f32(int m, int n, uint64_t seed, float* W, int64_t ld,
                              cudaStream_t stream);

// Multi-RHS solve pieces (rhs.cu).
template <typename T>
cudaError_t launch_transpose(int m, int n, const T* src, int64_t lds, T* dst, int64_t ldd,
                             cudaStream_t st);
// The unit-lower jb x jb matrix (leading dimension jb) equivalent to the
// diagonal block T (leading dimension ldt) of the LU factors for a solve:
//   kind 0 (U):   J D^-1 U J,   with D = diag(U) written to d
//   kind 1 (L^T): J L^T J
//   kind 2 (U^T): (D^-1 U)^T,   with D to d
// (J reverses the order of rows and columns.)
cudaError_t launch_unit_lower_view(int kind, int jb, const double* T, int64_t ldt, double* out,
                                   double* d, cudaStream_t st);
// out (jb x n, leading dimension ldo) = in with rows reversed (flip) and / or
// divided by d (scale; d indexed by the source row).
cudaError_t launch_rows_xform(int jb, int n, const double* in, int64_t ldi, double* out,
                              int64_t ldo, const double* d, bool flip, bool scale,
                              cudaStream_t st);
// X (jb x ncols) <- L^-1 X, unit-lower L, for few right-hand sides: one CTA per
// column (dinv: the 32 x 32 diagonal inverses of L).
cudaError_t launch_trsm_small(int jb, int ncols, double* X, int64_t ldx, const double* L,
                              int64_t ldl, const double* dinv, cudaStream_t st);
// C (jb x nrhs) -= M (jb x K) Y (K x nrhs) for K >> jb, nrhs: split-k partial
// products into ws (splitk_ws_doubles) and a fixed-order reduction.
size_t      splitk_ws_doubles(int jb, int nrhs, int K);
cudaError_t launch_splitk_sub(int jb, int nrhs, int K, const double* M, int64_t ldm,
                              const double* Y, int64_t ldy, double* C, int64_t ldc, double* ws,
                              cudaStream_t st);
// C (m x nrhs) -= M (m x K) Y (K x nrhs) for tall M and few right-hand sides
// (one row per thread, the whole K per CTA).
cudaError_t launch_rows_sub(int m, int nrhs, int K, const double* M, int64_t ldm,
                            const double* Y, int64_t ldy, double* C, int64_t ldc,
                            cudaStream_t st);
// Inverse of a panel's row map on columns [0, n) of B: rows moved back to where
// the forward interchanges took them from.
cudaError_t launch_laswp_inverse(double* B, int64_t ldb, int ia, int jb, const int* permU, int n,
                                 cudaStream_t st);
// C = alpha A B^T (+ C when accumulate); A m x k, B n x k, k <= 64.
cudaError_t launch_rank_k(int m, int n, int k, double alpha, const double* A, int64_t lda,
                          const double* B, int64_t ldb, double* C, int64_t ldc, bool accumulate,
                          cudaStream_t st);
// status[ST_INFO] = first i (1-based) with ipiv[i] outside [i, n), else untouched.
cudaError_t launch_check_ipiv(int n, const int* ipiv, int* status, cudaStream_t st);
cudaError_t launch_check_ipiv_range(int count, int first, int nrows, const int* ipiv,
                                    int* status, cudaStream_t st);

// Batched solver kernels (batch.cu); the plan and C ABI are in batch_api.cu.
size_t      batch_static_smem();
size_t      batch_rec_stage_bytes();  // dynamic shared memory of the recursive mode
int         batch_threads();
int         batch_nb_max();
// Sets the kernels' dynamic shared-memory limits; *budget = what a plan may use.
cudaError_t batch_set_smem(size_t* budget);
// mode: 0 gesv, 1 getrs, 2 getrs transposed, 3 rank-k, 4 matgen, 5 residual.
cudaError_t launch_batch(int mode, const void* d_args, int grid, size_t dyn_bytes,
                         cudaStream_t st);
size_t      batch_args_bytes();
void        batch_fill_args(void* host_args, double* A, const double* LU, double* B, int* ipiv,
                            const int* ipivc, int* info, const void* sys, const int* order,
                            int count, int* counter, double alpha, const double* X,
                            const double* Y, double* C, const unsigned long long* seeds,
                            double* resid);
size_t      batch_sys_bytes();
void        batch_fill_sys(void* dst, int i, int n, int nrhs, int nb, long long a_off,
                           long long b_off, long long p_off);

// FP64 issue-rate probes (TFLOP/s) and the bounded-wait self test.
cudaError_t fp64_peak(int num_sms, int iters, double* dmma_tflops, double* dfma_tflops,
                      cudaStream_t stream);
cudaError_t launch_wait_selftest(const int* flag, int* status, unsigned long long budget_ns,
                                 cudaStream_t stream);

// Mixed-precision trailing update on tcgen05: C (fp32, column-major) -=
// sA[tile_m] sB[tile_n] A16 B16^T, A16 m x k and B16 n x k row-major 16-bit
// (BF16 when bf16, else FP16), tiles of gemm_lp_tile_m() x gemm_lp_tile_n().
int         gemm_lp_tile_m();
int         gemm_lp_tile_n();
cudaError_t launch_gemm_lp(bool bf16, int m, int n, int k, const void* A16, int64_t lda,
                           const void* B16, int64_t ldb, const float* sA, const float* sB,
                           float* C, int64_t ldc, int* status, cudaStream_t stream);

}  // namespace hplb
