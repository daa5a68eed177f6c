// hplb_getrs and hplb_rank_k: solves with the stored HPL factors for many
// right-hand sides, plain or transposed, and the fused rank-k product.  These
// serve the differentiable solve (the adjoint of X = A^-1 B is
// Bbar = A^-T Xbar, Abar = -Bbar X^T) and have no counterpart in the reference.
//
// The HPL factorisation (src/pgesv/HPL_pdgesv.cpp:168-362) leaves, per panel
// p at rows/columns [j, j + jb): the panel's interchanges P_p, applied to the
// rows below j only; the unit-lower L of the panel, in the row order the panel
// ended with (later panels' interchanges never reach it); and U.  So
//   A^-1 = U^-1 E_{np-1} P_{np-1} ... E_0 P_0,  E_p = [L11^-1 0; -L21 L11^-1 I]
// and
//   A^-T = P_0^T E_0^T ... P_{np-1}^T E_{np-1}^T U^-T.
// The off-diagonal block products are DMMA GEMMs of this library; the
// diagonal blocks are solved by the blocked substitution kernel (explicit
// inverses of 512 x 512 blocks would cost far more than a few right-hand
// sides); the transposed solve reads a transposed copy of the factors so that
// its GEMMs are plain NN.
#include <algorithm>

#include "ctx.h"

using namespace hplb;

namespace {

struct Rhs {
  hplb_ctx*     ctx;
  int           n, nb, nrhs;
  const double* LU;
  int64_t       ld;
  const int*    ipiv;
  double*       B;
  int64_t       ldb;
  double *      W, *M1, *dvec, *dinv, *T, *SK;  // SK: split-k partial products
  int64_t       ldt;  // rows of T: n rounded up to 16, + 16, so a 16-row slab never leaves it
  int*          perm;
  cudaStream_t  st;

  static size_t ws_doubles(int n, int nb, int nrhs) {
    const size_t nblk = (size_t)nb / 32 + 1;
    return (size_t)nb * nrhs + (size_t)nb * nb + nb + nblk * 1024 + 64 +
           splitk_ws_doubles(nb, nrhs, std::max(n, 1));
  }
  void carve(double* base) {
    W    = base;
    M1   = W + (size_t)nb * nrhs;
    dvec = M1 + (size_t)nb * nb;
    dinv = dvec + nb;
    SK   = dinv + ((size_t)nb / 32 + 1) * 1024 + 64;
  }
  // C (m x nrhs) -= M (m x k) Y: the row-parallel kernel for few right-hand
  // sides, the DMMA GEMM otherwise.
  cudaError_t update(int m, int k, const double* M, int64_t ldm, const double* Y, int64_t ldy,
                     double* C, int64_t ldc) {
    if(nrhs <= 128) return launch_rows_sub(m, nrhs, k, M, ldm, Y, ldy, C, ldc, st);
    return launch_dgemm_sub(m, nrhs, k, M, ldm, Y, ldy, C, ldc, ctx->d_status, st);
  }
  // Few right-hand sides: one CTA per column; many: the blocked kernel.
  cudaError_t trsm(double* X, int64_t ldx, int jb, const double* L, int64_t ldl) {
    if(nrhs <= 128) return launch_trsm_small(jb, nrhs, X, ldx, L, ldl, dinv, st);
    return launch_trsm_unit_lower(X, ldx, jb, L, ldl, dinv, nrhs, st);
  }

  const double* lu(int i, int j) const { return LU + (size_t)i + (size_t)j * (size_t)ld; }
  double*       b(int i) const { return B + i; }
  const double* t(int i, int j) const { return T + (size_t)i + (size_t)j * (size_t)ldt; }

  // B[j : j + jb] <- L11^-1 B[j : j + jb], the unit-lower diagonal block of
  // panel j, by the blocked substitution (32 x 32 diagonal inverses, then
  // updates of the rows below), in place.
  hplb_status solve_lower(int j, int jb) {
    hplb_ctx* ctx = this->ctx;
    CK(launch_diag_inv<double>(LU, ld, j, j, jb, dinv, st));
    CK(trsm(b(j), ldb, jb, lu(j, j), ld));
    ctx->launches += 2;
    return HPLB_OK;
  }
  // B[j : j + jb] <- S^-1 B[j : j + jb] for S = U11 (kind 0), L11^T (kind 1)
  // or U11^T (kind 2), each solved as the unit-lower system it is equivalent
  // to (launch_unit_lower_view): U x = b is (J D^-1 U J)(J x) = J D^-1 b,
  // L^T x = b is (J L^T J)(J x) = J b, U^T x = b is (D^-1 U)^T (D x) = b.
  hplb_status solve_view(int kind, int j, int jb) {
    hplb_ctx* ctx = this->ctx;
    CK(launch_unit_lower_view(kind, jb, lu(j, j), ld, M1, dvec, st));
    CK(launch_diag_inv<double>(M1, jb, 0, 0, jb, dinv, st));
    CK(launch_rows_xform(jb, nrhs, b(j), ldb, W, jb, dvec, kind != 2, kind == 0, st));
    CK(trsm(W, jb, jb, M1, jb));
    CK(launch_rows_xform(jb, nrhs, W, jb, b(j), ldb, dvec, kind != 2, kind == 2, st));
    ctx->launches += 5;
    return HPLB_OK;
  }

  // B <- E_{np-1} P_{np-1} ... E_0 P_0 B, then B <- U^-1 B.
  hplb_status solve() {
    hplb_ctx*   ctx = this->ctx;
    hplb_status s;
    for(int j = 0; j < n; j += nb) {
      const int jb = std::min(nb, n - j);
      CK(launch_perm(ipiv + j, j, jb, perm, st));
      CK(launch_laswp_gather<double>(B, ldb, j, jb, perm, W, jb, 0, nrhs, st));
      CK(cudaMemcpy2DAsync(b(j), (size_t)ldb * sizeof(double), W, (size_t)jb * sizeof(double),
                           (size_t)jb * sizeof(double), nrhs, cudaMemcpyDeviceToDevice, st));
      if((s = solve_lower(j, jb)) != HPLB_OK) return s;
      CK(update(n - j - jb, jb, lu(j + jb, j), ld, b(j), ldb, b(j + jb), ldb));
      ctx->launches += 3;
    }
    if(nrhs <= 128) {  // U X = Y in one persistent launch per 32 right-hand sides
      CK(launch_trsm_upper(LU, ld, n, nrhs, B, ldb, B, ldb, ctx->d_trsv, ctx->d_status, st,
                           &ctx->launches));
      return HPLB_OK;
    }
    for(int j = (n - 1) / nb * nb; j >= 0; j -= nb) {
      const int jb = std::min(nb, n - j);
      if((s = solve_view(0, j, jb)) != HPLB_OK) return s;
      CK(update(j, jb, lu(0, j), ld, b(j), ldb, b(0), ldb));
      ctx->launches += 1;
    }
    return HPLB_OK;
  }

  // B <- U^-T B, then B <- P_0^T E_0^T ... P_{np-1}^T E_{np-1}^T B.
  hplb_status solve_t() {
    hplb_ctx*   ctx = this->ctx;
    hplb_status s;
    CK(launch_transpose<double>(n, n, LU, ld, T, ldt, st));
    ctx->launches += 1;
    for(int j = 0; j < n; j += nb) {  // U^T y = b, forward
      const int jb = std::min(nb, n - j);
      if((s = solve_view(2, j, jb)) != HPLB_OK) return s;
      CK(update(n - j - jb, jb, t(j + jb, j), ldt, b(j), ldb, b(j + jb), ldb));
      ctx->launches += 1;
    }
    for(int j = (n - 1) / nb * nb; j >= 0; j -= nb) {
      const int jb = std::min(nb, n - j);
      // y_top <- L11^-T (y_top - L21^T y_rest); the product has a long k and
      // few outputs, so it is split over k.
      const int K = n - j - jb;
      if(K > 4 * jb && nrhs <= 128) {
        CK(launch_splitk_sub(jb, nrhs, K, t(j, j + jb), ldt, b(j + jb), ldb, b(j), ldb, SK, st));
        ctx->launches += 2;
      } else {
        CK(launch_dgemm_sub(jb, nrhs, K, t(j, j + jb), ldt, b(j + jb), ldb, b(j), ldb,
                            ctx->d_status, st));
        ctx->launches += 1;
      }
      if((s = solve_view(1, j, jb)) != HPLB_OK) return s;
      CK(launch_perm(ipiv + j, j, jb, perm, st));
      CK(launch_laswp_inverse(B, ldb, j, jb, perm, nrhs, st));
      ctx->launches += 2;
    }
    return HPLB_OK;
  }
};

}  // namespace

extern "C" {

hplb_status hplb_getrs(hplb_ctx* ctx, int trans, int n, int nb, int nrhs, const double* dLU,
                       int64_t ld, const int* d_ipiv, double* dB, int64_t ldb) {
  if(!ctx) return HPLB_ERR_ARG;
  if(trans != 0 && trans != 1) return set_err(ctx, HPLB_ERR_ARG, "hplb_getrs: trans must be 0 or 1");
  if(n < 0 || nrhs < 0) return set_err(ctx, HPLB_ERR_ARG, "hplb_getrs: negative size");
  if(nb < 1 || nb > 2048) return set_err(ctx, HPLB_ERR_ARG, "hplb_getrs: NB must be in [1, 2048]");
  if(nrhs > 65535) return set_err(ctx, HPLB_ERR_UNSUPPORTED, "hplb_getrs: more than 65535 RHS");
  if(ld < std::max(1, n) || ldb < std::max(1, n))
    return set_err(ctx, HPLB_ERR_ARG, "hplb_getrs: leading dimension below max(1, n)");
  ctx->timing = hplb_timing{};
  if(n == 0 || nrhs == 0) return HPLB_OK;
  if(!dLU || !d_ipiv || !dB) return set_err(ctx, HPLB_ERR_ARG, "hplb_getrs: null pointer");
  ENTER(ctx);
  Rhs R{};
  R.ctx  = ctx;
  R.n    = n;
  R.nb   = std::min(nb, n);
  R.nrhs = nrhs;
  R.LU   = dLU;
  R.ld   = ld;
  R.ipiv = d_ipiv;
  R.B    = dB;
  R.ldb  = ldb;
  R.st   = ctx->s_upd;
  R.ldt  = ((int64_t)n + 15) / 16 * 16 + 16;
  hplb_status s;
  if((s = grow(ctx, &ctx->r_ws, &ctx->r_ws_cap, Rhs::ws_doubles(n, R.nb, nrhs))) != HPLB_OK ||
     (s = grow(ctx, &ctx->r_perm, &ctx->r_perm_cap, 2 * (size_t)R.nb)) != HPLB_OK)
    return s;
  if(trans && (s = grow(ctx, &ctx->r_t, &ctx->r_t_cap, (size_t)R.ldt * n)) != HPLB_OK) return s;
  if((s = grow(ctx, &ctx->d_trsv, &ctx->trsv_cap, trsv_flag_ints(n))) != HPLB_OK) return s;
  R.carve(ctx->r_ws);
  R.perm = ctx->r_perm;
  R.T    = ctx->r_t;

  // Pivots index rows: check them before any kernel uses them.
  CK(cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), R.st));
  CK(launch_check_ipiv(n, d_ipiv, ctx->d_status, R.st));
  CK(cudaStreamSynchronize(R.st));
  int bad = 0;
  if((s = read_status(ctx, &bad)) != HPLB_OK) return s;
  if(bad) return set_err(ctx, HPLB_ERR_ARG, "hplb_getrs: ipiv[%d] outside [%d, n)", bad - 1, bad - 1);

  ctx->ev_next  = 0;
  ctx->launches = 0;
  cudaEvent_t e0 = next_event(ctx), e1 = next_event(ctx);
  CK(cudaEventRecord(e0, R.st));
  if((s = trans ? R.solve_t() : R.solve()) != HPLB_OK) return s;
  CK(cudaEventRecord(e1, R.st));
  {
    cudaError_t e = cudaStreamSynchronize(R.st);
    if(e != cudaSuccess) return set_err(ctx, HPLB_ERR_CUDA, "hplb_getrs: %s", cudaGetErrorString(e));
  }
  if((s = read_status(ctx, nullptr)) != HPLB_OK) return s;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  ctx->timing.total_ms        = ms;
  ctx->timing.trsv_ms         = ms;
  ctx->timing.kernel_launches = ctx->launches;
  return HPLB_OK;
}

hplb_status hplb_rank_k(hplb_ctx* ctx, int m, int n, int k, double alpha, const double* dA,
                        int64_t lda, const double* dB, int64_t ldb, double* dC, int64_t ldc,
                        int accumulate) {
  if(!ctx) return HPLB_ERR_ARG;
  if(m < 0 || n < 0 || k < 0) return set_err(ctx, HPLB_ERR_ARG, "hplb_rank_k: negative size");
  if(k > 64) return set_err(ctx, HPLB_ERR_UNSUPPORTED, "hplb_rank_k: k above 64");
  if(lda < std::max(1, m) || ldb < std::max(1, n) || ldc < std::max(1, m))
    return set_err(ctx, HPLB_ERR_ARG, "hplb_rank_k: leading dimension too small");
  if(m == 0 || n == 0) return HPLB_OK;
  if(!dC || (k > 0 && (!dA || !dB))) return set_err(ctx, HPLB_ERR_ARG, "hplb_rank_k: null pointer");
  if((n + 63) / 64 > 65535) return set_err(ctx, HPLB_ERR_UNSUPPORTED, "hplb_rank_k: n too large");
  ENTER(ctx);
  ctx->ev_next   = 0;
  cudaEvent_t e0 = next_event(ctx), e1 = next_event(ctx);
  CK(cudaEventRecord(e0, ctx->s_upd));
  CK(launch_rank_k(m, n, k, alpha, dA, lda, dB, ldb, dC, ldc, accumulate != 0, ctx->s_upd));
  CK(cudaEventRecord(e1, ctx->s_upd));
  CK(cudaStreamSynchronize(ctx->s_upd));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  ctx->timing                 = hplb_timing{};
  ctx->timing.total_ms        = ms;
  ctx->timing.kernel_launches = 1;
  return HPLB_OK;
}

}  // extern "C"
