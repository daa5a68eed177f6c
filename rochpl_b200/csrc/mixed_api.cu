// hplb_pdgesv_mixed: low-precision LU + GMRES iterative refinement.
//
// Factorisation (FP32 storage, same panel order, pivoting and look-ahead as the
// FP64 path of src/pgesv/HPL_pdgesv.cpp):
//   W = fp32(A)                                   (stored A, or the LCG itself)
//   panel stream, per panel p: FP32 recursive panel (FP32 leaf with partial
//     pivoting), its row map, and L11^-1 and U11^-1 kept for the preconditioner;
//   update stream: U12 = L11^-1 P A12 in FP32, then A22 -= L21 U12 on the tensor
//     cores from per-tile scaled 16-bit copies with FP32 accumulation
//     (gemm_lp.cu); the next panel is factored while the bulk update runs.
// Refinement (FP64): x = M^-1 b with M^-1 = U^-1 L^-1 P applied block by
// block from the stored inverses and the FP32 factors; then while the HPL
// scaled residual is above target: r = b - A x against the FP64 A, one cycle
// of right-preconditioned flexible GMRES for A d = r, x += d.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ctx.h"

using namespace hplb;

namespace {

struct Mixed {
  hplb_ctx*        ctx;
  const hplb_algo* algo;
  int              n, nb, npan, ldp;
  int64_t          ldw;
  bool             bf16;
  bool             split;  // hi/lo 16-bit parts: K = 3 jb
  float*           W;
  cudaStream_t     st;     // stream of the recursion (the panel stream while factoring)
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> gemm_ev, panel_ev;
  std::vector<double>                              gemm_flops;

  float* w(int i, int j) const { return W + (size_t)i + (size_t)j * (size_t)ldw; }
  float* linv(int p) const { return ctx->m_linv + (size_t)p * nb * nb; }
  float* uinv(int p) const { return ctx->m_uinv + (size_t)p * nb * nb; }
  int*   perm(int p) const { return ctx->m_perm + (size_t)p * 2 * nb; }
  float* dinv() const { return ctx->m_small; }  // (nb/32+1)*1024
  float* dinv_piece() const { return ctx->m_small + ((size_t)nb / 32 + 1) * 1024; }
  float* upper_work() const { return ctx->m_small + 2 * ((size_t)nb / 32 + 1) * 1024; }

  hplb_status leaf(int r0, int c0, int wdt, int pc, int pw) {
    hplb_ctx* ctx  = this->ctx;
    const int grid = leaf_grid_size(ctx->num_sms, n - r0);
    bool swapped = false;
    CK(launch_leaf<float>(W, ldw, r0, n, c0, wdt, pc, pw, ctx->d_ipiv, ctx->d_cand, ctx->d_cur,
                          ctx->d_bar, ctx->d_status, grid, ctx->leaf_kind, st, &swapped));
    ctx->launches += 1;
    if(!swapped) {
      CK(launch_panel_swap<float>(W, ldw, ctx->d_ipiv, r0, c0, wdt, pc, pw, st));
      ctx->launches += 1;
    }
    return HPLB_OK;
  }

  // FP32 recursive panel, with the orderings of the FP64 driver.
  hplb_status rpanel(int r0, int c0, int N, int pc, int pw) {
    hplb_ctx*   ctx   = this->ctx;
    const int   nbmin = std::min(std::max(algo->nbmin, 1), kMaxLeaf);
    const int   ndiv  = std::max(algo->ndiv, 2);
    hplb_status s;
    if(N <= nbmin) return leaf(r0, c0, N, pc, pw);
    const int nbs = (((N + nbmin - 1) / nbmin + ndiv - 1) / ndiv) * nbmin;
    int       jj = 0, rem = N, jb = nbs;
    if(algo->rfact == 2) {
      do {
        rem -= jb;
        if((s = rpanel(r0 + jj, c0 + jj, jb, pc, pw)) != HPLB_OK) return s;
        if(rem > 0) {
          CK(launch_trsm_node<float>(W, ldw, r0 + jj, jb, c0 + jj, dinv_piece(), c0 + jj + jb,
                                     rem, st, &ctx->launches));
          CK(launch_sgemm(n - (r0 + jj + jb), rem, jb, w(r0 + jj + jb, c0 + jj), ldw,
                          w(r0 + jj, c0 + jj + jb), ldw, w(r0 + jj + jb, c0 + jj + jb), ldw,
                          true, st));
          ctx->launches += 1;
        }
        jj += jb;
        jb = std::min(rem, nbs);
      } while(rem > 0);
    } else {
      do {
        rem -= jb;
        const int cj = c0 + jj;
        if(jj > 0) {
          CK(launch_trsm_node<float>(W, ldw, r0, jj, c0, dinv_piece(), cj, jb, st,
                                     &ctx->launches));
          CK(launch_sgemm(n - (r0 + jj), jb, jj, w(r0 + jj, c0), ldw, w(r0, cj), ldw,
                          w(r0 + jj, cj), ldw, true, st));
          ctx->launches += 1;
        }
        if((s = rpanel(r0 + jj, cj, jb, pc, pw)) != HPLB_OK) return s;
        jj += jb;
        jb = std::min(rem, nbs);
      } while(rem > 0);
    }
    return HPLB_OK;
  }

  // Panel p on the panel stream: recursive FP32 factorisation, its row map and
  // the diagonal-block inverses the update and the preconditioner use.
  hplb_status panel(int p, cudaEvent_t done) {
    hplb_ctx*    ctx = this->ctx;
    hplb_status  s;
    const int    j = p * nb, jb = std::min(nb, n - j);
    cudaStream_t keep = st;
    st = ctx->s_pan;
    cudaEvent_t p0 = next_event(ctx), p1 = next_event(ctx);
    CK(cudaEventRecord(p0, st));
    if((s = rpanel(j, j, jb, j, jb)) != HPLB_OK) return s;
    CK(launch_perm(ctx->d_ipiv + j, j, jb, perm(p), st));
    CK(launch_diag_inv<float>(W, ldw, j, j, jb, dinv(), st));
    CK(launch_unit_lower_inverse<float>(w(j, j), ldw, jb, dinv(), linv(p), jb, st));
    CK(launch_upper_inverse(jb, w(j, j), ldw, uinv(p), upper_work(), dinv_piece(), st));
    ctx->launches += 9;
    CK(cudaEventRecord(p1, st));
    CK(cudaEventRecord(done, st));
    panel_ev.emplace_back(p0, p1);
    st = keep;
    return HPLB_OK;
  }

  // Update of panel p on columns [c, c + wd) (update stream): interchanges,
  // U12 = L11^-1 W in FP32, then the 16-bit tensor-core update.  pack_l packs
  // L21 (once per panel, on its first call).
  hplb_status update(int p, int c, int wd, bool pack_l) {
    hplb_ctx* ctx = this->ctx;
    if(wd <= 0) return HPLB_OK;
    const int    j = p * nb, jb = std::min(nb, n - j), c1 = j + jb, m = n - c1;
    cudaStream_t su = ctx->s_upd;
    float*       sL = ctx->m_scale;
    float*       sU = ctx->m_scale + ((size_t)n + 127) / 128 + 1;
    CK(launch_laswp_gather<float>(W, ldw, j, jb, perm(p), ctx->m_g, jb, c, wd, su));
    if(split) {
      // U12 = L11^-1 G on the tensor cores, with the split operands of the
      // trailing update (FP32-accurate): C = 0, then C -= (-L11^-1) G.
      float* sLi = sU + ((size_t)n + 255) / 256 + 1;
      float* sG  = sLi + 32;
      CK(launch_pack_l(bf16, true, jb, jb, linv(p), jb, ctx->m_li16, ldp, sLi, su, -1.f));
      CK(launch_pack_u(bf16, true, jb, wd, ctx->m_g, jb, ctx->m_u16, ldp, sG, su));
      CK(cudaMemset2DAsync(w(j, c), (size_t)ldw * sizeof(float), 0, (size_t)jb * sizeof(float), wd,
                           su));
      CK(launch_gemm_lp(bf16, jb, wd, 3 * jb, ctx->m_li16, ldp, ctx->m_u16, ldp, sLi, sG, w(j, c),
                        ldw, ctx->d_status, su));
      ctx->launches += 5;
    } else {
      CK(launch_sgemm(jb, wd, jb, linv(p), jb, ctx->m_g, jb, w(j, c), ldw, false, su));
      ctx->launches += 2;
    }
    if(m <= 0) return HPLB_OK;
    if(pack_l) CK(launch_pack_l(bf16, split, m, jb, w(c1, j), ldw, ctx->m_l16, ldp, sL, su));
    CK(launch_pack_u(bf16, split, jb, wd, w(j, c), ldw, ctx->m_u16, ldp, sU, su));
    ctx->launches += pack_l ? 3 : 2;
    const int   kk = split ? 3 * jb : jb;
    cudaEvent_t g0 = next_event(ctx), g1 = next_event(ctx);
    CK(cudaEventRecord(g0, su));
    CK(launch_gemm_lp(bf16, m, wd, kk, ctx->m_l16, ldp, ctx->m_u16, ldp, sL, sU, w(c1, c), ldw,
                      ctx->d_status, su));
    CK(cudaEventRecord(g1, su));
    gemm_ev.emplace_back(g0, g1);
    gemm_flops.push_back(2.0 * m * (double)wd * kk);
    return HPLB_OK;
  }

  // Look-ahead depth 1, as the FP64 driver: the next panel is factored on the
  // panel stream while the rest of the current update runs.
  hplb_status factor() {
    hplb_ctx*   ctx = this->ctx;
    hplb_status s;
    cudaEvent_t evp[2] = {next_event(ctx), next_event(ctx)};
    cudaEvent_t start  = next_event(ctx);
    CK(cudaEventRecord(start, ctx->s_upd));
    CK(cudaStreamWaitEvent(ctx->s_pan, start, 0));
    if((s = panel(0, evp[0])) != HPLB_OK) return s;
    for(int p = 0; p < npan; ++p) {
      const int j = p * nb, jb = std::min(nb, n - j), c1 = j + jb;
      CK(cudaStreamWaitEvent(ctx->s_upd, evp[p & 1], 0));
      const int la = c1 < n ? std::min(nb, n - c1) : 0;
      if((s = update(p, c1, la, true)) != HPLB_OK) return s;
      if(la > 0) {
        cudaEvent_t ev_la = next_event(ctx);
        CK(cudaEventRecord(ev_la, ctx->s_upd));
        CK(cudaStreamWaitEvent(ctx->s_pan, ev_la, 0));
        if((s = panel(p + 1, evp[(p + 1) & 1])) != HPLB_OK) return s;
      }
      if((s = update(p, c1 + la, n - (c1 + la), false)) != HPLB_OK) return s;
    }
    return HPLB_OK;
  }

  // The preconditioner M^-1 = U^-1 L^-1 P applied to the fixed vector pv
  // (update stream): per panel forward, the row map, pv_top = L11^-1 pv_top
  // (out of place through ptmp), pv_rest -= L21 pv_top; per panel backward,
  // pv_top = U11^-1 pv_top, pv_above -= U12' pv_top.
  double*         pv     = nullptr;  // n doubles
  double*         ptmp   = nullptr;  // nb doubles
  cudaGraphExec_t pgraph = nullptr;
  int             plaunches = 0;

  hplb_status precond_body() {
    hplb_ctx*    ctx = this->ctx;
    cudaStream_t su  = ctx->s_upd;
    for(int p = 0; p < npan; ++p) {
      const int j = p * nb, jb = std::min(nb, n - j);
      CK(launch_perm_vec(pv, j, jb, perm(p), su));
      CK(launch_gemv_set(jb, jb, linv(p), jb, pv + j, ptmp, su));
      CK(cudaMemcpyAsync(pv + j, ptmp, (size_t)jb * sizeof(double), cudaMemcpyDeviceToDevice, su));
      CK(launch_gemv_sub(n - j - jb, jb, w(j + jb, j), ldw, pv + j, pv + j + jb, su));
      plaunches += j + jb < n ? 3 : 2;
    }
    for(int p = npan - 1; p >= 0; --p) {
      const int j = p * nb, jb = std::min(nb, n - j);
      CK(launch_gemv_set(jb, jb, uinv(p), jb, pv + j, ptmp, su));
      CK(cudaMemcpyAsync(pv + j, ptmp, (size_t)jb * sizeof(double), cudaMemcpyDeviceToDevice, su));
      CK(launch_gemv_sub(j, jb, w(0, j), ldw, pv + j, pv, su));
      plaunches += j > 0 ? 2 : 1;
    }
    return HPLB_OK;
  }

  // The sweep is captured once per factorisation as a CUDA graph (about
  // 1800 small launches per application otherwise).
  hplb_status build_precond() {
    hplb_ctx*   ctx = this->ctx;
    cudaGraph_t g   = nullptr;
    plaunches       = 0;
    CK(cudaStreamBeginCapture(ctx->s_upd, cudaStreamCaptureModeThreadLocal));
    hplb_status s  = precond_body();
    cudaError_t e  = cudaStreamEndCapture(ctx->s_upd, &g);
    if(s == HPLB_OK && e == cudaSuccess) e = cudaGraphInstantiate(&pgraph, g, 0);
    if(g) cudaGraphDestroy(g);
    if(s != HPLB_OK) return s;
    if(e != cudaSuccess) {
      cudaGetLastError();
      pgraph = nullptr;
      return set_err(ctx, HPLB_ERR_CUDA, "preconditioner graph: %s", cudaGetErrorString(e));
    }
    return HPLB_OK;
  }

  // z <- M^-1 z (update stream).
  hplb_status precond(double* z) {
    hplb_ctx*    ctx = this->ctx;
    cudaStream_t su  = ctx->s_upd;
    hplb_status  s;
    if(!pgraph && (s = build_precond()) != HPLB_OK) return s;
    CK(cudaMemcpyAsync(pv, z, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, su));
    CK(cudaGraphLaunch(pgraph, su));
    CK(cudaMemcpyAsync(z, pv, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, su));
    ctx->launches += plaunches;
    return HPLB_OK;
  }

  ~Mixed() {
    if(pgraph) cudaGraphExecDestroy(pgraph);
  }
};

// FP64 refinement state: the GMRES basis V (restart+1 vectors), the
// preconditioned directions Z (restart), b, r, x and a scratch vector, all on
// the device; the Hessenberg matrix and the rotations on the host.
struct Refine {
  hplb_ctx*     ctx;
  Mixed*        M;
  int           n, restart;
  const double* A;  // stored FP64 A, or null for the LCG
  int64_t       ld;
  bool          lcg;
  uint64_t      seed;
  double *      V, *Z, *b, *r, *t, *part, *sc;
  double        anorm = 0, bnorm = 0, eps = 0;

  double* v(int i) const { return V + (size_t)i * n; }
  double* z(int i) const { return Z + (size_t)i * n; }

  static size_t nparts(int restart) {
    return std::max(mdot_partials(restart + 1), (size_t)vec_partials());
  }
  static size_t doubles(int n, int restart) {
    return (size_t)(2 * restart + 4) * n + nparts(restart) + 4 * (restart + 2) + 8;
  }
  void carve(double* base) {
    V    = base;
    Z    = V + (size_t)(restart + 1) * n;
    b    = Z + (size_t)restart * n;
    r    = b + n;
    t    = r + n;
    part = t + n;
    sc   = part + nparts(restart);
  }

  // y = A x in FP64 (stored A or the LCG regenerated).
  hplb_status amul(const double* x, double* y) {
    hplb_ctx* ctx = this->ctx;
    CK(launch_gemv_hpl(n, A, ld, lcg, seed, x, y, ctx->d_res, ctx->s_upd));
    ctx->launches += 2;
    return HPLB_OK;
  }

  // r = b - A x and the HPL scaled residual of x.
  hplb_status residual(const double* x, double* resid) {
    hplb_ctx*   ctx = this->ctx;
    hplb_status s;
    if((s = amul(x, t)) != HPLB_OK) return s;
    CK(launch_sub(n, b, t, r, ctx->s_upd));
    CK(launch_amax(n, r, part, sc, ctx->s_upd));
    CK(launch_amax(n, x, part, sc + 1, ctx->s_upd));
    ctx->launches += 5;
    double h[2];
    CK(cudaMemcpyAsync(h, sc, sizeof h, cudaMemcpyDeviceToHost, ctx->s_upd));
    CK(cudaStreamSynchronize(ctx->s_upd));
    *resid = h[0] / (eps * (anorm * h[1] + bnorm) * (double)n);
    return HPLB_OK;
  }

  // One cycle of right-preconditioned flexible GMRES for A d = r, x += d.
  // Gram-Schmidt is classical with one re-orthogonalisation pass (CGS2), so a
  // step needs a single device-to-host read.
  hplb_status cycle(double* x, double tol, int* iters) {
    hplb_ctx*    ctx = this->ctx;
    cudaStream_t su  = ctx->s_upd;
    hplb_status  s;
    const int    R = restart;
    std::vector<double> H((size_t)(R + 1) * R, 0.0), cs(R), sn(R), g(R + 1, 0.0);
    auto hh = [&](int i, int k) -> double& { return H[(size_t)i + (size_t)k * (R + 1)]; };

    CK(launch_dot(n, r, r, part, sc, su));
    ctx->launches += 2;
    double beta = 0;
    CK(cudaMemcpyAsync(&beta, sc, sizeof beta, cudaMemcpyDeviceToHost, su));
    CK(cudaStreamSynchronize(su));
    beta = std::sqrt(beta);
    *iters = 0;
    if(!(beta > 0)) return HPLB_OK;
    CK(launch_scal_copy(n, 1.0 / beta, r, v(0), su));
    ctx->launches += 1;
    g[0]   = beta;
    int it = 0;
    std::vector<double> hv(2 * (R + 1) + 1);
    for(int k = 0; k < R; ++k) {
      CK(cudaMemcpyAsync(z(k), v(k), (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, su));
      if((s = M->precond(z(k))) != HPLB_OK) return s;
      if((s = amul(z(k), t)) != HPLB_OK) return s;
      double* h1 = sc;
      double* h2 = sc + (R + 1);
      double* nr = sc + 2 * (R + 1);
      CK(launch_mdot(n, k + 1, V, n, t, part, h1, su));
      CK(launch_mgemv_sub(n, k + 1, V, n, h1, t, nullptr, su));
      CK(launch_mdot(n, k + 1, V, n, t, part, h2, su));
      CK(launch_mgemv_sub(n, k + 1, V, n, h2, t, nullptr, su));
      CK(launch_dot(n, t, t, part, nr, su));
      ctx->launches += 8;
      CK(cudaMemcpyAsync(hv.data(), sc, hv.size() * sizeof(double), cudaMemcpyDeviceToHost, su));
      CK(cudaStreamSynchronize(su));
      for(int i = 0; i <= k; ++i) hh(i, k) = hv[i] + hv[R + 1 + i];
      const double hk1 = std::sqrt(std::max(hv[2 * (R + 1)], 0.0));
      hh(k + 1, k)     = hk1;
      if(hk1 > 0) {
        CK(launch_scal_copy(n, 1.0 / hk1, t, v(k + 1), su));
        ctx->launches += 1;
      }
      for(int i = 0; i < k; ++i) {  // previous rotations on column k
        const double a = hh(i, k), c = hh(i + 1, k);
        hh(i, k)       = cs[i] * a + sn[i] * c;
        hh(i + 1, k)   = -sn[i] * a + cs[i] * c;
      }
      const double a = hh(k, k), c = hh(k + 1, k), d = std::hypot(a, c);
      cs[k]          = d > 0 ? a / d : 1.0;
      sn[k]          = d > 0 ? c / d : 0.0;
      hh(k, k)       = d;
      hh(k + 1, k)   = 0.0;
      g[k + 1]       = -sn[k] * g[k];
      g[k]           = cs[k] * g[k];
      it             = k + 1;
      if(std::fabs(g[k + 1]) <= tol * beta || !(hk1 > 0)) break;
    }
    // y = H^-1 g (upper triangular), then x += Z y.
    std::vector<double> y(it);
    for(int i = it - 1; i >= 0; --i) {
      double acc = g[i];
      for(int j = i + 1; j < it; ++j) acc -= hh(i, j) * y[j];
      y[i] = hh(i, i) != 0 ? acc / hh(i, i) : 0.0;
    }
    for(int i = 0; i < it; ++i) CK(launch_axpy(n, y[i], z(i), x, su));
    ctx->launches += it;
    *iters = it;
    return HPLB_OK;
  }
};

}  // namespace

extern "C" hplb_status hplb_pdgesv_mixed(hplb_ctx* ctx, const hplb_algo* algo,
                                         const hplb_mixed_opts* opts, int n, const double* dA,
                                         int64_t ld, uint64_t seed, double* dX, int* ipiv_out,
                                         hplb_mixed_report* report) {
  if(!ctx) return HPLB_ERR_ARG;
  hplb_status s = check_algo(ctx, algo, n, ld, dA != nullptr);
  if(s != HPLB_OK) return s;
  hplb_mixed_opts o{2, 20, 20, 16.0, 1e-6};
  if(opts) {
    o.precision = opts->precision;
    if(opts->restart > 0) o.restart = opts->restart;
    if(opts->max_outer > 0) o.max_outer = opts->max_outer;
    if(opts->target_resid > 0) o.target_resid = opts->target_resid;
    if(opts->gmres_tol > 0) o.gmres_tol = opts->gmres_tol;
  }
  if(o.precision < 0 || o.precision > 3)
    return set_err(ctx, HPLB_ERR_ARG, "hplb_pdgesv_mixed: precision %d out of range", o.precision);
  if(o.restart > 60)
    return set_err(ctx, HPLB_ERR_UNSUPPORTED, "hplb_pdgesv_mixed: restart above 60");
  hplb_mixed_report rep{};
  if(report) *report = rep;
  ctx->timing = hplb_timing{};
  if(n == 0) return HPLB_OK;
  if(!dX) return set_err(ctx, HPLB_ERR_ARG, "hplb_pdgesv_mixed: null solution");
  ENTER(ctx);

  Mixed M{};
  M.ctx   = ctx;
  M.algo  = algo;
  M.n     = n;
  M.nb    = std::min(algo->nb, n);
  M.npan  = (n + M.nb - 1) / M.nb;
  M.bf16  = (o.precision & 1) == 0;
  M.split = o.precision >= 2;
  M.ldp   = ((M.split ? 3 : 1) * M.nb + 7) / 8 * 8;
  M.ldw   = ((int64_t)n + 31) / 32 * 32;
  const int    nb   = M.nb;
  const size_t nblk = (size_t)nb / 32 + 1;
  const size_t nn   = (size_t)M.ldw * (size_t)n;
  if((s = ensure_leaf_ws(ctx, n, algo->nbmin)) != HPLB_OK ||
     (s = grow(ctx, &ctx->m_w, &ctx->m_w_cap, nn)) != HPLB_OK ||
     (s = grow(ctx, &ctx->m_linv, &ctx->m_linv_cap, (size_t)M.npan * nb * nb)) != HPLB_OK ||
     (s = grow(ctx, &ctx->m_uinv, &ctx->m_uinv_cap, (size_t)M.npan * nb * nb)) != HPLB_OK ||
     (s = grow(ctx, &ctx->m_perm, &ctx->m_perm_cap, (size_t)M.npan * 2 * nb)) != HPLB_OK ||
     (s = grow(ctx, &ctx->m_g, &ctx->m_g_cap, (size_t)nb * n)) != HPLB_OK ||
     (s = grow(ctx, &ctx->m_l16, &ctx->m_l16_cap, (size_t)M.ldp * n)) != HPLB_OK ||
     (s = grow(ctx, &ctx->m_u16, &ctx->m_u16_cap, (size_t)M.ldp * n)) != HPLB_OK ||
     (s = grow(ctx, &ctx->m_scale, &ctx->m_scale_cap, (size_t)n / 64 + 96)) != HPLB_OK ||
     (s = grow(ctx, &ctx->m_li16, &ctx->m_li16_cap, (size_t)M.ldp * nb)) != HPLB_OK ||
     (s = grow(ctx, &ctx->m_small, &ctx->m_small_cap,
               2 * nblk * 1024 + 2 * (size_t)nb * nb + nb + 64)) != HPLB_OK ||
     (s = grow(ctx, &ctx->m_vec, &ctx->m_vec_cap,
               Refine::doubles(n, o.restart) + (size_t)n + nb + 16)) != HPLB_OK ||
     (s = grow(ctx, &ctx->d_res, &ctx->res_cap, residual_ws_doubles(n))) != HPLB_OK)
    return s;
  M.W = ctx->m_w;

  ctx->ev_next  = 0;
  ctx->launches = 0;
  cudaStream_t su = ctx->s_upd;
  CK(cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), su));
  cudaEvent_t e0 = next_event(ctx), e1 = next_event(ctx), e2 = next_event(ctx);
  CK(cudaEventRecord(e0, su));
  if(dA)
    CK(launch_f64_to_f32(n, n, dA, ld, M.W, M.ldw, su));
  else
    CK(launch_matgen_f32(n, n, seed, M.W, M.ldw, su));
  ctx->launches += 1;
  M.st = ctx->s_pan;
  if((s = M.factor()) != HPLB_OK) return s;
  CK(cudaEventRecord(e1, su));
  if(ipiv_out)
    CK(cudaMemcpyAsync(ipiv_out, ctx->d_ipiv, (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice,
                       su));
  {
    cudaError_t e = cudaStreamSynchronize(su);
    if(e == cudaSuccess) e = cudaStreamSynchronize(ctx->s_pan);
    if(e != cudaSuccess)
      return set_err(ctx, HPLB_ERR_CUDA, "mixed LU failed: %s", cudaGetErrorString(e));
  }
  int info = 0;
  if((s = read_status(ctx, &info)) != HPLB_OK) return s;
  rep.info = info;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  rep.lu_ms = ms;
  for(size_t i = 0; i < M.gemm_ev.size(); ++i) {
    cudaEventElapsedTime(&ms, M.gemm_ev[i].first, M.gemm_ev[i].second);
    rep.gemm_ms += ms;
    rep.gemm_flops += M.gemm_flops[i];
  }
  for(auto& p : M.panel_ev) {
    cudaEventElapsedTime(&ms, p.first, p.second);
    rep.panel_ms += ms;
  }
  if(info != 0) {
    if(report) *report = rep;
    return set_err(ctx, HPLB_ERR_SINGULAR, "zero pivot in column %d of the FP32 panel", info);
  }

  // ---- refinement ----
  Refine F{};
  F.ctx     = ctx;
  F.M       = &M;
  F.n       = n;
  F.restart = o.restart;
  F.A       = dA;
  F.ld      = ld;
  F.lcg     = dA == nullptr;
  F.seed    = seed;
  F.carve(ctx->m_vec);
  M.pv   = ctx->m_vec + Refine::doubles(n, o.restart);
  M.ptmp = M.pv + n;
  // ||A||oo, ||b||oo and eps from the residual kernels at x = 0.
  CK(cudaMemsetAsync(dX, 0, (size_t)n * sizeof(double), su));
  CK(launch_residual(n, dA, ld, F.lcg, seed, dX, ctx->d_res, ctx->d_out8, su));
  CK(launch_column_hpl(n, n, dA, ld, F.lcg, seed, F.b, ctx->d_res, su));
  ctx->launches += 5;
  double o8[8];
  CK(cudaMemcpyAsync(o8, ctx->d_out8, sizeof o8, cudaMemcpyDeviceToHost, su));
  CK(cudaStreamSynchronize(su));
  F.anorm = o8[3];
  F.bnorm = o8[6];
  F.eps   = o8[7];

  CK(cudaMemcpyAsync(dX, F.b, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, su));
  if((s = M.precond(dX)) != HPLB_OK) return s;
  double resid = 0;
  if((s = F.residual(dX, &resid)) != HPLB_OK) return s;
  rep.resid_lu = resid;
  while(!(resid < o.target_resid) && rep.outer_iters < o.max_outer) {
    int it = 0;
    if((s = F.cycle(dX, o.gmres_tol, &it)) != HPLB_OK) return s;
    rep.outer_iters += 1;
    rep.gmres_iters += it;
    if((s = F.residual(dX, &resid)) != HPLB_OK) return s;
    if(it == 0) break;
  }
  CK(cudaEventRecord(e2, su));
  CK(cudaEventSynchronize(e2));
  if((s = read_status(ctx, nullptr)) != HPLB_OK) return s;
  cudaEventElapsedTime(&ms, e1, e2);
  rep.ir_ms     = ms;
  rep.total_ms  = rep.lu_ms + rep.ir_ms;
  rep.resid     = resid;
  rep.converged = resid < o.target_resid ? 1 : 0;
  if(report) *report = rep;

  hplb_timing& T    = ctx->timing;
  T.total_ms        = rep.total_ms;
  T.lu_ms           = rep.lu_ms;
  T.trsv_ms         = rep.ir_ms;
  T.gemm_ms         = rep.gemm_ms;
  T.gemm_flops      = rep.gemm_flops;
  T.panel_ms        = rep.panel_ms;
  T.gemm_launches   = (int)M.gemm_ev.size();
  T.kernel_launches = ctx->launches;
  return HPLB_OK;
}
