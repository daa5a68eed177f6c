// Host runtime and C ABI of libhplb200 (include/hplb.h).
//
// hplb_pdgesv is the single-process HPL_pdgesv (src/pgesv/HPL_pdgesv.cpp:19-368)
// with look-ahead depth 1 made real on the GPU: the panel factorisation runs on
// a high-priority stream concurrently with the bulk of the previous panel's
// trailing update on the update stream.  Per panel j:
//
//   update stream : wait(panel j) -> swap+TRSM and DGEMM on the next panel's
//                   columns (look-ahead) -> record -> swap+TRSM and DGEMM on
//                   the rest of the trailing matrix, b included
//   panel stream  :                       wait(look-ahead) -> factor panel j+1
//
// which is the order of :182-191 with the two halves genuinely overlapped.
// Pivots never leave the device: the leaf kernel records them and a tiny
// kernel turns them into the row map the trailing swap uses (the reference
// copies pivots to the host and back once per panel, HPL_pdpanel_swapids.cpp).
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.h"

using namespace hplb;

namespace {

hplb_status ensure_solve_ws(hplb_ctx* ctx, int n, int nb, int nbmin, int nrhs = 1) {
  hplb_status s;
  if((s = grow(ctx, &ctx->d_ipiv, &ctx->ipiv_cap, (size_t)std::max(n, 1))) != HPLB_OK) return s;
  if(nb > ctx->nb_cap) {
    for(int i = 0; i < 2; ++i) {
      if(ctx->d_perm[i]) cudaFree(ctx->d_perm[i]);
      if(ctx->d_dinv[i]) cudaFree(ctx->d_dinv[i]);
      if(ctx->d_linv[i]) cudaFree(ctx->d_linv[i]);
      ctx->d_perm[i] = nullptr;
      ctx->d_dinv[i] = nullptr;
      ctx->d_linv[i] = nullptr;
    }
    if(ctx->d_dinv_piece) cudaFree(ctx->d_dinv_piece);
    ctx->d_dinv_piece = nullptr;
    const size_t nblk = (size_t)(nb + 31) / 32 + 1;
    for(int i = 0; i < 2; ++i) {
      if(cudaMalloc(&ctx->d_perm[i], 2 * (size_t)nb * sizeof(int)) != cudaSuccess ||
         cudaMalloc(&ctx->d_dinv[i], nblk * 32 * 32 * sizeof(double)) != cudaSuccess ||
         cudaMalloc(&ctx->d_linv[i], (size_t)nb * nb * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return set_err(ctx, HPLB_ERR_OOM, "panel workspace allocation failed");
      }
    }
    if(cudaMalloc(&ctx->d_dinv_piece, nblk * 32 * 32 * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      return set_err(ctx, HPLB_ERR_OOM, "panel workspace allocation failed");
    }
    ctx->nb_cap = nb;
  }
  if(n > 0 &&
     (s = grow(ctx, &ctx->d_w, &ctx->w_cap, (size_t)nb * (size_t)(n + std::max(nrhs, 1)))) !=
         HPLB_OK)
    return s;
  if((s = grow(ctx, &ctx->d_trsv, &ctx->trsv_cap, trsv_flag_ints(std::max(n, 1)))) != HPLB_OK)
    return s;
  return ensure_leaf_ws(ctx, n, nbmin);
}

struct Solve {
  hplb_ctx*        ctx;
  const hplb_algo* algo;
  double*          A;
  int64_t          ld;
  int              n;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> gemm_ev;
  std::vector<double>                              gemm_flops;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> panel_ev;

  double* a(int i, int j) const { return A + (size_t)i + (size_t)j * (size_t)ld; }

  // Leaf plus the propagation of its interchanges to the rest of the panel.
  hplb_status leaf(int r0, int c0, int w, int pc, int pw) {
    hplb_ctx* ctx  = this->ctx;
    const int grid = leaf_grid_size(ctx->num_sms, n - r0);
    bool swapped = false;
    CK(launch_leaf(A, ld, r0, n, c0, w, pc, pw, ctx->d_ipiv, ctx->d_cand, ctx->d_cur,
                   ctx->d_bar, ctx->d_status, grid, ctx->leaf_kind, ctx->s_pan, &swapped));
    ctx->launches += 1;
    if(!swapped) {
      CK(launch_panel_swap(A, ld, ctx->d_ipiv, r0, c0, w, pc, pw, ctx->s_pan));
      ctx->launches += 1;
    }
    return HPLB_OK;
  }

  // Recursive panel factorisation of rows [r0, n) x columns [c0, c0+N) of the
  // panel [pc, pc+pw) (src/pfact/HPL_pdrpanrlT.cpp:74-160 and the left / Crout
  // orderings of HPL_pdrpanllT.cpp / HPL_pdrpancrT.cpp).
  hplb_status rpanel(int r0, int c0, int N, int pc, int pw) {
    hplb_ctx*   ctx   = this->ctx;
    const int   nbmin = std::min(std::max(algo->nbmin, 1), kMaxLeaf);
    const int   ndiv  = std::max(algo->ndiv, 2);
    hplb_status s;
    if(N <= nbmin) return leaf(r0, c0, N, pc, pw);
    const int nbs = (((N + nbmin - 1) / nbmin + ndiv - 1) / ndiv) * nbmin;
    int       jj = 0, rem = N, jb = nbs;
    cudaStream_t st = ctx->s_pan;
    if(algo->rfact == 2) {
      do {
        rem -= jb;
        if((s = rpanel(r0 + jj, c0 + jj, jb, pc, pw)) != HPLB_OK) return s;
        if(rem > 0) {
          CK(launch_trsm_node(A, ld, r0 + jj, jb, c0 + jj, ctx->d_dinv_piece, c0 + jj + jb, rem,
                              st, &ctx->launches));
          CK(launch_dgemm_sub(n - (r0 + jj + jb), rem, jb, a(r0 + jj + jb, c0 + jj), ld,
                              a(r0 + jj, c0 + jj + jb), ld, a(r0 + jj + jb, c0 + jj + jb), ld,
                              ctx->d_status, st));
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
          CK(launch_trsm_node(A, ld, r0, jj, c0, ctx->d_dinv_piece, cj, jb, st, &ctx->launches));
          CK(launch_dgemm_sub(n - (r0 + jj), jb, jj, a(r0 + jj, c0), ld, a(r0, cj), ld,
                              a(r0 + jj, cj), ld, ctx->d_status, st));
          ctx->launches += 1;
        }
        if((s = rpanel(r0 + jj, cj, jb, pc, pw)) != HPLB_OK) return s;
        jj += jb;
        jb = std::min(rem, nbs);
      } while(rem > 0);
    }
    return HPLB_OK;
  }

  // Factor panel j on the panel stream and build its row map and diagonal
  // inverses; records `done` when finished.
  hplb_status panel(int j, int set, cudaEvent_t done) {
    hplb_ctx*   ctx = this->ctx;
    const int   jb  = std::min(algo->nb, n - j);
    cudaEvent_t e0  = next_event(ctx), e1 = next_event(ctx);
    CK(cudaEventRecord(e0, ctx->s_pan));
    hplb_status s = rpanel(j, j, jb, j, jb);
    if(s != HPLB_OK) return s;
    CK(launch_perm(ctx->d_ipiv + j, j, jb, ctx->d_perm[set], ctx->s_pan));
    CK(launch_diag_inv(A, ld, j, j, jb, ctx->d_dinv[set], ctx->s_pan));
    ctx->launches += 2;
    CK(launch_unit_lower_inverse(a(j, j), ld, jb, ctx->d_dinv[set], ctx->d_linv[set], jb,
                                 ctx->s_pan));
    ctx->launches += 2;
    CK(cudaEventRecord(e1, ctx->s_pan));
    CK(cudaEventRecord(done, ctx->s_pan));
    panel_ev.emplace_back(e0, e1);
    return HPLB_OK;
  }

  // Row interchanges + U12 + trailing DGEMM of panel j on columns [c, c+w).
  // max_ctas > 0 caps the grids of the update's DGEMMs (SMs left to the panel).
  hplb_status update(int j, int set, int c, int w, int max_ctas = 0) {
    hplb_ctx* ctx = this->ctx;
    if(w <= 0) return HPLB_OK;
    const int jb = std::min(algo->nb, n - j);
    // Interchanges into W, then U12 = L11^-1 W straight into the top rows
    // (rocHPL: HPL_dlaswp00N + rocblas_dtrsm, src/pgesv/HPL_pdupdateTT.cpp:95-106).
    CK(launch_laswp_gather(A, ld, j, jb, ctx->d_perm[set], ctx->d_w, jb, c, w, ctx->s_upd));
    CK(launch_dgemm_set(jb, w, jb, ctx->d_linv[set], jb, ctx->d_w, jb, a(j, c), ld,
                        ctx->d_status, ctx->s_upd));
    ctx->launches += 2;
    const int m = n - (j + jb);
    if(m > 0) {
      cudaEvent_t e0 = next_event(ctx), e1 = next_event(ctx);
      CK(cudaEventRecord(e0, ctx->s_upd));
      CK(launch_dgemm_sub(m, w, jb, a(j + jb, j), ld, a(j, c), ld, a(j + jb, c), ld,
                          ctx->d_status, ctx->s_upd, max_ctas));
      CK(cudaEventRecord(e1, ctx->s_upd));
      ctx->launches += 1;
      gemm_ev.emplace_back(e0, e1);
      gemm_flops.push_back(2.0 * m * (double)w * jb);
    }
    return HPLB_OK;
  }
};

}  // namespace

extern "C" {

const char* hplb_status_string(hplb_status s) {
  switch(s) {
    case HPLB_OK: return "ok";
    case HPLB_ERR_ARG: return "invalid argument";
    case HPLB_ERR_OOM: return "out of device memory";
    case HPLB_ERR_SINGULAR: return "matrix is singular (zero pivot)";
    case HPLB_ERR_TIMEOUT: return "device wait timed out";
    case HPLB_ERR_CUDA: return "CUDA error";
    case HPLB_ERR_UNSUPPORTED: return "unsupported parameter";
  }
  return "unknown status";
}

const char* hplb_last_error(const hplb_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

hplb_status hplb_set_option(hplb_ctx* ctx, int option, int value) {
  if(!ctx) return HPLB_ERR_ARG;
  switch(option) {
    case HPLB_OPT_LEAF:
      if(value < HPLB_LEAF_AUTO || value > HPLB_LEAF_REGISTERS)
        return set_err(ctx, HPLB_ERR_ARG, "hplb_set_option: leaf kind %d out of range", value);
      ctx->leaf_kind = value;
      return HPLB_OK;
    case HPLB_OPT_PANEL_SMS:
      if(value < HPLB_PANEL_SMS_AUTO || value >= ctx->num_sms)
        return set_err(ctx, HPLB_ERR_ARG, "hplb_set_option: panel SMs %d out of range [-1, %d)",
                       value, ctx->num_sms);
      ctx->panel_sms = value;
      return HPLB_OK;
  }
  return set_err(ctx, HPLB_ERR_ARG, "hplb_set_option: unknown option %d", option);
}

hplb_status hplb_set_stream(hplb_ctx* ctx, void* stream) {
  if(!ctx) return HPLB_ERR_ARG;
  ctx->caller = static_cast<cudaStream_t>(stream);
  return HPLB_OK;
}

int64_t hplb_default_ld(int n) { return ((int64_t)std::max(1, n) + 95) / 128 * 128 + 32; }

hplb_ctx* hplb_create(int device, hplb_status* status) {
  auto fail = [&](hplb_status s) -> hplb_ctx* {
    if(status) *status = s;
    return nullptr;
  };
  int ndev = 0;
  if(cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return fail(ndev == 0 ? HPLB_ERR_CUDA : HPLB_ERR_ARG);
  }
  // Some kernels' shared-memory limits are raised once per process, on the
  // device current at the time: every context of a process is on one device.
  static std::atomic<int> process_device{-1};
  int first = -1;
  if(!process_device.compare_exchange_strong(first, device) && first != device) {
    std::fprintf(stderr, "hplb_create: device %d, but this process already uses device %d "
                         "(one process drives one GPU)\n", device, first);
    return fail(HPLB_ERR_UNSUPPORTED);
  }
  if(cudaSetDevice(device) != cudaSuccess) return fail(HPLB_ERR_CUDA);
  hplb_ctx* ctx = new hplb_ctx();
  ctx->device   = device;
  cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  int lo = 0, hi = 0;
  cudaDeviceGetStreamPriorityRange(&lo, &hi);
  bool ok = cudaStreamCreateWithPriority(&ctx->s_upd, cudaStreamNonBlocking, lo) == cudaSuccess &&
            cudaStreamCreateWithPriority(&ctx->s_pan, cudaStreamNonBlocking, hi) == cudaSuccess &&
            cudaEventCreateWithFlags(&ctx->ev_enter, cudaEventDisableTiming) == cudaSuccess &&
            cudaMalloc(&ctx->d_status, ST_COUNT * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&ctx->d_bar, 2 * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&ctx->d_out8, 8 * sizeof(double)) == cudaSuccess;
  if(!ok) {
    cudaGetLastError();
    hplb_destroy(ctx);
    return fail(HPLB_ERR_CUDA);
  }
  cudaMemset(ctx->d_status, 0, ST_COUNT * sizeof(int));
  cudaMemset(ctx->d_bar, 0, 2 * sizeof(int));
  if(status) *status = HPLB_OK;
  return ctx;
}

void hplb_destroy(hplb_ctx* ctx) {
  if(!ctx) return;
  cudaSetDevice(ctx->device);
  if(ctx->s_upd) cudaStreamSynchronize(ctx->s_upd);
  if(ctx->s_pan) cudaStreamSynchronize(ctx->s_pan);
  for(auto e : ctx->events) cudaEventDestroy(e);
  if(ctx->ev_enter) cudaEventDestroy(ctx->ev_enter);
  void* bufs[] = {ctx->d_status, ctx->d_bar,      ctx->d_out8,        ctx->d_ipiv,
                  ctx->d_perm[0], ctx->d_perm[1], ctx->d_dinv[0],     ctx->d_dinv[1],
                  ctx->d_dinv_piece, ctx->d_cand, ctx->d_res, ctx->d_linv[0], ctx->d_linv[1],
                  ctx->d_w,       ctx->m_w,       ctx->m_linv,        ctx->m_uinv,
                  ctx->m_perm,    ctx->m_g,       ctx->m_l16,         ctx->m_u16,
                  ctx->m_scale,   ctx->m_small,   ctx->m_vec,         ctx->r_t,
                  ctx->r_ws,      ctx->r_perm,    ctx->m_li16,        ctx->d_trsv};
  for(void* b : bufs)
    if(b) cudaFree(b);
  if(ctx->s_upd) cudaStreamDestroy(ctx->s_upd);
  if(ctx->s_pan) cudaStreamDestroy(ctx->s_pan);
  delete ctx;
}

hplb_status hplb_matgen(hplb_ctx* ctx, int m, int n, int nb, uint64_t seed, double* dA,
                        int64_t ld) {
  if(!ctx) return HPLB_ERR_ARG;
  (void)nb;
  if(m < 0 || n < 0) return set_err(ctx, HPLB_ERR_ARG, "hplb_matgen: negative size");
  if(ld < std::max(1, m)) return set_err(ctx, HPLB_ERR_ARG, "hplb_matgen: ld < max(1,m)");
  if(m > 0 && n > 0 && !dA) return set_err(ctx, HPLB_ERR_ARG, "hplb_matgen: null matrix");
  ENTER(ctx);
  CK(launch_matgen(m, n, seed, dA, ld, ctx->s_upd));
  CK(cudaStreamSynchronize(ctx->s_upd));
  return HPLB_OK;
}

hplb_status hplb_matgen_block(hplb_ctx* ctx, int64_t mg, int64_t ng, int64_t i0, int64_t j0,
                              int m, int n, uint64_t seed, double* dA, int64_t ld) {
  if(!ctx) return HPLB_ERR_ARG;
  if(m < 0 || n < 0 || mg < 0 || ng < 0 || i0 < 0 || j0 < 0 || i0 + m > mg || j0 + n > ng)
    return set_err(ctx, HPLB_ERR_ARG, "hplb_matgen_block: block outside the %lld x %lld matrix",
                   (long long)mg, (long long)ng);
  if(ld < std::max(1, m)) return set_err(ctx, HPLB_ERR_ARG, "hplb_matgen_block: ld < max(1,m)");
  if(m > 0 && n > 0 && !dA) return set_err(ctx, HPLB_ERR_ARG, "hplb_matgen_block: null matrix");
  ENTER(ctx);
  CK(launch_matgen_block(mg, i0, j0, m, n, seed, dA, ld, ctx->s_upd));
  CK(cudaStreamSynchronize(ctx->s_upd));
  return HPLB_OK;
}

}  // extern "C"

// Grid cap of the trailing-update DGEMM (m x w) of a step whose next panel
// is factored beside it (0: none), from HPLB_OPT_PANEL_SMS.  Automatic: 32 SMs
// stay with the panel once the update is at most 4 waves of 128 x 128 tiles
// (the steps where the panel, not the update, is the longer of the two).
static int update_cap(const hplb_ctx* ctx, int m, int w) {
  int keep = ctx->panel_sms;
  if(keep == HPLB_PANEL_SMS_AUTO) {
    const long long tiles = (long long)((m + 127) / 128) * ((w + 127) / 128);
    keep = tiles <= 4LL * ctx->num_sms ? 32 : 0;
  }
  return keep > 0 ? std::max(1, ctx->num_sms - keep) : 0;
}

// The factorisation loop shared by hplb_pdgesv (nrhs = 1: column n of A is b,
// carried through the updates, then the back-solve into dX), hplb_gesv
// (columns n .. n + nrhs - 1 are B, then the multi-RHS back-solve into dX,
// leading dimension ldx) and hplb_getrf (nrhs = 0: A alone, no back-solve).
static hplb_status factor_driver(hplb_ctx* ctx, const hplb_algo* algo, int n, double* dA,
                                 int64_t ld, double* dX, int64_t ldx, int* ipiv_out, int* info,
                                 int nrhs) {
  const bool rhs = nrhs > 0;
  if(!ctx) return HPLB_ERR_ARG;
  hplb_status s = check_algo(ctx, algo, n, ld, true);
  if(s != HPLB_OK) return s;
  if(info) *info = 0;
  ctx->timing = hplb_timing{};
  ctx->step_col.clear();
  ctx->step_ms.clear();
  if(n == 0) return HPLB_OK;
  if(!dA || (rhs && !dX)) return set_err(ctx, HPLB_ERR_ARG, "null matrix or solution");
  ENTER(ctx);
  s = ensure_solve_ws(ctx, n, algo->nb, algo->nbmin, nrhs);
  if(s != HPLB_OK) return s;

  ctx->ev_next  = 0;
  ctx->launches = 0;
  CK(cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->s_upd));
  Solve S{ctx, algo, dA, ld, n, {}, {}, {}};
  cudaEvent_t ev_start = next_event(ctx), ev_lu = next_event(ctx), ev_end = next_event(ctx);
  cudaEvent_t ev_panel[2] = {next_event(ctx), next_event(ctx)};
  CK(cudaEventRecord(ev_start, ctx->s_upd));
  CK(cudaStreamWaitEvent(ctx->s_pan, ev_start, 0));

  const int nb = algo->nb;
  std::vector<cudaEvent_t> step_end;
  step_end.reserve((size_t)(n + nb - 1) / nb);
  if((s = S.panel(0, 0, ev_panel[0])) != HPLB_OK) return s;
  for(int j = 0; j < n; j += nb) {
    const int set = (j / nb) & 1;
    const int jb  = std::min(nb, n - j);
    CK(cudaStreamWaitEvent(ctx->s_upd, ev_panel[set], 0));
    const int c1 = j + jb;                              // first trailing column
    const int la = c1 < n ? std::min(nb, n - c1) : 0;   // look-ahead width
    if((s = S.update(j, set, c1, la)) != HPLB_OK) return s;
    if(la > 0) {
      cudaEvent_t ev_la = next_event(ctx);
      CK(cudaEventRecord(ev_la, ctx->s_upd));
      CK(cudaStreamWaitEvent(ctx->s_pan, ev_la, 0));
      if((s = S.panel(c1, set ^ 1, ev_panel[set ^ 1])) != HPLB_OK) return s;
    }
    const int cap = la > 0 ? update_cap(ctx, n - c1, n + nrhs - (c1 + la)) : 0;
    if((s = S.update(j, set, c1 + la, n + nrhs - (c1 + la), cap)) != HPLB_OK) return s;
    // Step j ends when its trailing update is done (the update stream has
    // already waited for panel j); the progress report reads these.
    step_end.push_back(next_event(ctx));
    CK(cudaEventRecord(step_end.back(), ctx->s_upd));
    ctx->step_col.push_back(j);
  }
  CK(cudaEventRecord(ev_lu, ctx->s_upd));
  if(nrhs == 1)
    CK(launch_trsv(dA, ld, n, dX, ctx->d_trsv, ctx->d_status, ctx->s_upd, &ctx->launches));
  else if(nrhs > 1)
    CK(launch_trsm_upper(dA, ld, n, nrhs, dA + (size_t)n * (size_t)ld, ld, dX, ldx, ctx->d_trsv,
                         ctx->d_status, ctx->s_upd, &ctx->launches));
  if(ipiv_out)
    CK(cudaMemcpyAsync(ipiv_out, ctx->d_ipiv, (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice,
                       ctx->s_upd));
  CK(cudaEventRecord(ev_end, ctx->s_upd));
  {
    cudaError_t e = cudaStreamSynchronize(ctx->s_upd);
    if(e == cudaSuccess) e = cudaStreamSynchronize(ctx->s_pan);
    if(e != cudaSuccess)
      return set_err(ctx, HPLB_ERR_CUDA, "solve failed: %s", cudaGetErrorString(e));
  }
  int inf = 0;
  s       = read_status(ctx, &inf);
  if(info) *info = inf;

  hplb_timing& T = ctx->timing;
  float        ms = 0.f;
  cudaEventElapsedTime(&ms, ev_start, ev_end);
  T.total_ms = ms;
  cudaEventElapsedTime(&ms, ev_start, ev_lu);
  T.lu_ms = ms;
  cudaEventElapsedTime(&ms, ev_lu, ev_end);
  T.trsv_ms = ms;
  for(size_t i = 0; i < S.gemm_ev.size(); ++i) {
    cudaEventElapsedTime(&ms, S.gemm_ev[i].first, S.gemm_ev[i].second);
    T.gemm_ms += ms;
    T.gemm_flops += S.gemm_flops[i];
  }
  for(auto& p : S.panel_ev) {
    cudaEventElapsedTime(&ms, p.first, p.second);
    T.panel_ms += ms;
  }
  for(size_t i = 0; i < step_end.size(); ++i) {
    cudaEventElapsedTime(&ms, i ? step_end[i - 1] : ev_start, step_end[i]);
    ctx->step_ms.push_back(ms);
  }
  T.gemm_launches   = (int)S.gemm_ev.size();
  T.kernel_launches = ctx->launches;
  if(s != HPLB_OK) return s;
  if(inf != 0) return set_err(ctx, HPLB_ERR_SINGULAR, "zero pivot in column %d", inf);
  return HPLB_OK;
}

extern "C" {

hplb_status hplb_pdgesv(hplb_ctx* ctx, const hplb_algo* algo, int n, double* dA, int64_t ld,
                        double* dX, int* ipiv_out, int* info) {
  return factor_driver(ctx, algo, n, dA, ld, dX, n, ipiv_out, info, 1);
}

hplb_status hplb_gesv(hplb_ctx* ctx, const hplb_algo* algo, int n, int nrhs, double* dA,
                      int64_t ld, double* dX, int64_t ldx, int* ipiv_out, int* info) {
  if(!ctx) return HPLB_ERR_ARG;
  if(nrhs < 1) return set_err(ctx, HPLB_ERR_ARG, "hplb_gesv: nrhs must be >= 1");
  if(n > 0 && ldx < n) return set_err(ctx, HPLB_ERR_ARG, "hplb_gesv: ldx < n");
  return factor_driver(ctx, algo, n, dA, ld, dX, ldx, ipiv_out, info, nrhs);
}

hplb_status hplb_getrf(hplb_ctx* ctx, const hplb_algo* algo, int n, double* dA, int64_t ld,
                       int* ipiv_out, int* info) {
  return factor_driver(ctx, algo, n, dA, ld, nullptr, 0, ipiv_out, info, 0);
}

static hplb_status residual_common(hplb_ctx* ctx, int n, const double* dA, int64_t ld, bool lcg,
                                   uint64_t seed, const double* dX, hplb_resid* out) {
  if(!ctx) return HPLB_ERR_ARG;
  if(n < 0 || !out) return set_err(ctx, HPLB_ERR_ARG, "hplb_residual: bad argument");
  if(!lcg && n > 0 && (!dA || ld < n)) return set_err(ctx, HPLB_ERR_ARG, "hplb_residual: bad matrix");
  if(n > 0 && !dX) return set_err(ctx, HPLB_ERR_ARG, "hplb_residual: null solution");
  ENTER(ctx);
  hplb_status s = grow(ctx, &ctx->d_res, &ctx->res_cap, residual_ws_doubles(std::max(n, 1)));
  if(s != HPLB_OK) return s;
  CK(launch_residual(n, dA, ld, lcg, seed, dX, ctx->d_res, ctx->d_out8, ctx->s_upd));
  double o[8];
  CK(cudaMemcpyAsync(o, ctx->d_out8, sizeof o, cudaMemcpyDeviceToHost, ctx->s_upd));
  CK(cudaStreamSynchronize(ctx->s_upd));
  out->resid     = o[0];
  out->rnorm_inf = o[1];
  out->anorm_1   = o[2];
  out->anorm_inf = o[3];
  out->xnorm_1   = o[4];
  out->xnorm_inf = o[5];
  out->bnorm_inf = o[6];
  out->eps       = o[7];
  return HPLB_OK;
}

hplb_status hplb_residual(hplb_ctx* ctx, int n, const double* dA, int64_t ld, const double* dX,
                          hplb_resid* out) {
  return residual_common(ctx, n, dA, ld, false, 0, dX, out);
}

hplb_status hplb_residual_lcg(hplb_ctx* ctx, int n, uint64_t seed, const double* dX,
                              hplb_resid* out) {
  return residual_common(ctx, n, nullptr, 0, true, seed, dX, out);
}

// ---------------------------------------------------------------------------
// Building blocks of the solve on a 1 x Q process grid (one process per GPU,
// block-cyclic columns; the driver is rochpl_b200/grid.py).
// ---------------------------------------------------------------------------

hplb_status hplb_panel_factor(hplb_ctx* ctx, const hplb_algo* algo, int n, int j, int jb,
                              double* dA, int64_t ld, int lc, int* d_ipiv, int* info) {
  if(!ctx) return HPLB_ERR_ARG;
  hplb_status s = check_algo(ctx, algo, n, ld, true);
  if(s != HPLB_OK) return s;
  if(j < 0 || jb < 1 || jb > 2048 || j + jb > n || lc < 0 || !dA || !d_ipiv)
    return set_err(ctx, HPLB_ERR_ARG, "hplb_panel_factor: bad panel (j %d, jb %d, lc %d, n %d)",
                   j, jb, lc, n);
  if(info) *info = 0;
  ENTER(ctx);
  if((s = ensure_solve_ws(ctx, n, std::max(algo->nb, jb), algo->nbmin)) != HPLB_OK) return s;
  if((s = grow(ctx, &ctx->d_ipiv, &ctx->ipiv_cap, (size_t)std::max(n, lc + jb))) != HPLB_OK)
    return s;
  ctx->ev_next  = 0;
  ctx->launches = 0;
  CK(cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->s_pan));
  Solve S{ctx, algo, dA, ld, n, {}, {}, {}};
  if((s = S.rpanel(j, lc, jb, lc, jb)) != HPLB_OK) return s;
  CK(cudaMemcpyAsync(d_ipiv, ctx->d_ipiv + lc, (size_t)jb * sizeof(int),
                     cudaMemcpyDeviceToDevice, ctx->s_pan));
  CK(cudaStreamSynchronize(ctx->s_pan));
  int inf = 0;
  if((s = read_status(ctx, &inf)) != HPLB_OK) return s;
  if(inf != 0) {
    const int col = j + (inf - 1 - lc) + 1;  // the leaf records local columns
    if(info) *info = col;
    return set_err(ctx, HPLB_ERR_SINGULAR, "zero pivot in column %d", col);
  }
  return HPLB_OK;
}

hplb_status hplb_panel_update(hplb_ctx* ctx, int n, int j, int jb, const double* dL,
                              int64_t ldl, const int* d_ipiv, double* dA, int64_t ld, int c0,
                              int ncols) {
  if(!ctx) return HPLB_ERR_ARG;
  if(n < 1 || j < 0 || jb < 1 || jb > 2048 || j + jb > n || ldl < n - j || ld < n || c0 < 0 ||
     ncols < 0 || ncols > n + 1 || !dL || !d_ipiv || (ncols > 0 && !dA))
    return set_err(ctx, HPLB_ERR_ARG, "hplb_panel_update: bad argument");
  if(ncols == 0) return HPLB_OK;
  ENTER(ctx);
  hplb_status s = ensure_solve_ws(ctx, n, jb, 1);
  if(s != HPLB_OK) return s;
  cudaStream_t st = ctx->s_upd;
  // Pivots index rows: check them before any kernel uses them.
  CK(cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), st));
  CK(launch_check_ipiv_range(jb, j, n, d_ipiv, ctx->d_status, st));
  CK(cudaStreamSynchronize(st));
  int bad = 0;
  if((s = read_status(ctx, &bad)) != HPLB_OK) return s;
  if(bad) return set_err(ctx, HPLB_ERR_ARG, "hplb_panel_update: ipiv[%d] outside [%d, n)", bad - 1,
                         j + bad - 1);
  double* top = dA + (size_t)j + (size_t)c0 * (size_t)ld;
  CK(launch_perm(d_ipiv, j, jb, ctx->d_perm[0], st));
  CK(launch_diag_inv(dL, ldl, 0, 0, jb, ctx->d_dinv[0], st));
  CK(launch_unit_lower_inverse(dL, ldl, jb, ctx->d_dinv[0], ctx->d_linv[0], jb, st));
  CK(launch_laswp_gather(dA, ld, j, jb, ctx->d_perm[0], ctx->d_w, jb, c0, ncols, st));
  CK(launch_dgemm_set(jb, ncols, jb, ctx->d_linv[0], jb, ctx->d_w, jb, top, ld, ctx->d_status,
                      st));
  if(n - j - jb > 0)
    CK(launch_dgemm_sub(n - j - jb, ncols, jb, dL + jb, ldl, top, ld, top + jb, ld,
                        ctx->d_status, st));
  CK(cudaStreamSynchronize(st));
  return read_status(ctx, nullptr);
}

hplb_status hplb_trsv_block(hplb_ctx* ctx, int n, int j, int jb, const double* dA, int64_t ld,
                            int lc, const double* dy, const double* ds, double* dx, double* dz) {
  if(!ctx) return HPLB_ERR_ARG;
  if(n < 1 || j < 0 || jb < 1 || j + jb > n || lc < 0 || ld < n || !dA || !dy || !ds || !dx ||
     !dz)
    return set_err(ctx, HPLB_ERR_ARG, "hplb_trsv_block: bad argument");
  ENTER(ctx);
  hplb_status s;
  if((s = grow(ctx, &ctx->d_trsv, &ctx->trsv_cap, trsv_flag_ints(jb))) != HPLB_OK ||
     (s = grow(ctx, &ctx->d_w, &ctx->w_cap, (size_t)jb)) != HPLB_OK)
    return s;
  cudaStream_t  st = ctx->s_upd;
  const double* U  = dA + (size_t)lc * (size_t)ld;  // this block's columns, all rows
  CK(cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), st));
  CK(launch_vsub(jb, dy + j, ds, ctx->d_w, st));
  int launches = 0;
  CK(launch_trsv_y(U + j, ld, jb, ctx->d_w, dx + j, ctx->d_trsv, ctx->d_status, st, &launches));
  CK(launch_gemv_acc(j, jb, U, ld, dx + j, dz, st));
  CK(cudaStreamSynchronize(st));
  return read_status(ctx, nullptr);
}

hplb_status hplb_col_argmax(hplb_ctx* ctx, const double* dA, int64_t ld, int r0, int r1, int col,
                            double* v_out, int* row_out) {
  if(!ctx) return HPLB_ERR_ARG;
  if(!v_out || !row_out || r0 < 0 || r1 < r0 || col < 0 || (r1 > r0 && (!dA || ld < r1)))
    return set_err(ctx, HPLB_ERR_ARG, "hplb_col_argmax: bad argument");
  *v_out   = 0.0;
  *row_out = -1;
  if(r1 == r0) return HPLB_OK;
  ENTER(ctx);
  CK(launch_col_argmax(dA, ld, r0, r1, col, ctx->d_out8, ctx->s_upd));
  double o[2];
  CK(cudaMemcpyAsync(o, ctx->d_out8, sizeof o, cudaMemcpyDeviceToHost, ctx->s_upd));
  CK(cudaStreamSynchronize(ctx->s_upd));
  *v_out   = o[0];
  *row_out = (int)o[1];
  return HPLB_OK;
}

hplb_status hplb_col_rank1(hplb_ctx* ctx, double* dA, int64_t ld, int r0, int r1, int c0, int k,
                           int kend, double piv, const double* du) {
  if(!ctx) return HPLB_ERR_ARG;
  if(r0 < 0 || r1 < r0 || c0 < 0 || k < 0 || kend <= k ||
     (r1 > r0 && (!dA || !du || ld < r1)))
    return set_err(ctx, HPLB_ERR_ARG, "hplb_col_rank1: bad argument");
  if(r1 == r0) return HPLB_OK;
  ENTER(ctx);
  CK(launch_col_rank1(dA, ld, r0, r1, c0, k, kend, piv, du, ctx->num_sms, ctx->s_upd));
  CK(cudaStreamSynchronize(ctx->s_upd));
  return HPLB_OK;
}

hplb_status hplb_trsm_lower_unit(hplb_ctx* ctx, int n, int nrhs, const double* dL, int64_t ldl,
                                 double* dX, int64_t ldx) {
  if(!ctx) return HPLB_ERR_ARG;
  if(n < 0 || nrhs < 0 || (n > 0 && nrhs > 0 && (!dL || !dX || ldl < n || ldx < n)))
    return set_err(ctx, HPLB_ERR_ARG, "hplb_trsm_lower_unit: bad argument");
  if(n > HPLB_TRSM_LOWER_MAX_N)
    return set_err(ctx, HPLB_ERR_ARG, "hplb_trsm_lower_unit: n above HPLB_TRSM_LOWER_MAX_N");
  if(n == 0 || nrhs == 0) return HPLB_OK;
  ENTER(ctx);
  hplb_status s = ensure_solve_ws(ctx, 1, n, 1);
  if(s != HPLB_OK) return s;
  CK(launch_diag_inv<double>(dL, ldl, 0, 0, n, ctx->d_dinv_piece, ctx->s_upd));
  CK(launch_trsm_unit_lower(dX, ldx, n, dL, ldl, ctx->d_dinv_piece, nrhs, ctx->s_upd));
  CK(cudaStreamSynchronize(ctx->s_upd));
  return HPLB_OK;
}

hplb_status hplb_trsm_upper(hplb_ctx* ctx, int n, int nrhs, const double* dU, int64_t ldu,
                            const double* dY, int64_t ldy, double* dX, int64_t ldx) {
  if(!ctx) return HPLB_ERR_ARG;
  if(n < 0 || nrhs < 0 ||
     (n > 0 && nrhs > 0 && (!dU || !dY || !dX || ldu < n || ldy < n || ldx < n)))
    return set_err(ctx, HPLB_ERR_ARG, "hplb_trsm_upper: bad argument");
  if(n == 0 || nrhs == 0) return HPLB_OK;
  ENTER(ctx);
  hplb_status s = grow(ctx, &ctx->d_trsv, &ctx->trsv_cap, trsv_flag_ints(n));
  if(s != HPLB_OK) return s;
  CK(cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->s_upd));
  int launches = 0;
  CK(launch_trsm_upper(dU, ldu, n, nrhs, dY, ldy, dX, ldx, ctx->d_trsv, ctx->d_status,
                       ctx->s_upd, &launches));
  CK(cudaStreamSynchronize(ctx->s_upd));
  return read_status(ctx, nullptr);
}

hplb_status hplb_last_timing(const hplb_ctx* ctx, hplb_timing* out) {
  if(!ctx || !out) return HPLB_ERR_ARG;
  *out = ctx->timing;
  return HPLB_OK;
}

hplb_status hplb_last_steps(const hplb_ctx* ctx, int cap, int* count, int* col, double* ms) {
  if(!ctx || !count || cap < 0 || (cap > 0 && (!col || !ms))) return HPLB_ERR_ARG;
  const int n = (int)ctx->step_ms.size();
  *count      = n;
  for(int i = 0; i < n && i < cap; ++i) {
    col[i] = ctx->step_col[i];
    ms[i]  = ctx->step_ms[i];
  }
  return HPLB_OK;
}

hplb_status hplb_dgemm_sub(hplb_ctx* ctx, int m, int n, int k, const double* dA, int64_t lda,
                           const double* dB, int64_t ldb, double* dC, int64_t ldc) {
  if(!ctx) return HPLB_ERR_ARG;
  if(m < 0 || n < 0 || k < 0) return set_err(ctx, HPLB_ERR_ARG, "hplb_dgemm_sub: negative size");
  if(lda < std::max(1, m) || ldb < std::max(1, k) || ldc < std::max(1, m))
    return set_err(ctx, HPLB_ERR_ARG, "hplb_dgemm_sub: leading dimension too small");
  ENTER(ctx);
  CK(cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->s_upd));
  CK(launch_dgemm_sub(m, n, k, dA, lda, dB, ldb, dC, ldc, ctx->d_status, ctx->s_upd));
  CK(cudaStreamSynchronize(ctx->s_upd));
  return read_status(ctx, nullptr);
}

hplb_status hplb_laswp_trsm(hplb_ctx* ctx, double* dA, int64_t ld, int ia, int jb, int lc,
                            const int* ipiv_host, int c0, int n) {
  if(!ctx) return HPLB_ERR_ARG;
  if(jb < 0 || jb > 2048 || n < 0 || ia < 0 || lc < 0 || c0 < 0)
    return set_err(ctx, HPLB_ERR_ARG, "hplb_laswp_trsm: bad argument");
  if(jb == 0 || n == 0) return HPLB_OK;
  ENTER(ctx);
  hplb_status s = ensure_solve_ws(ctx, ia + jb, std::max(jb, 1), 1);
  if(s != HPLB_OK) return s;
  const int* perm = nullptr;
  if(ipiv_host) {
    for(int i = 0; i < jb; ++i)
      if(ipiv_host[i] < ia + i || ipiv_host[i] >= ld)
        return set_err(ctx, HPLB_ERR_ARG, "hplb_laswp_trsm: ipiv[%d] = %d out of range", i,
                       ipiv_host[i]);
    CK(cudaMemcpyAsync(ctx->d_ipiv, ipiv_host, (size_t)jb * sizeof(int), cudaMemcpyHostToDevice,
                       ctx->s_upd));
    CK(launch_perm(ctx->d_ipiv, ia, jb, ctx->d_perm[0], ctx->s_upd));
    perm = ctx->d_perm[0];
  }
  CK(launch_diag_inv(dA, ld, ia, lc, jb, ctx->d_dinv[0], ctx->s_upd));
  CK(launch_laswp_trsm(dA, ld, ia, jb, lc, perm, ctx->d_dinv[0], c0, n, ctx->s_upd));
  CK(cudaStreamSynchronize(ctx->s_upd));
  return HPLB_OK;
}

hplb_status hplb_gemm_lp_sub(hplb_ctx* ctx, int bf16, int m, int n, int k, const void* dA16,
                             int64_t lda, const void* dB16, int64_t ldb, const float* dsA,
                             const float* dsB, float* dC, int64_t ldc) {
  if(!ctx) return HPLB_ERR_ARG;
  if(m < 0 || n < 0 || k < 0 || lda < std::max(1, k) || ldb < std::max(1, k) ||
     ldc < std::max(1, m) || lda % 8 || ldb % 8)
    return set_err(ctx, HPLB_ERR_ARG, "hplb_gemm_lp_sub: bad sizes or leading dimensions");
  ENTER(ctx);
  CK(cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->s_upd));
  CK(launch_gemm_lp(bf16 != 0, m, n, k, dA16, lda, dB16, ldb, dsA, dsB, dC, ldc, ctx->d_status,
                    ctx->s_upd));
  CK(cudaStreamSynchronize(ctx->s_upd));
  return read_status(ctx, nullptr);
}

hplb_status hplb_fp64_peak(hplb_ctx* ctx, int iters, double* dmma_tflops, double* dfma_tflops) {
  if(!ctx || iters < 1 || !dmma_tflops || !dfma_tflops) return HPLB_ERR_ARG;
  ENTER(ctx);
  CK(fp64_peak(ctx->num_sms, iters, dmma_tflops, dfma_tflops, ctx->s_upd));
  return HPLB_OK;
}

hplb_status hplb_selftest_wait_timeout(hplb_ctx* ctx, uint64_t budget_ns) {
  if(!ctx) return HPLB_ERR_ARG;
  if(budget_ns > 10000000000ull)
    return set_err(ctx, HPLB_ERR_ARG, "hplb_selftest_wait_timeout: budget above 10 s");
  ENTER(ctx);
  CK(cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->s_upd));
  // d_bar[0] is the flag: zeroed and never set.
  CK(cudaMemsetAsync(ctx->d_bar, 0, 2 * sizeof(int), ctx->s_upd));
  CK(launch_wait_selftest(ctx->d_bar, ctx->d_status, budget_ns, ctx->s_upd));
  CK(cudaStreamSynchronize(ctx->s_upd));
  hplb_status s = read_status(ctx, nullptr);
  CK(cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->s_upd));
  CK(cudaStreamSynchronize(ctx->s_upd));
  return s;
}

}  // extern "C"
