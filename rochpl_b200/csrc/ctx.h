// Context object of libhplb200 and the helpers its drivers share (private).
#pragma once
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "common.cuh"
#include "internal.h"

struct hplb_ctx {
  int          device  = 0;
  int          num_sms = 0;
  cudaStream_t s_upd   = nullptr;
  cudaStream_t s_pan   = nullptr;
  std::string  err;
  hplb_timing  timing{};
  std::vector<int>    step_col;  // first column of each step of the last factorisation
  std::vector<double> step_ms;   // its time, previous step's end to this step's end (ms)

  int*    d_status = nullptr;  // ST_COUNT ints
  int*    d_bar    = nullptr;  // 2 ints
  double* d_out8   = nullptr;  // residual outputs

  int*    d_ipiv   = nullptr;
  size_t  ipiv_cap = 0;
  int*    d_perm[2] = {nullptr, nullptr};
  double* d_dinv[2] = {nullptr, nullptr};
  double* d_linv[2] = {nullptr, nullptr};  // L11^-1 per panel set (nb x nb)
  double* d_dinv_piece = nullptr;
  double* d_w          = nullptr;  // gathered top rows of the trailing columns (nb x (n+1))
  size_t  w_cap        = 0;        // doubles
  int     nb_cap       = 0;
  double* d_cand       = nullptr;
  double* d_cur        = nullptr;
  size_t  cand_cap     = 0;  // doubles
  int*    d_trsv       = nullptr;  // back-solve flags and ticket
  size_t  trsv_cap     = 0;        // ints
  double* d_res        = nullptr;
  size_t  res_cap      = 0;  // doubles

  // Mixed-precision workspaces (FP32 factors and their by-products).
  float*          m_w     = nullptr;  size_t m_w_cap     = 0;  // FP32 working matrix
  float*          m_linv  = nullptr;  size_t m_linv_cap  = 0;  // per-panel L11^-1
  float*          m_uinv  = nullptr;  size_t m_uinv_cap  = 0;  // per-panel U11^-1
  int*            m_perm  = nullptr;  size_t m_perm_cap  = 0;  // per-panel row maps
  float*          m_g     = nullptr;  size_t m_g_cap     = 0;  // gathered rows
  unsigned short* m_l16   = nullptr;  size_t m_l16_cap   = 0;  // packed L21
  unsigned short* m_u16   = nullptr;  size_t m_u16_cap   = 0;  // packed U12
  unsigned short* m_li16  = nullptr;  size_t m_li16_cap  = 0;  // packed -L11^-1
  float*          m_scale = nullptr;  size_t m_scale_cap = 0;  // tile scales
  float*          m_small = nullptr;  size_t m_small_cap = 0;  // inverses' scratch
  double*         m_vec   = nullptr;  size_t m_vec_cap   = 0;  // FP64 vectors

  // Multi-RHS solve workspaces (hplb_getrs).
  double* r_t    = nullptr;  size_t r_t_cap    = 0;  // transposed factors (trans = 1)
  double* r_ws   = nullptr;  size_t r_ws_cap   = 0;  // block copies and inverses
  int*    r_perm = nullptr;  size_t r_perm_cap = 0;  // one panel's row map

  int          leaf_kind = HPLB_LEAF_AUTO;  // hplb_set_option(HPLB_OPT_LEAF)
  int          panel_sms = HPLB_PANEL_SMS_AUTO;  // hplb_set_option(HPLB_OPT_PANEL_SMS)
  cudaStream_t caller   = nullptr;  // hplb_set_stream (null: the legacy default stream)
  cudaEvent_t  ev_enter = nullptr;  // recorded on `caller` at every entry

  std::vector<cudaEvent_t> events;  // pool
  size_t                   ev_next = 0;
  int                      launches = 0;
};

namespace hplb {

inline hplb_status set_err(hplb_ctx* c, hplb_status s, const char* fmt, ...) {
  char    buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if(c) c->err = buf;
  return s;
}

#define CK(expr)                                                                       \
  do {                                                                                 \
    cudaError_t e__ = (expr);                                                          \
    if(e__ != cudaSuccess)                                                             \
      return set_err(ctx, HPLB_ERR_CUDA, "%s failed: %s (%s:%d)", #expr,               \
                     cudaGetErrorString(e__), __FILE__, __LINE__);                     \
  } while(0)

template <class T>
inline hplb_status grow(hplb_ctx* ctx, T** p, size_t* cap, size_t need) {
  if(*cap >= need && *p) return HPLB_OK;
  if(*p) cudaFree(*p);
  *p   = nullptr;
  *cap = 0;
  if(cudaMalloc((void**)p, need * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return set_err(ctx, HPLB_ERR_OOM, "workspace allocation of %zu bytes failed",
                   need * sizeof(T));
  }
  *cap = need;
  return HPLB_OK;
}

// The HPL.dat checks of HPL_pdinfo (src/pauxil/HPL_pdinfo.cpp) that concern
// the solve, plus this library's own limits.
inline hplb_status check_algo(hplb_ctx* ctx, const hplb_algo* algo, int n, int64_t ld,
                              bool need_ld) {
  if(!algo) return set_err(ctx, HPLB_ERR_ARG, "null algo");
  if(n < 0) return set_err(ctx, HPLB_ERR_ARG, "Value of N less than 0");
  if(algo->nb < 1) return set_err(ctx, HPLB_ERR_ARG, "Value of NB less than 1");
  if(algo->nbmin < 1) return set_err(ctx, HPLB_ERR_ARG, "Value of NBMIN less than 1");
  if(algo->ndiv < 2) return set_err(ctx, HPLB_ERR_ARG, "Value of NDIV less than 2");
  if(algo->pfact < 0 || algo->pfact > 2)
    return set_err(ctx, HPLB_ERR_ARG, "Value of PFACT out of range");
  if(algo->rfact < 0 || algo->rfact > 2)
    return set_err(ctx, HPLB_ERR_ARG, "Value of RFACT out of range");
  if(algo->depth != 1)
    return set_err(ctx, HPLB_ERR_UNSUPPORTED, "Only lookahead depth 1 is supported");
  if(algo->nbmin > kMaxLeaf)
    return set_err(ctx, HPLB_ERR_UNSUPPORTED, "NBMIN above %d is not supported", kMaxLeaf);
  if(algo->nb > 2048) return set_err(ctx, HPLB_ERR_UNSUPPORTED, "NB above 2048 is not supported");
  if(need_ld && ld < (n > 1 ? n : 1)) return set_err(ctx, HPLB_ERR_ARG, "ld < max(1,N)");
  return HPLB_OK;
}

// Pivot vector and the leaf kernel's candidate / current-row scratch.
inline hplb_status ensure_leaf_ws(hplb_ctx* ctx, int n, int nbmin) {
  hplb_status s;
  if((s = grow(ctx, &ctx->d_ipiv, &ctx->ipiv_cap, (size_t)(n > 1 ? n : 1))) != HPLB_OK) return s;
  const int    gmax = leaf_grid_size(ctx->num_sms, n > 1 ? n : 1);
  // Slots of 2 + w doubles, rounded up to an even count so that the register
  // leaf's 16-byte (value, row) accesses stay aligned.
  const size_t cand = 2 * (size_t)gmax * (size_t)((3 + (nbmin < kMaxLeaf ? nbmin : kMaxLeaf)) & ~1);
  if((s = grow(ctx, &ctx->d_cand, &ctx->cand_cap, cand + 2 * kMaxLeaf)) != HPLB_OK) return s;
  ctx->d_cur = ctx->d_cand + cand;
  return HPLB_OK;
}

inline cudaEvent_t next_event(hplb_ctx* ctx) {
  if(ctx->ev_next == ctx->events.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    ctx->events.push_back(e);
  }
  return ctx->events[ctx->ev_next++];
}

// Every entry point starts here: the library's streams wait for the work the
// caller queued on its stream before the call (inputs written by the caller's
// kernels are complete before any kernel of the call reads them).
inline hplb_status enter(hplb_ctx* ctx) {
  CK(cudaSetDevice(ctx->device));
  CK(cudaEventRecord(ctx->ev_enter, ctx->caller));
  CK(cudaStreamWaitEvent(ctx->s_upd, ctx->ev_enter, 0));
  CK(cudaStreamWaitEvent(ctx->s_pan, ctx->ev_enter, 0));
  return HPLB_OK;
}

#define ENTER(ctx)                          \
  do {                                      \
    hplb_status e__ = hplb::enter(ctx);     \
    if(e__ != HPLB_OK) return e__;          \
  } while(0)

inline hplb_status read_status(hplb_ctx* ctx, int* info_out) {
  int st[ST_COUNT];
  CK(cudaMemcpy(st, ctx->d_status, sizeof st, cudaMemcpyDeviceToHost));
  if(info_out) *info_out = st[ST_INFO];
  if(st[ST_TIMEOUT] != 0)
    return set_err(ctx, HPLB_ERR_TIMEOUT, "a bounded device wait expired (site %d)",
                   st[ST_TIMEOUT]);
  return HPLB_OK;
}


}  // namespace hplb
