// Batched solver plan and C ABI (hplb_batch_*).  No counterpart in the
// reference, which solves one system per run.
//
// A plan fixes, for a list of system sizes: the packed layout of the A, B and
// pivot pools; the panel width of every system from its size class (the
// autotuner's table, or the built-in one); the work order (largest cost first,
// so the persistent CTAs finish together); and, per mode, a CUDA graph of
// [argument upload from pinned host memory -> work-counter reset -> one
// persistent kernel].  Every call is one graph launch.
#include <algorithm>
#include <climits>
#include <numeric>
#include <vector>

#include "ctx.h"

using namespace hplb;

static const int kClassUpper[HPLB_BATCH_CLASSES] = {48, 96, 192, 384, 768, INT_MAX};
static const int kDefaultNb[HPLB_BATCH_CLASSES]  = {8, 16, 16, 16, 16, 16};
static const int kTuneN[HPLB_BATCH_CLASSES]      = {40, 80, 160, 320, 640, 1024};

static int size_class(int n) {
  for(int c = 0; c < HPLB_BATCH_CLASSES; ++c)
    if(n < kClassUpper[c]) return c;
  return HPLB_BATCH_CLASSES - 1;
}

struct hplb_batch {
  hplb_ctx*                   ctx = nullptr;
  int                         count = 0;
  std::vector<int>            n, nrhs, nb;
  std::vector<int64_t>        a_off, b_off, p_off;
  int64_t                     a_total = 0, b_total = 0, p_total = 0;
  int                         n_max = 0, grid = 0;
  size_t                      dyn = 0;
  void*                       d_sys = nullptr;
  int*                        d_order = nullptr;
  int*                        d_counter = nullptr;
  void*                       d_args = nullptr;
  void*                       h_args = nullptr;  // pinned
  unsigned long long*         d_seeds = nullptr;
  cudaGraphExec_t             graph[6] = {};
  cudaEvent_t                 e0 = nullptr, e1 = nullptr;
  float                       last_ms = 0.f;
};

namespace {

hplb_status batch_err(hplb_batch* b, hplb_status s, const char* msg) {
  return set_err(b ? b->ctx : nullptr, s, "%s", msg);
}

// Dynamic shared memory of each mode: the gesv panel (nb x n doubles), the
// permutation gather of the solves (2n ints + 8n doubles), the residual's
// staged solution columns (8n doubles).
size_t dyn_bytes(const hplb_batch* b) {
  size_t m = 8;
  for(int i = 0; i < b->count; ++i)
    m = std::max(m, b->nb[i] == HPLB_BATCH_RECURSIVE
                        ? batch_rec_stage_bytes()
                        : (size_t)b->nb[i] * ((b->n[i] + 15) / 16 * 16 + 4) * sizeof(double));
  m = std::max(m, (size_t)9 * b->n_max * sizeof(double));
  return m;
}

// Dynamic shared memory a plan may use (and the kernels' limits set to it).
hplb_status dyn_budget(hplb_ctx* ctx, size_t* budget) {
  const cudaError_t e = batch_set_smem(budget);
  if(e != cudaSuccess) {
    cudaGetLastError();
    return set_err(ctx, HPLB_ERR_CUDA, "batch kernels' shared-memory limits: %s",
                   cudaGetErrorString(e));
  }
  return HPLB_OK;
}

// Capture (once) and launch the graph of `mode` with the arguments already in
// h_args; times the launch with events.
hplb_status run_mode(hplb_batch* b, int mode) {
  hplb_ctx*    ctx = b->ctx;
  cudaStream_t st  = ctx->s_upd;
  if(!b->graph[mode]) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaMemcpyAsync(b->d_args, b->h_args, batch_args_bytes(),
                                    cudaMemcpyHostToDevice, st);
    if(e == cudaSuccess) e = cudaMemsetAsync(b->d_counter, 0, sizeof(int), st);
    if(e == cudaSuccess) e = launch_batch(mode, b->d_args, b->grid, b->dyn, st);
    cudaError_t e2 = cudaStreamEndCapture(st, &g);
    if(e == cudaSuccess) e = e2;
    if(e == cudaSuccess) e = cudaGraphInstantiate(&b->graph[mode], g, 0);
    if(g) cudaGraphDestroy(g);
    if(e != cudaSuccess) {
      cudaGetLastError();
      b->graph[mode] = nullptr;
      return set_err(ctx, HPLB_ERR_CUDA, "batch graph capture (mode %d) failed: %s", mode,
                     cudaGetErrorString(e));
    }
  }
  CK(cudaEventRecord(b->e0, st));
  CK(cudaGraphLaunch(b->graph[mode], st));
  CK(cudaEventRecord(b->e1, st));
  CK(cudaStreamSynchronize(st));
  cudaEventElapsedTime(&b->last_ms, b->e0, b->e1);
  ctx->timing                 = hplb_timing{};
  ctx->timing.total_ms        = b->last_ms;
  ctx->timing.kernel_launches = 1;
  return HPLB_OK;
}

void fill(hplb_batch* b, double* A, const double* LU, double* B, int* ipiv, const int* ipivc,
          int* info, double alpha, const double* X, const double* Y, double* C,
          double* resid) {
  batch_fill_args(b->h_args, A, LU, B, ipiv, ipivc, info, b->d_sys, b->d_order, b->count,
                  b->d_counter, alpha, X, Y, C, b->d_seeds, resid);
}

hplb_status upload_seeds(hplb_batch* b, const uint64_t* seeds) {
  hplb_ctx* ctx = b->ctx;
  if(!seeds) return set_err(ctx, HPLB_ERR_ARG, "hplb_batch: null seeds");
  CK(cudaMemcpyAsync(b->d_seeds, seeds, (size_t)b->count * sizeof(uint64_t),
                     cudaMemcpyHostToDevice, ctx->s_upd));
  return HPLB_OK;
}

}  // namespace

extern "C" {

hplb_status hplb_batch_create(hplb_ctx* ctx, int count, const int* n, const int* nrhs,
                              const int* nb_by_class, hplb_batch** out) {
  if(!ctx) return HPLB_ERR_ARG;
  if(!out) return set_err(ctx, HPLB_ERR_ARG, "hplb_batch_create: null output");
  *out = nullptr;
  if(count < 0 || (count > 0 && (!n || !nrhs)))
    return set_err(ctx, HPLB_ERR_ARG, "hplb_batch_create: bad count or null size arrays");
  for(int i = 0; i < count; ++i) {
    if(n[i] < 1 || nrhs[i] < 0)
      return set_err(ctx, HPLB_ERR_ARG, "hplb_batch_create: system %d has n = %d, nrhs = %d", i,
                     n[i], nrhs[i]);
    if(n[i] > HPLB_BATCH_MAX_N)
      return set_err(ctx, HPLB_ERR_UNSUPPORTED, "hplb_batch_create: n = %d above %d", n[i],
                     HPLB_BATCH_MAX_N);
  }
  if(nb_by_class)
    for(int c = 0; c < HPLB_BATCH_CLASSES; ++c)
      if(nb_by_class[c] != 8 && nb_by_class[c] != 16 && nb_by_class[c] != 32 &&
         nb_by_class[c] != HPLB_BATCH_RECURSIVE)
        return set_err(ctx, HPLB_ERR_ARG,
                       "hplb_batch_create: class entries must be 8, 16, 32 or HPLB_BATCH_RECURSIVE");
  ENTER(ctx);
  size_t      budget = 0;
  hplb_status sb     = dyn_budget(ctx, &budget);
  if(sb != HPLB_OK) return sb;
  auto* b  = new hplb_batch();
  b->ctx   = ctx;
  b->count = count;
  b->n.assign(n, n + count);
  b->nrhs.assign(nrhs, nrhs + count);
  b->nb.resize(count);
  b->a_off.resize(count);
  b->b_off.resize(count);
  b->p_off.resize(count);
  for(int i = 0; i < count; ++i) {
    int w = (nb_by_class ? nb_by_class : kDefaultNb)[size_class(n[i])];
    if(w == HPLB_BATCH_RECURSIVE && n[i] > HPLB_BATCH_RECURSIVE_MAX_N) w = 16;
    while(w != HPLB_BATCH_RECURSIVE && w > 8 &&
          (size_t)w * ((n[i] + 15) / 16 * 16 + 4) * sizeof(double) > budget)
      w /= 2;
    b->nb[i]    = w;
    b->a_off[i] = b->a_total;
    b->b_off[i] = b->b_total;
    b->p_off[i] = b->p_total;
    b->a_total += (int64_t)n[i] * n[i];
    b->b_total += (int64_t)n[i] * nrhs[i];
    b->p_total += n[i];
    b->n_max = std::max(b->n_max, n[i]);
  }
  b->dyn = dyn_bytes(b);
  auto fail = [&](hplb_status s, const char* m) {
    hplb_status r = set_err(ctx, s, "hplb_batch_create: %s", m);
    hplb_batch_destroy(b);
    return r;
  };
  if(b->dyn > budget) return fail(HPLB_ERR_UNSUPPORTED, "systems too large for shared memory");
  // Largest cost first.
  std::vector<int> order(count);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    const double cx = (double)n[x] * n[x] * (n[x] + 3.0 * nrhs[x]);
    const double cy = (double)n[y] * n[y] * (n[y] + 3.0 * nrhs[y]);
    return cx > cy;
  });
  std::vector<unsigned char> sys(batch_sys_bytes() * std::max(count, 1));
  for(int i = 0; i < count; ++i)
    batch_fill_sys(sys.data(), i, n[i], nrhs[i], b->nb[i], b->a_off[i], b->b_off[i], b->p_off[i]);
  const size_t cnt = (size_t)std::max(count, 1);
  if(cudaMalloc(&b->d_sys, sys.size()) != cudaSuccess ||
     cudaMalloc(&b->d_order, cnt * sizeof(int)) != cudaSuccess ||
     cudaMalloc(&b->d_counter, sizeof(int)) != cudaSuccess ||
     cudaMalloc(&b->d_args, batch_args_bytes()) != cudaSuccess ||
     cudaMalloc(&b->d_seeds, cnt * sizeof(unsigned long long)) != cudaSuccess ||
     cudaHostAlloc(&b->h_args, batch_args_bytes(), cudaHostAllocDefault) != cudaSuccess ||
     cudaEventCreate(&b->e0) != cudaSuccess || cudaEventCreate(&b->e1) != cudaSuccess) {
    cudaGetLastError();
    return fail(HPLB_ERR_OOM, "plan allocation failed");
  }
  if(cudaMemcpy(b->d_sys, sys.data(), sys.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
     (count > 0 && cudaMemcpy(b->d_order, order.data(), (size_t)count * sizeof(int),
                              cudaMemcpyHostToDevice) != cudaSuccess)) {
    cudaGetLastError();
    return fail(HPLB_ERR_CUDA, "plan upload failed");
  }
  // One CTA per SM (the kernels are built for one 512-thread CTA per SM);
  // never more CTAs than systems.
  b->grid = std::max(1, std::min(ctx->num_sms, count));
  *out    = b;
  return HPLB_OK;
}

void hplb_batch_destroy(hplb_batch* b) {
  if(!b) return;
  if(b->ctx) {
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->s_upd);
  }
  for(auto& g : b->graph)
    if(g) cudaGraphExecDestroy(g);
  if(b->d_sys) cudaFree(b->d_sys);
  if(b->d_order) cudaFree(b->d_order);
  if(b->d_counter) cudaFree(b->d_counter);
  if(b->d_args) cudaFree(b->d_args);
  if(b->d_seeds) cudaFree(b->d_seeds);
  if(b->h_args) cudaFreeHost(b->h_args);
  if(b->e0) cudaEventDestroy(b->e0);
  if(b->e1) cudaEventDestroy(b->e1);
  delete b;
}

hplb_status hplb_batch_layout(const hplb_batch* b, int64_t* a_elems, int64_t* b_elems,
                              int64_t* p_elems, int64_t* a_off, int64_t* b_off, int64_t* p_off,
                              int* nb) {
  if(!b) return HPLB_ERR_ARG;
  if(a_elems) *a_elems = b->a_total;
  if(b_elems) *b_elems = b->b_total;
  if(p_elems) *p_elems = b->p_total;
  for(int i = 0; i < b->count; ++i) {
    if(a_off) a_off[i] = b->a_off[i];
    if(b_off) b_off[i] = b->b_off[i];
    if(p_off) p_off[i] = b->p_off[i];
    if(nb) nb[i] = b->nb[i];
  }
  return HPLB_OK;
}

hplb_status hplb_batch_matgen(hplb_batch* b, const uint64_t* seeds, double* dA, double* dB) {
  if(!b) return HPLB_ERR_ARG;
  hplb_ctx* ctx = b->ctx;
  if(b->count == 0) return HPLB_OK;
  if(!dA || (b->b_total > 0 && !dB)) return batch_err(b, HPLB_ERR_ARG, "hplb_batch_matgen: null pool");
  ENTER(ctx);
  hplb_status s = upload_seeds(b, seeds);
  if(s != HPLB_OK) return s;
  fill(b, dA, nullptr, dB, nullptr, nullptr, nullptr, 0.0, nullptr, nullptr, nullptr, nullptr);
  return run_mode(b, 4);
}

hplb_status hplb_batch_gesv(hplb_batch* b, double* dA, double* dB, int* dipiv, int* dinfo) {
  if(!b) return HPLB_ERR_ARG;
  hplb_ctx* ctx = b->ctx;
  if(b->count == 0) return HPLB_OK;
  if(!dA || !dipiv || !dinfo || (b->b_total > 0 && !dB))
    return batch_err(b, HPLB_ERR_ARG, "hplb_batch_gesv: null pool");
  ENTER(ctx);
  fill(b, dA, nullptr, dB, dipiv, nullptr, dinfo, 0.0, nullptr, nullptr, nullptr, nullptr);
  return run_mode(b, 0);
}

hplb_status hplb_batch_getrs(hplb_batch* b, int trans, const double* dLU, const int* dipiv,
                             double* dB) {
  if(!b) return HPLB_ERR_ARG;
  hplb_ctx* ctx = b->ctx;
  if(trans != 0 && trans != 1) return batch_err(b, HPLB_ERR_ARG, "hplb_batch_getrs: trans must be 0 or 1");
  if(b->count == 0 || b->b_total == 0) return HPLB_OK;
  if(!dLU || !dipiv || !dB) return batch_err(b, HPLB_ERR_ARG, "hplb_batch_getrs: null pool");
  ENTER(ctx);
  fill(b, nullptr, dLU, dB, nullptr, dipiv, nullptr, 0.0, nullptr, nullptr, nullptr, nullptr);
  return run_mode(b, trans ? 2 : 1);
}

hplb_status hplb_batch_rank_k(hplb_batch* b, double alpha, const double* dX, const double* dY,
                              double* dC) {
  if(!b) return HPLB_ERR_ARG;
  hplb_ctx* ctx = b->ctx;
  if(b->count == 0) return HPLB_OK;
  if(!dC || (b->b_total > 0 && (!dX || !dY)))
    return batch_err(b, HPLB_ERR_ARG, "hplb_batch_rank_k: null pool");
  ENTER(ctx);
  fill(b, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, alpha, dX, dY, dC, nullptr);
  return run_mode(b, 3);
}

hplb_status hplb_batch_residual(hplb_batch* b, const uint64_t* seeds, const double* dX,
                                double* dresid) {
  if(!b) return HPLB_ERR_ARG;
  hplb_ctx* ctx = b->ctx;
  if(b->count == 0) return HPLB_OK;
  if(!dresid || (b->b_total > 0 && !dX))
    return batch_err(b, HPLB_ERR_ARG, "hplb_batch_residual: null pool");
  ENTER(ctx);
  hplb_status s = upload_seeds(b, seeds);
  if(s != HPLB_OK) return s;
  fill(b, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0.0, dX, nullptr, nullptr, dresid);
  return run_mode(b, 5);
}

hplb_status hplb_batch_last_ms(const hplb_batch* b, double* ms) {
  if(!b || !ms) return HPLB_ERR_ARG;
  *ms = b->last_ms;
  return HPLB_OK;
}

// The autotuner: for each size class, a batch of 2 x (SM count) systems of the
// class's representative size is generated and solved with each candidate
// (right-looking panels of 8, 16 or 32 columns, or the recursive
// factorisation); the fastest (best of three timed graph launches after a
// warm-up) goes into nb_by_class.
hplb_status hplb_batch_tune(hplb_ctx* ctx, int nrhs, int* nb_by_class, double* ms_table) {
  if(!ctx) return HPLB_ERR_ARG;
  if(!nb_by_class || nrhs < 0) return set_err(ctx, HPLB_ERR_ARG, "hplb_batch_tune: bad argument");
  ENTER(ctx);
  static const int cand[4] = {8, 16, 32, HPLB_BATCH_RECURSIVE};
  size_t           budget  = 0;
  hplb_status      sb      = dyn_budget(ctx, &budget);
  if(sb != HPLB_OK) return sb;
  const int        count   = 2 * ctx->num_sms;
  for(int c = 0; c < HPLB_BATCH_CLASSES; ++c) {
    const int n    = kTuneN[c];
    double    best = 1e30;
    nb_by_class[c] = kDefaultNb[c];
    for(int q = 0; q < 4; ++q) {
      if(ms_table) ms_table[c * 4 + q] = -1.0;
      if(cand[q] != HPLB_BATCH_RECURSIVE &&
         (size_t)cand[q] * ((n + 15) / 16 * 16 + 4) * sizeof(double) > budget)
        continue;
      int table[HPLB_BATCH_CLASSES];
      for(int z = 0; z < HPLB_BATCH_CLASSES; ++z) table[z] = cand[q];
      std::vector<int> nv(count, n), rv(count, nrhs);
      hplb_batch*      b = nullptr;
      hplb_status      s = hplb_batch_create(ctx, count, nv.data(), rv.data(), table, &b);
      if(s != HPLB_OK) return s;
      double *dA = nullptr, *dB = nullptr;
      int *   dP = nullptr, *dI = nullptr;
      bool    ok = cudaMalloc(&dA, (size_t)b->a_total * sizeof(double)) == cudaSuccess &&
                cudaMalloc(&dB, (size_t)std::max<int64_t>(b->b_total, 1) * sizeof(double)) ==
                    cudaSuccess &&
                cudaMalloc(&dP, (size_t)b->p_total * sizeof(int)) == cudaSuccess &&
                cudaMalloc(&dI, (size_t)count * sizeof(int)) == cudaSuccess;
      std::vector<uint64_t> seeds(count);
      for(int i = 0; i < count; ++i) seeds[i] = 1000 + i;
      double t = 1e30;
      if(ok) {
        for(int rep = 0; rep < 4 && s == HPLB_OK; ++rep) {
          s = hplb_batch_matgen(b, seeds.data(), dA, dB);
          if(s == HPLB_OK) s = hplb_batch_gesv(b, dA, dB, dP, dI);
          if(s == HPLB_OK && rep > 0) t = std::min(t, (double)b->last_ms);
        }
      } else {
        cudaGetLastError();
        s = set_err(ctx, HPLB_ERR_OOM, "hplb_batch_tune: allocation failed");
      }
      cudaFree(dA);
      cudaFree(dB);
      cudaFree(dP);
      cudaFree(dI);
      hplb_batch_destroy(b);
      if(s != HPLB_OK) return s;
      if(ms_table) ms_table[c * 4 + q] = t;
      if(t < best) {
        best           = t;
        nb_by_class[c] = cand[q];
      }
    }
  }
  return HPLB_OK;
}

}  // extern "C"
