// srmg_engine.cu -- host side of the persistent V-cycle engine (srmg_engine.cuh).
#include <cstring>

#include "srmg_ctx.h"
#include "srmg_engine.cuh"
#include "srmg_internal.h"

using namespace srmg;

#define CK(call)                                              \
  do {                                                        \
    int _rc = cuda_check(ctx, (call), #call);                 \
    if (_rc) return _rc;                                      \
  } while (0)
#define RC(call)               \
  do {                         \
    int _rc = (call);          \
    if (_rc) return _rc;       \
  } while (0)

namespace {

template <typename T>
WTab<T> wtab_of(srmg_ctx *ctx);
template <>
WTab<double> wtab_of<double>(srmg_ctx *ctx) { return WTab<double>{ctx->d_wm64, ctx->d_wp64}; }
template <>
WTab<float> wtab_of<float>(srmg_ctx *ctx) { return WTab<float>{ctx->d_wm32, ctx->d_wp32}; }
template <typename T>
const T *wrow_of(srmg_ctx *ctx);
template <>
const double *wrow_of<double>(srmg_ctx *ctx) { return ctx->d_wrow64; }
template <>
const float *wrow_of<float>(srmg_ctx *ctx) { return ctx->d_wrow32; }

// Threads per CTA for this context: the "engine_threads" option, else by tree size
// (measured: 768 threads are faster up to ~16k blocks, 1024 above).
int engine_threads_of(const srmg_ctx *ctx) {
  if (ctx->engine_threads) return ctx->engine_threads;
  return ctx->max_blk <= 16384 ? kEngineNarrow : kEngineWide;
}

template <typename T>
const void *engine_kernel(int threads) {
  return threads == kEngineNarrow ? (const void *)k_engine_vcycle<T, kEngineNarrow>
                                  : (const void *)k_engine_vcycle<T, kEngineWide>;
}

template <typename T>
int engine_grid(srmg_ctx *ctx, int threads, int *grid) {
  if (ctx->num_sms == 0) CK(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->device));
  const size_t smem = engine_smem_bytes<T>(threads);
  CK(cudaFuncSetAttribute(engine_kernel<T>(threads), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, engine_kernel<T>(threads), threads, smem));
  if (per_sm < 1) return fail(ctx, SRMG_ERR_CUDA, "engine kernel cannot be resident (occupancy 0)");
  *grid = ctx->num_sms * std::min(per_sm, 1);
  return SRMG_OK;
}

}  // namespace

// Levels 1..K run in CTA 0: the largest K such that every level 1..K holds at most
// ctx->local_max_blocks blocks.
int srmg::engine_local_top(srmg_ctx *ctx, int lmax) {
  int K = 0;
  for (int l = 1; l <= lmax; l++) {
    if (ctx->nblk_host[l - 1] > ctx->local_max_blocks) break;
    K = l;
  }
  return K;
}

// Launch state shared by every engine launch: tree tables, item tables, barrier and
// error words, the frozen flags (zeroed) and norm scratch.
template <typename T>
static int engine_common(srmg_ctx *ctx, EngArgs<T> &A, T *u, const ItemTabs &tabs, int geom) {
  memset(&A, 0, sizeof A);
  A.u = u;
  {
    DevBuf &alt = (sizeof(T) == 8) ? ctx->f64[5] : ctx->f32[5];
    RC(ensure(ctx, alt, (size_t)ctx->max_blk * kSS * sizeof(T)));
    A.ualt = (T *)alt.p;
  }
  for (int l = 0; l < ctx->nlev; l++) {
    A.tr.lvl_rec[l] = ctx->lv[l].rec;
    A.tr.lvl_blocks[l] = ctx->lv[l].blocks;
    A.tr.lvl_child[l] = ctx->lv[l].child;
    A.tr.nblk[l] = ctx->nblk_host[l];
    A.tr.nch[l] = ctx->nch_host[l];
  }
  A.tr.info = ctx->d_info;
  A.tr.faces = ctx->d_faceb;
  A.tr.kids = ctx->d_kids;
  A.wt = wtab_of<T>(ctx);
  A.wrow = (geom == 1 || geom == 2) ? wrow_of<T>(ctx) : nullptr;
  A.geom = geom;
  A.nitems = ctx->nitems;
  A.nlev_tab = ctx->nlev;
  A.it_par = (sizeof(T) == 8) ? (const T *)(const void *)tabs.par64 : (const T *)(const void *)tabs.par32;
  A.it_sgbits = tabs.sgbits;
  A.it_lrange = ctx->d_it_lrange;
  const size_t sync_bytes = 256 + sizeof(int) * (size_t)ctx->nitems;
  RC(ensure(ctx, ctx->sync, sync_bytes));
  A.bar = (unsigned *)ctx->sync.p;
  A.err = (int *)((char *)ctx->sync.p + 128);
  A.frozen = (int *)((char *)ctx->sync.p + 256);
  A.timeout_ns = 2000000000LL;  // 2 s per barrier wait
  if (ctx->trace_on) {
    RC(ensure(ctx, ctx->trace, kTraceMax * sizeof(long long)));
    A.trace = (long long *)ctx->trace.p;
  }
  CK(cudaMemsetAsync(ctx->sync.p, 0, sync_bytes, ctx->stream));
  return SRMG_OK;
}

template <typename T>
static int engine_launch(srmg_ctx *ctx, EngArgs<T> &A) {
  int grid = 0;
  const int threads = engine_threads_of(ctx);
  RC(engine_grid<T>(ctx, threads, &grid));  // also raises the dynamic shared-memory limit
  if (ctx->engine_ctas > 0 && ctx->engine_ctas < grid) grid = ctx->engine_ctas;
  void *args[] = {&A};
  CK(cudaLaunchCooperativeKernel(engine_kernel<T>(threads), dim3(grid), dim3(threads), args,
                                 engine_smem_bytes<T>(threads), ctx->stream));
  ctx->launches++;
  return SRMG_OK;
}

template <typename T>
int srmg::engine_vcycle(srmg_ctx *ctx, T *u, T *b, T *u1, T *e, const ItemTabs &tabs, int geom, int lmax,
                        int ndown, int ntop, int nup, const EngineRun *run) {
  const EngineRun none;
  if (!run) run = &none;
  if (ctx->nlev > kMaxLev) return fail(ctx, SRMG_ERR_UNSUPPORTED, "engine supports at most %d levels", kMaxLev);
  if (lmax == 0) lmax = ctx->nlev;
  int L = 0;
  for (int l = 1; l <= lmax; l++)
    if (ctx->nblk_host[l - 1] > 0) L = l;
  if (L == 0) return SRMG_OK;
  EngArgs<T> A;
  RC(engine_common<T>(ctx, A, u, tabs, geom));
  A.b = b;
  // Tolerance-driven solves run on the engine's own copy of b (FP64: a copy of the
  // caller's b; mixed: the FP32 defect), whose ghost cells then carry the neighbours'
  // edge values, filled once per launch (FP64) or with every defect (mixed).  One
  // V-cycle per launch (vcycle!) leaves the caller's b ghosts alone.
  A.bghost = run->max_cycles > 0 ? 1 : 0;
  A.u1 = u1;
  A.e = e;
  A.lmax = L;
  A.ndown = ndown;
  A.ntop = ntop;
  A.nup = nup;
  A.local_top = engine_local_top(ctx, L);
  A.top = 1;
  if (run->direct && tabs.P) {
    A.it_P = tabs.P;
    if (tabs.top == 2 && L >= 2) {
      // level 2 is solved directly by every CTA: no level below it is visited, and none
      // runs CTA-locally
      A.top = 2;
      A.local_top = 0;
    }
  }
  A.max_cycles = run->max_cycles;
  A.tol = run->tol;
  if (run->max_cycles > 0) {
    const int64_t total = std::max(ctx->nchunk, 1);
    RC(ensure(ctx, ctx->part, sizeof(double) * 2 * (size_t)total));
    A.bpart = (double *)ctx->part.p;
    A.bpart_b = A.bpart + total;
    A.chunks = ctx->d_chunks;
    A.nchunk = ctx->nchunk;
    A.it_chunks = ctx->d_it_chunks;
    RC(ensure(ctx, ctx->istat, sizeof(double) * (kItemRec * (size_t)ctx->nitems + 8)));
    A.inorm = (double *)ctx->istat.p;
    A.out = A.inorm + kItemRec * ctx->nitems;
  }
  if (run->u64) {
    if (run->max_cycles <= 0) return fail(ctx, SRMG_ERR_BADARG, "mixed engine step needs the device loop");
    A.mx.u64 = run->u64;
    A.mx.b64 = run->b64;
    A.mx.wt64 = WTab<double>{ctx->d_wm64, ctx->d_wp64};
    A.mx.it_par64 = tabs.par64;
    A.mx.refbnd_levels = ctx->refbnd_levels;
    A.mx.apply_update = run->apply_update;
    A.inner = std::max(1, run->inner);
  }
  return engine_launch<T>(ctx, A);
}

// gauss_seidel_iter! on one level through the persistent kernel (tabs built with the
// level's scale).
template <typename T>
int srmg::engine_smooth(srmg_ctx *ctx, T *u, const T *b, const ItemTabs &tabs, int geom, int level, int n) {
  if (n <= 0 || ctx->nblk_host[level - 1] == 0) return SRMG_OK;
  EngArgs<T> A;
  RC(engine_common<T>(ctx, A, u, tabs, geom));
  A.b = const_cast<T *>(b);  // read only: bghost stays 0
  A.lmax = level;
  A.smooth_level = level;
  A.smooth_n = n;
  return engine_launch<T>(ctx, A);
}
template int srmg::engine_smooth<double>(srmg_ctx *, double *, const double *, const ItemTabs &, int, int, int);

template int srmg::engine_vcycle<double>(srmg_ctx *, double *, double *, double *, double *, const ItemTabs &,
                                         int, int, int, int, int, const EngineRun *);
template int srmg::engine_vcycle<float>(srmg_ctx *, float *, float *, float *, float *, const ItemTabs &, int,
                                        int, int, int, int, const EngineRun *);

extern "C" int srmg_get_trace(srmg_ctx *ctx, int64_t *out, int max_entries) {
  if (!ctx || !out || max_entries < 0) return SRMG_ERR_BADARG;
  if (!ctx->trace.p) return 0;
  const int n = std::min(max_entries, kTraceMax);
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpy(out, ctx->trace.p, n * sizeof(long long), cudaMemcpyDeviceToHost));
  int k = 0;
  while (k < n && out[k] != 0) k++;
  return k;
}

// Reads the engine's error word (after the stream has been synchronised by the caller).
int srmg::engine_check(srmg_ctx *ctx) {
  if (!ctx->sync.p) return SRMG_OK;
  int err = 0;
  CK(cudaMemcpy(&err, (char *)ctx->sync.p + 128, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) return fail(ctx, SRMG_ERR_TIMEOUT, "engine barrier timed out (error word %d)", err);
  return SRMG_OK;
}
