// srmg_solve.cu -- tolerance-driven solves on top of the V-cycle:
//   * FP64 mode: repeated reference V-cycles (vcycle!, src/multigrid.jl:60-106) with
//     the resnorm! residual (src/multigrid.jl:391-417) checked after every cycle;
//   * mixed mode: FP64 defect correction around FP32 V-cycles whose coarsest level
//     is solved directly in FP64.
#include <cmath>
#include <cstring>
#include <vector>

#include "srmg_ctx.h"
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

// Defect of the FP64 iterate on one level, written as the FP32 right-hand side of the
// correction problem (b_e = -r, i.e. L e + s (-r) = 0), the FP32 correction zeroed
// (whole block), and the leaf-cell squared norm of r accumulated per CTA.
template <int NT>
__global__ void __launch_bounds__(NT) k_defect(float *__restrict__ be, float *__restrict__ e,
                                               double *__restrict__ part,
                                               const double *__restrict__ u,
                                               const double *__restrict__ b, LevelView lv,
                                               OpParams<double> p, WTab<double> wt, double wl) {
  double acc = 0.0;
  const int64_t total = (int64_t)lv.nblk * 256;
  for (int64_t t = blockIdx.x * (int64_t)NT + threadIdx.x; t < total; t += (int64_t)gridDim.x * NT) {
    const int bi = (int)(t >> 8), c = (int)(t & 255);
    const int x = 2 + (c & 15), y = 2 + (c >> 4);
    const int4 bk = lv.blocks[bi];
    const int64_t base = (int64_t)bk.x * kSS;
    const W5<double> w = weights<double>(wt, p.geom, bk.y, bk.z, x, y);
    const double Lu = apply5<double>(u + base, x, y, w, p.centre);
    const int64_t o = base + x + kS * y;
    const double r = -(b[o] + Lu / p.s);
    be[o] = (float)(-r);
    const int sub = ((x - 2) >> 3) + 2 * ((y - 2) >> 3);
    if (!((bk.w >> sub) & 1)) acc = fma(r, r, acc);
  }
  // zero the correction, ghosts included
  const int64_t tz = (int64_t)lv.nblk * kSS;
  for (int64_t t = blockIdx.x * (int64_t)NT + threadIdx.x; t < tz; t += (int64_t)gridDim.x * NT) {
    const int bi = (int)(t / kSS), c = (int)(t % kSS);
    e[(int64_t)lv.blocks[bi].x * kSS + c] = 0.f;
  }
  __shared__ double sh[NT / 32];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = (threadIdx.x < NT / 32) ? sh[threadIdx.x] : 0.0;
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if (threadIdx.x == 0) part[blockIdx.x] = v * wl;
  }
}

// u += e on the valid cells of one level.
__global__ void k_update(double *__restrict__ u, const float *__restrict__ e, LevelView lv) {
  const int64_t total = (int64_t)lv.nblk * 256;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t >> 8), c = (int)(t & 255);
    const int64_t o = (int64_t)lv.blocks[bi].x * kSS + (2 + (c & 15)) + kS * (2 + (c >> 4));
    u[o] += (double)e[o];
  }
}

// Coarsest level, direct: e = P b with P = -s A^{-1} precomputed in FP64 (one warp per
// row).  Unknown q of level 1 is cell (x, y) of the level's block q / 256.
__global__ void k_coarse_direct(float *__restrict__ e, const float *__restrict__ b,
                                const double *__restrict__ P, LevelView lv, int n) {
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (row >= n) return;
  const double *pr = P + (int64_t)row * n;
  double acc = 0.0;
  for (int j = lane; j < n; j += 32) {
    const int bj = j >> 8, cj = j & 255;
    const int64_t o = (int64_t)lv.blocks[bj].x * kSS + (2 + (cj & 15)) + kS * (2 + (cj >> 4));
    acc = fma(pr[j], (double)b[o], acc);
  }
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if (lane == 0) {
    const int bi = row >> 8, ci = row & 255;
    const int64_t o = (int64_t)lv.blocks[bi].x * kSS + (2 + (ci & 15)) + kS * (2 + (ci >> 4));
    e[o] = (float)acc;
  }
}

int grid_for(int64_t work, int threads, int cap) {
  int64_t g = (work + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

// FP32 V-cycle with the FP64 direct coarsest-level solve (when available), on the
// per-operation kernels (used when the persistent engine is switched off).  Same
// structure as the reference V-cycle; only the top changes.
int vcycle_mixed(srmg_ctx *ctx, float *e, float *b, float *r, float *u1, double s, int op, double k2,
                 int geom, const Signs &sg, int ndown, int ntop, int nup, double omega, const ItemTabs &tabs) {
  const int lmax = ctx->nlev;
  for (int l = lmax; l >= 2; l--) {
    if (ctx->nblk_host[l - 1] == 0) continue;
    const double sl = level_scale(s, l);
    const OpParams<float> p = op_params<float>(op, geom, k2, sl, omega);
    const OpParams<float> pc = op_params<float>(op, geom, k2, 4 * sl, omega);
    RC(L_gs_iter<float>(ctx, e, b, l, p, ndown, sg));
    RC(L_restrict<float>(ctx, e, l));
    RC(L_fill_ghost<float>(ctx, e, l - 1, sg, 7));
    RC(L_copy<float>(ctx, u1, e, l - 1));
    RC(L_residual<float>(ctx, r, e, b, l, p));
    RC(L_restrict<float>(ctx, r, l));
    RC(L_postrestrict<float>(ctx, b, e, r, l, pc));
  }
  if (tabs.P0) {
    const int n = tabs.n0;
    k_coarse_direct<<<(n + 7) / 8, 256, 0, ctx->stream>>>(e, b, tabs.P0, ctx->lv[0].view(1), n);
    ctx->launches++;
    RC(L_fill_ghost<float>(ctx, e, 1, sg, 3));
  } else {
    const OpParams<float> p = op_params<float>(op, geom, k2, s, omega);
    RC(L_gs_iter<float>(ctx, e, b, 1, p, std::max(ntop, 64), sg));
  }
  for (int l = 2; l <= lmax; l++) {
    if (ctx->nblk_host[l - 1] == 0) continue;
    const double sl = level_scale(s, l);
    const OpParams<float> p = op_params<float>(op, geom, k2, sl, omega);
    RC(L_diff<float>(ctx, u1, e, u1, l - 1));
    RC(L_fill_ghost<float>(ctx, u1, l - 1, sg, 7));
    RC(L_interp_add<float>(ctx, e, u1, l));
    RC(L_fill_ghost<float>(ctx, e, l, sg, 7));
    RC(L_gs_iter<float>(ctx, e, b, l, p, nup, sg));
    RC(L_fill_ghost<float>(ctx, e, l, sg, 7));
  }
  return SRMG_OK;
}

// Restrict u onto every covered subblock (finest first) and refill ghosts level by
// level, so that the FP64 iterate is the composite-grid function of its leaf cells.
int make_consistent(srmg_ctx *ctx, double *u, const Signs &sg) {
  for (int l = ctx->nlev; l >= 2; l--) RC(L_restrict<double>(ctx, u, l));
  for (int l = 1; l <= ctx->nlev; l++) RC(L_fill_ghost<double>(ctx, u, l, sg, 7));
  return SRMG_OK;
}

// Defect + norm over all levels; result (sqrt of the weighted sum) in small[slot].
int defect_all(srmg_ctx *ctx, float *be, float *e, const double *u, const double *b, double s, int op,
               double k2, int geom, int slot) {
  constexpr int NT = 256;
  int total = 0;
  std::vector<int> grids(ctx->nlev);
  for (int l = 1; l <= ctx->nlev; l++) {
    const int n = ctx->nblk_host[l - 1];
    grids[l - 1] = n ? grid_for((int64_t)n * 256, NT, 148 * 4) : 0;
    total += grids[l - 1];
  }
  RC(ensure(ctx, ctx->part, sizeof(double) * std::max(total, 1)));
  double *part = (double *)ctx->part.p;
  int off = 0;
  for (int l = 1; l <= ctx->nlev; l++) {
    if (!grids[l - 1]) continue;
    const double sl = level_scale(s, l);
    const OpParams<double> p = op_params<double>(op, geom, k2, sl, 1.0);
    const double wl = 1.0 / (double)((int64_t)1 << (2 * (l - 1)));
    k_defect<NT><<<grids[l - 1], NT, 0, ctx->stream>>>(be, e, part + off, u, b, ctx->lv[l - 1].view(l), p,
                                                      WTab<double>{ctx->d_wm64, ctx->d_wp64}, wl);
    ctx->launches++;
    off += grids[l - 1];
  }
  k_reduce_sqrt<1024><<<1, 1024, 0, ctx->stream>>>((double *)ctx->small.p + slot, part, total);
  ctx->launches++;
  return SRMG_OK;
}

}  // namespace

extern "C" void srmg_solve_opts_default(srmg_solve_opts *o) {
  if (!o) return;
  memset(o, 0, sizeof *o);
  o->tol = 1e-8;
  o->max_cycles = 1000;
  o->mode = SRMG_MODE_FP64;
  o->ndown = 2;
  o->ntop = 4;
  o->nup = 2;
  o->omega = 1.0;
  o->inner_cycles = 2;
  o->warm_start = 0;
}

// Per-item statistics from the device loop's results (read_items).
static void item_stats(srmg_ctx *ctx, int k, srmg_stats *st) {
  const double *io = ctx->h_items + kItemRec * k;
  const double bn = io[1] > 0 ? io[1] : 1.0;
  st->bnorm = io[1];
  st->rel_residual = io[0] / bn;
  st->initial_rel = io[2] / bn;
  st->cycles = (int)io[3];
  st->outer = (int)io[4];
  st->status = std::isfinite(st->rel_residual) ? SRMG_OK : SRMG_ERR_DIVERGED;
}

bool srmg::engine_ok(srmg_ctx *ctx, const srmg_solve_opts *o, std::initializer_list<const void *> ptrs) {
  uintptr_t a = 0;
  for (const void *p : ptrs) a |= reinterpret_cast<uintptr_t>(p);
  return ctx->use_engine && !ctx->has_corners && (a & 15) == 0 && o->ndown >= 1 && o->ntop >= 1 && o->nup >= 1 &&
         ctx->nlev <= 30;
}

// Work buffers of a solve (allocated before any capture: nothing allocates later).
int srmg::solve_reserve(srmg_ctx *ctx, int64_t nblk_alloc, int mode) {
  if (mode != SRMG_MODE_MIXED) {
    const size_t bytes = (size_t)nblk_alloc * kSS * sizeof(double);
    for (int i : {2, 3, 4}) RC(ensure(ctx, ctx->f64[i], bytes));
  } else {
    const size_t b32 = (size_t)nblk_alloc * kSS * sizeof(float);
    for (int i = 0; i < 4; i++) RC(ensure(ctx, ctx->f32[i], b32));
  }
  return SRMG_OK;
}

// The engine solve of every item, enqueued on the stream without any host
// synchronisation (so that it can be captured); read_items / items_stats finish it.
int srmg::solve_enqueue(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, const ItemTabs &tabs,
                        int geom, const srmg_solve_opts *o) {
  RC(solve_reserve(ctx, nblk_alloc, o->mode));
  EngineRun run;
  run.max_cycles = std::max(1, o->max_cycles);
  run.tol = o->tol;
  if (o->mode != SRMG_MODE_MIXED) {
    const size_t bytes = (size_t)nblk_alloc * kSS * sizeof(double);
    double *bw = (double *)ctx->f64[4].p, *r = (double *)ctx->f64[2].p, *u1 = (double *)ctx->f64[3].p;
    CK(cudaMemcpyAsync(bw, b, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    run.direct = o->mode == SRMG_MODE_FP64_DIRECT;
    return engine_vcycle<double>(ctx, u, bw, u1, r, tabs, geom, 0, o->ndown, o->ntop, o->nup, &run);
  }
  const size_t b32 = (size_t)nblk_alloc * kSS * sizeof(float);
  float *e = (float *)ctx->f32[0].p, *be = (float *)ctx->f32[1].p, *r = (float *)ctx->f32[2].p,
        *u1 = (float *)ctx->f32[3].p;
  CK(cudaMemsetAsync(r, 0, b32, ctx->stream));
  CK(cudaMemsetAsync(u1, 0, b32, ctx->stream));
  run.direct = true;
  run.u64 = u;
  run.b64 = b;
  run.inner = std::max(1, o->inner_cycles);
  // max_cycles caps defect-correction steps in mixed mode; the device loop counts V-cycles
  run.max_cycles = (int)std::min<int64_t>((int64_t)run.max_cycles * run.inner, 1 << 30);
  return engine_vcycle<float>(ctx, e, be, u1, r, tabs, geom, 0, o->ndown, o->ntop, o->nup, &run);
}

void srmg::items_stats(srmg_ctx *ctx, const srmg_solve_opts *o, srmg_stats *st) {
  for (int k = 0; k < ctx->nitems; k++) {
    item_stats(ctx, k, &st[k]);
  }
}

// FP64 solve of every item: the whole tolerance loop in one persistent launch.
static int solve_fp64(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, const ItemSpec *specs,
                      int geom, const srmg_solve_opts *o, srmg_stats *st) {
  RC(solve_reserve(ctx, nblk_alloc, SRMG_MODE_FP64));
  double *bw = (double *)ctx->f64[4].p, *r = (double *)ctx->f64[2].p, *u1 = (double *)ctx->f64[3].p;
  const bool direct = o->mode == SRMG_MODE_FP64_DIRECT;
  if (direct)
    for (int k = 0; k < ctx->nitems; k++)
      if (specs[k].op == SRMG_OP_LAPLACIAN4)
        return fail(ctx, SRMG_ERR_UNSUPPORTED, "the direct coarsest solve supports order-2 discretisations");
  if (engine_ok(ctx, o, {u, b, bw, r, u1})) {
    ItemTabs tabs;
    RC(prepare_items(ctx, specs, geom, o->omega, direct, 0, 0.0, &tabs, direct_top(ctx)));
    RC(solve_enqueue(ctx, u, b, nblk_alloc, tabs, geom, o));
    RC(read_items(ctx));
    items_stats(ctx, o, st);
    return SRMG_OK;
  }
  if (direct) return fail(ctx, SRMG_ERR_UNSUPPORTED, "SRMG_MODE_FP64_DIRECT needs the persistent engine");
  const size_t bytes = (size_t)nblk_alloc * kSS * sizeof(double);
  CK(cudaMemcpyAsync(bw, b, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  // per-operation kernels, host loop (one item)
  if (ctx->nitems != 1) return fail(ctx, SRMG_ERR_UNSUPPORTED, "batched solves need the persistent engine");
  const ItemSpec &sp = specs[0];
  RC(leafnorm_dev<double>(ctx, u, b, sp.s, sp.op, sp.k2, geom, 1, 1));
  RC(leafnorm_dev<double>(ctx, u, bw, sp.s, sp.op, sp.k2, geom, 0, 0));
  RC(read_small(ctx, 2));
  const double bn = ctx->h_small[1] > 0 ? ctx->h_small[1] : 1.0;
  st->bnorm = ctx->h_small[1];
  double rel = ctx->h_small[0] / bn;
  st->initial_rel = rel;
  int c = 0;
  while (rel > o->tol && c < o->max_cycles) {
    RC(vcycle_ops(ctx, u, bw, r, u1, sp.s, sp.op, sp.k2, geom, sp.bc, 0, o->ndown, o->ntop, o->nup, o->omega, 1));
    c++;
    RC(leafnorm_dev<double>(ctx, u, bw, sp.s, sp.op, sp.k2, geom, 0, 0));
    RC(read_small(ctx, 1));
    const double nrel = ctx->h_small[0] / bn;
    if (!std::isfinite(nrel)) {
      st->cycles = c;
      st->rel_residual = nrel;
      st->status = SRMG_ERR_DIVERGED;
      return SRMG_OK;
    }
    rel = nrel;
  }
  st->cycles = c;
  st->rel_residual = rel;
  return SRMG_OK;
}

// Mixed-precision solve of every item.  With the engine, every defect-correction step
// (FP64 update, composite consistency, FP64 defect and its leaf norm, FP32 V-cycle
// with the FP64 direct coarsest-level solve) runs in one persistent launch until each
// item's defect norm is <= tol * leafnorm(b).
static int solve_mixed(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, const ItemSpec *specs,
                       int geom, const srmg_solve_opts *o, srmg_stats *st) {
  for (int k = 0; k < ctx->nitems; k++)
    if (specs[k].op == SRMG_OP_LAPLACIAN4)
      return fail(ctx, SRMG_ERR_UNSUPPORTED, "mixed precision supports order-2 discretisations; use FP64 mode");
  ItemTabs tabs;
  // the persistent engine solves directly on level 2 where it can (direct_top), the
  // per-operation path on level 1
  const bool engine = engine_ok(ctx, o, {u, b});
  RC(prepare_items(ctx, specs, geom, o->omega, true, 0, 0.0, &tabs, engine ? direct_top(ctx) : 1));
  if (engine) {
    RC(solve_enqueue(ctx, u, b, nblk_alloc, tabs, geom, o));
    RC(read_items(ctx));
    items_stats(ctx, o, st);
    return SRMG_OK;
  }
  RC(solve_reserve(ctx, nblk_alloc, SRMG_MODE_MIXED));
  const size_t b32 = (size_t)nblk_alloc * kSS * sizeof(float);
  float *e = (float *)ctx->f32[0].p, *be = (float *)ctx->f32[1].p, *r = (float *)ctx->f32[2].p,
        *u1 = (float *)ctx->f32[3].p;
  CK(cudaMemsetAsync(r, 0, b32, ctx->stream));
  CK(cudaMemsetAsync(u1, 0, b32, ctx->stream));
  // per-operation kernels, host loop (one item)
  if (ctx->nitems != 1) return fail(ctx, SRMG_ERR_UNSUPPORTED, "batched solves need the persistent engine");
  const ItemSpec &sp = specs[0];
  const double s = sp.s, k2 = sp.k2;
  const int op = sp.op;
  const Signs sg = make_signs(sp.bc);
  RC(leafnorm_dev<double>(ctx, u, b, s, op, k2, geom, 1, 1));
  RC(make_consistent(ctx, u, sg));
  RC(defect_all(ctx, be, e, u, b, s, op, k2, geom, 0));
  RC(read_small(ctx, 2));
  const double bn = ctx->h_small[1] > 0 ? ctx->h_small[1] : 1.0;
  st->bnorm = ctx->h_small[1];
  double rel = ctx->h_small[0] / bn;
  st->initial_rel = rel;
  int outer = 0, cycles = 0;
  const int inner = std::max(1, o->inner_cycles);
  double prev = rel;
  while (rel > o->tol && outer < o->max_cycles) {
    for (int i = 0; i < inner; i++) {
      RC(vcycle_mixed(ctx, e, be, r, u1, s, op, k2, geom, sg, o->ndown, o->ntop, o->nup, o->omega, tabs));
      cycles++;
    }
    for (int l = 1; l <= ctx->nlev; l++) {
      const int n = ctx->nblk_host[l - 1];
      if (!n) continue;
      k_update<<<grid_for((int64_t)n * 256, 256, 148 * 16), 256, 0, ctx->stream>>>(u, e, ctx->lv[l - 1].view(l));
      ctx->launches++;
    }
    RC(make_consistent(ctx, u, sg));
    RC(defect_all(ctx, be, e, u, b, s, op, k2, geom, 0));
    RC(read_small(ctx, 1));
    outer++;
    const double nrel = ctx->h_small[0] / bn;
    if (!std::isfinite(nrel) || (outer > 3 && nrel > 10 * prev && nrel > st->initial_rel)) {
      st->cycles = cycles;
      st->outer = outer;
      st->rel_residual = nrel;
      st->status = SRMG_ERR_DIVERGED;
      return SRMG_OK;
    }
    prev = nrel;
    rel = nrel;
  }
  st->cycles = cycles;
  st->outer = outer;
  st->rel_residual = rel;
  return SRMG_OK;
}

int srmg::solve_items(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, const ItemSpec *specs,
                      int geom, const srmg_solve_opts *opts, srmg_stats *st) {
  srmg_solve_opts o;
  if (opts) o = *opts; else srmg_solve_opts_default(&o);
  if (!(o.tol > 0) || o.max_cycles < 0 || o.ndown < 0 || o.nup < 0 || o.ntop < 0)
    return fail(ctx, SRMG_ERR_BADARG, "srmg_solve: bad options");
  for (int k = 0; k < ctx->nitems; k++) memset(&st[k], 0, sizeof(srmg_stats));
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  int rc;
  if (o.mode == SRMG_MODE_FP64 || o.mode == SRMG_MODE_FP64_DIRECT) rc = solve_fp64(ctx, u, b, nblk_alloc, specs, geom, &o, st);
  else if (o.mode == SRMG_MODE_MIXED) rc = solve_mixed(ctx, u, b, nblk_alloc, specs, geom, &o, st);
  else rc = fail(ctx, SRMG_ERR_BADARG, "unknown solve mode %d", o.mode);
  cudaEventRecord(ctx->ev1, ctx->stream);
  cudaEventSynchronize(ctx->ev1);
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  for (int k = 0; k < ctx->nitems; k++) st[k].device_ms = ms;
  if (rc) return rc;
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_solve_dev(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, double s,
                              int op, double k2, int geom, const int8_t bc[9],
                              const srmg_solve_opts *opts, srmg_stats *stats) {
  RC(check_call_any(ctx, nblk_alloc, op, geom, bc));
  if (!u || !b) return fail(ctx, SRMG_ERR_BADARG, "srmg_solve: null field");
  if (ctx->D == 3) {
    srmg_solve_opts o;
    if (opts) o = *opts; else srmg_solve_opts_default(&o);
    srmg_stats st;
    const int rc = d3_solve(ctx, u, b, nblk_alloc, s, op, k2, bc, &o, &st);
    if (stats) *stats = st;
    return rc;
  }
  const std::vector<ItemSpec> specs = uniform_items(ctx, s, op, k2, bc);
  std::vector<srmg_stats> st((size_t)ctx->nitems);
  const int rc = solve_items(ctx, u, b, nblk_alloc, specs.data(), geom, opts, st.data());
  // one set of statistics: the worst item
  srmg_stats agg = st[0];
  for (const srmg_stats &x : st) {
    agg.cycles = std::max(agg.cycles, x.cycles);
    agg.outer = std::max(agg.outer, x.outer);
    if (!(x.rel_residual <= agg.rel_residual)) agg.rel_residual = x.rel_residual;
    agg.initial_rel = std::max(agg.initial_rel, x.initial_rel);
    if (x.status) agg.status = x.status;
  }
  if (rc) agg.status = rc;
  if (stats) *stats = agg;
  if (rc) return rc;
  if (agg.status)
    return fail(ctx, agg.status, "residual is not finite after %d cycles", agg.cycles);
  return SRMG_OK;
}

extern "C" int srmg_solve(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, double s, int op,
                          double k2, int geom, const int8_t bc[9], const srmg_solve_opts *opts,
                          srmg_stats *stats) {
  RC(check_call_any(ctx, nblk_alloc, op, geom, bc));
  if (!u || !b) return fail(ctx, SRMG_ERR_BADARG, "srmg_solve: null field");
  double *du, *db;
  RC(stage_in(ctx, 0, u, nblk_alloc, &du));
  RC(stage_in(ctx, 1, b, nblk_alloc, &db));
  RC(srmg_solve_dev(ctx, du, db, nblk_alloc, s, op, k2, geom, bc, opts, stats));
  RC(stage_out(ctx, u, du, nblk_alloc));
  CK(cudaStreamSynchronize(ctx->stream));
  return SRMG_OK;
}

// ---- asynchronous host-array solve ----------------------------------------------------
// srmg_solve split at its host synchronisation: the copies of u and b in, the persistent
// solve, the copy of u out and the read-back of the solve's record are enqueued on the
// context's stream, and srmg_solve_wait finishes them.  A caller with several
// independent problems alternates two contexts on the same tree, so that one problem's
// copies overlap the other's solve.
extern "C" int srmg_solve_async(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, double s, int op,
                                double k2, int geom, const int8_t bc[9], const srmg_solve_opts *opts) {
  RC(check_call_any(ctx, nblk_alloc, op, geom, bc));
  if (!u || !b) return fail(ctx, SRMG_ERR_BADARG, "srmg_solve_async: null field");
  if (ctx->D != 2 || ctx->nitems != 1)
    return fail(ctx, SRMG_ERR_UNSUPPORTED, "srmg_solve_async: single two-dimensional trees only; use srmg_solve");
  srmg_solve_opts o;
  if (opts) o = *opts; else srmg_solve_opts_default(&o);
  if (!(o.tol > 0) || o.max_cycles < 0 || o.ndown < 0 || o.nup < 0 || o.ntop < 0)
    return fail(ctx, SRMG_ERR_BADARG, "srmg_solve_async: bad options");
  if (o.mode != SRMG_MODE_FP64 && o.mode != SRMG_MODE_MIXED && o.mode != SRMG_MODE_FP64_DIRECT)
    return fail(ctx, SRMG_ERR_BADARG, "unknown solve mode %d", o.mode);
  if (o.warm_start) return fail(ctx, SRMG_ERR_UNSUPPORTED, "srmg_solve_async: no learned warm start; use srmg_solve");
  const std::vector<ItemSpec> specs = uniform_items(ctx, s, op, k2, bc);
  if (o.mode != SRMG_MODE_FP64 && specs[0].op == SRMG_OP_LAPLACIAN4)
    return fail(ctx, SRMG_ERR_UNSUPPORTED, "mixed and direct modes support order-2 discretisations");
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  double *du, *db;
  RC(stage_in(ctx, 0, u, nblk_alloc, &du));
  RC(stage_in(ctx, 1, b, nblk_alloc, &db));
  RC(solve_reserve(ctx, nblk_alloc, o.mode));
  if (!engine_ok(ctx, &o, {du, db}))
    return fail(ctx, SRMG_ERR_UNSUPPORTED, "srmg_solve_async needs the persistent engine; use srmg_solve");
  ItemTabs tabs;
  RC(prepare_items(ctx, specs.data(), geom, o.omega, o.mode != SRMG_MODE_FP64, 0, 0.0, &tabs, direct_top(ctx)));
  RC(solve_enqueue(ctx, du, db, nblk_alloc, tabs, geom, &o));
  RC(items_host_reserve(ctx));
  RC(items_d2h(ctx));
  RC(stage_out(ctx, u, du, nblk_alloc));
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  ctx->async_pending = true;
  return SRMG_OK;
}

extern "C" int srmg_solve_wait(srmg_ctx *ctx, srmg_stats *stats) {
  if (!ctx) return SRMG_ERR_BADARG;
  if (!ctx->async_pending) return fail(ctx, SRMG_ERR_BADARG, "srmg_solve_wait: no asynchronous solve in flight");
  ctx->async_pending = false;
  CK(cudaEventSynchronize(ctx->ev1));
  RC(engine_check(ctx));
  srmg_stats st;
  memset(&st, 0, sizeof st);
  item_stats(ctx, 0, &st);
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  st.device_ms = ms;
  if (stats) *stats = st;
  if (st.status) return fail(ctx, st.status, "residual is not finite after %d cycles", st.cycles);
  return SRMG_OK;
}
