// srmg_tune.cu -- autotuner of the persistent engine's launch shape and of the
// multigrid sweep counts (no reference counterpart: the reference's cycle parameters
// are fixed inputs, src/simulate.jl:145).
//
// A trial is one complete tolerance-driven solve from the caller's initial guess on the
// caller's own problem; its cost is the device time to reach the tolerance.  The
// candidates are
//   * grid size ("engine_ctas"): one CTA per SM, or fewer CTAs (more blocks per CTA,
//     cheaper grid barriers);
//   * CTA-local coarse levels ("local_max_blocks"): how many blocks a level may hold
//     and still run inside CTA 0 with CTA barriers instead of grid barriers;
//   * sweep counts (ndown, nup): smoothing per level on the way down and up; ntop
//     only matters when the coarsest level is smoothed rather than solved directly;
//   * the relaxation factor omega of the red-black Gauss-Seidel sweeps (1, 1.1, 1.2):
//     over-relaxed smoothing contracts more per V-cycle (measured on the 1.5M-leaf
//     tree: 7 instead of 8 FP64-direct cycles at (2, 2), 9 instead of 12 at (1, 1)).
//   * mixed solves: FP32 V-cycles per defect-correction step (inner_cycles 1..4): more
//     cycles per step mean fewer FP64 update/defect passes, until the FP32 correction
//     stops contracting (measured on the 1.5M-leaf tree with the level-2 direct solve:
//     9 cycles in 3 steps, 1.97 ms, against 9 in 5, 2.16 ms, at 2 per step).
// The launch shape is tuned first at the caller's sweeps and omega (6 candidates), then
// the sweeps and omega at that shape (15 candidates), then for mixed solves the inner
// cycles at those (4 candidates).
// The tile shape is fixed by the data layout (one 20 x 20 block per 256-thread slot,
// four slots per CTA).  The fastest trial's settings are applied to the context and
// written to *opts; the caller's fields are restored after every trial.
#include <algorithm>
#include <cstring>
#include <functional>
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

struct Cand {
  int ctas, local_max, ndown, nup;
  double omega;
  int inner;
};

// Run every candidate with `solve` (which restores its own inputs), keep the fastest.
int tune(srmg_ctx *ctx, srmg_solve_opts *opts, srmg_tune_trial *trials, int max_trials,
         const std::function<int(const srmg_solve_opts &, double *ms, int *cycles, bool *ok)> &solve) {
  int nsm = 0;
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device));
  const int sweeps[][2] = {{2, 2}, {1, 1}, {1, 2}, {2, 1}, {3, 3}};
  const double omegas[] = {1.0, 1.1, 1.2};
  const int save_ctas = ctx->engine_ctas, save_lm = ctx->local_max_blocks;
  double best = 1e300;
  Cand pick{save_ctas, save_lm, opts->ndown, opts->nup, opts->omega, std::max(1, opts->inner_cycles)};
  int n = 0;
  const int nstage = opts->mode == SRMG_MODE_MIXED ? 3 : 2;
  for (int stage = 0; stage < nstage; ++stage) {
  std::vector<Cand> cands;
  if (stage == 0) {
    for (int ctas : {0, nsm / 2})
      for (int lm : {4, 16, 64}) cands.push_back({ctas, lm, opts->ndown, opts->nup, opts->omega, pick.inner});
  } else if (stage == 1) {
    for (const auto &sw : sweeps)
      for (double om : omegas) cands.push_back({pick.ctas, pick.local_max, sw[0], sw[1], om, pick.inner});
  } else {
    for (int in : {1, 2, 3, 4}) cands.push_back({pick.ctas, pick.local_max, pick.ndown, pick.nup, pick.omega, in});
  }
  for (const Cand &c : cands) {
    ctx->engine_ctas = c.ctas;
    ctx->local_max_blocks = c.local_max;
    srmg_solve_opts o = *opts;
    o.ndown = c.ndown;
    o.nup = c.nup;
    o.omega = c.omega;
    o.inner_cycles = c.inner;
    double ms = 0.0, ms2 = 0.0;
    int cyc = 0;
    bool ok = false;
    int rc = solve(o, &ms, &cyc, &ok);   // first run also sizes buffers
    if (!rc && ok) rc = solve(o, &ms2, &cyc, &ok);
    if (rc) {
      ctx->engine_ctas = save_ctas;
      ctx->local_max_blocks = save_lm;
      return rc;
    }
    const double t = std::min(ms, ms2);
    if (trials && n < max_trials) {
      srmg_tune_trial &tr = trials[n];
      tr.engine_ctas = c.ctas;
      tr.local_max_blocks = c.local_max;
      tr.ndown = c.ndown;
      tr.nup = c.nup;
      tr.ntop = o.ntop;
      tr.ms = ok ? t : -1.0;
      tr.cycles = cyc;
      tr.omega = c.omega;
      tr.inner_cycles = c.inner;
    }
    n++;
    if (ok && t < best) {
      best = t;
      pick = c;
    }
  }
  }
  ctx->engine_ctas = pick.ctas;
  ctx->local_max_blocks = pick.local_max;
  opts->ndown = pick.ndown;
  opts->nup = pick.nup;
  opts->omega = pick.omega;
  opts->inner_cycles = pick.inner;
  return n;
}

}  // namespace

extern "C" int srmg_autotune(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, double s, int op,
                             double k2, int geom, const int8_t bc[9], srmg_solve_opts *opts,
                             srmg_tune_trial *trials, int max_trials) {
  RC(check_call(ctx, nblk_alloc, op, geom, bc));
  if (!u || !b || !opts || max_trials < 0) return fail(ctx, SRMG_ERR_BADARG, "srmg_autotune: bad arguments");
  if (op == SRMG_OP_LAPLACIAN4 || ctx->has_corners)
    return fail(ctx, SRMG_ERR_UNSUPPORTED, "srmg_autotune tunes the persistent engine (StarStencil, order 2)");
  const size_t bytes = (size_t)nblk_alloc * kSS * sizeof(double);
  DevBuf u0;
  RC(ensure(ctx, u0, bytes));
  CK(cudaMemcpyAsync(u0.p, u, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  const std::vector<ItemSpec> specs = uniform_items(ctx, s, op, k2, bc);
  std::vector<srmg_stats> st((size_t)ctx->nitems);
  auto solve = [&](const srmg_solve_opts &o, double *ms, int *cycles, bool *ok) -> int {
    if (cudaMemcpyAsync(u, u0.p, bytes, cudaMemcpyDeviceToDevice, ctx->stream) != cudaSuccess)
      return fail(ctx, SRMG_ERR_CUDA, "autotune: restore of u failed");
    RC(solve_items(ctx, u, b, nblk_alloc, specs.data(), geom, &o, st.data()));
    *ms = st[0].device_ms;
    *cycles = 0;
    *ok = true;
    for (const srmg_stats &x : st) {
      *cycles = std::max(*cycles, x.cycles);
      if (x.status || !(x.rel_residual <= o.tol)) *ok = false;
    }
    return SRMG_OK;
  };
  const int n = tune(ctx, opts, trials, max_trials, solve);
  cudaMemcpyAsync(u, u0.p, bytes, cudaMemcpyDeviceToDevice, ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  cudaFree(u0.p);
  return n;
}

extern "C" int srmg_batch_autotune(srmg_ctx *ctx, double *const *u, const double *const *b, srmg_solve_opts *opts,
                                   srmg_tune_trial *trials, int max_trials) {
  if (!ctx) return SRMG_ERR_BADARG;
  if (!ctx->has_tree || (int)ctx->batch_items.size() != ctx->nitems)
    return fail(ctx, SRMG_ERR_NOTREE, "no batch: call srmg_batch_set first");
  if (!u || !b || !opts || max_trials < 0) return fail(ctx, SRMG_ERR_BADARG, "srmg_batch_autotune: bad arguments");
  cudaSetDevice(ctx->device);
  const size_t bytes = (size_t)ctx->max_blk * kSS * sizeof(double);
  DevBuf u0, fu, fb;
  RC(ensure(ctx, u0, bytes));
  RC(ensure(ctx, fu, bytes));
  RC(ensure(ctx, fb, bytes));
  for (int k = 0; k < ctx->nitems; k++) {
    const size_t off = (size_t)ctx->item_first[k] * kSS, nb = (size_t)ctx->item_nblk[k] * kSS * sizeof(double);
    CK(cudaMemcpyAsync((double *)u0.p + off, u[k], nb, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync((double *)fb.p + off, b[k], nb, cudaMemcpyDeviceToDevice, ctx->stream));
  }
  std::vector<srmg_stats> st((size_t)ctx->nitems);
  auto solve = [&](const srmg_solve_opts &o, double *ms, int *cycles, bool *ok) -> int {
    if (cudaMemcpyAsync(fu.p, u0.p, bytes, cudaMemcpyDeviceToDevice, ctx->stream) != cudaSuccess)
      return fail(ctx, SRMG_ERR_CUDA, "autotune: restore of u failed");
    RC(solve_items(ctx, (double *)fu.p, (const double *)fb.p, ctx->max_blk, ctx->batch_items.data(),
                   ctx->geom_forest, &o, st.data()));
    *ms = st[0].device_ms;
    *cycles = 0;
    *ok = true;
    for (const srmg_stats &x : st) {
      *cycles = std::max(*cycles, x.cycles);
      if (x.status || !(x.rel_residual <= o.tol)) *ok = false;
    }
    return SRMG_OK;
  };
  const int n = tune(ctx, opts, trials, max_trials, solve);
  cudaStreamSynchronize(ctx->stream);
  cudaFree(u0.p);
  cudaFree(fu.p);
  cudaFree(fb.p);
  return n;
}
