// srmg_batch.cu -- batched field solves: several independent problems (trees, and per
// tree the Poisson potential plus the photoionization Helmholtz terms) solved by one
// persistent launch over a forest.
//
// The reference solves each field with its own calls: the Poisson potential in
// src/streamer.jl:322-334 and the photoionization terms, one Helmholtz problem per
// screening constant, in src/photo.jl (the same vcycle!/fmg! entry points with a
// HelmholtzDiscretization).  Here those problems become the items of one forest: each
// item gets its own copy of its tree's blocks (block ids shifted by the item's offset),
// its operator, and its own convergence test; an item that converges is frozen while
// the others continue, so each result is the one a solo solve would give.
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

extern "C" int srmg_batch_set(srmg_ctx *ctx, int nitems, const srmg_item *items, int geom) {
  if (!ctx) return SRMG_ERR_BADARG;
  if (ctx->D != 2) return fail(ctx, SRMG_ERR_UNSUPPORTED, "srmg_batch_set: batches take two-dimensional trees");
  if (nitems < 1 || nitems > (1 << 22) || !items) return fail(ctx, SRMG_ERR_BADARG, "srmg_batch_set: bad item list");
  if (geom < 0 || geom > 2) return fail(ctx, SRMG_ERR_UNSUPPORTED, "unsupported geometry %d", geom);
  int nlev = 0;
  int64_t total = 0;
  for (int k = 0; k < nitems; k++) {
    const srmg_ctx *t = items[k].tree;
    if (t && t->D != 2)
      return fail(ctx, SRMG_ERR_UNSUPPORTED, "item %d: batches take two-dimensional trees", k);
    if (!t || !t->has_tree || t->htree.nlev < 1)
      return fail(ctx, SRMG_ERR_NOTREE, "item %d: its context holds no tree", k);
    if (items[k].op != SRMG_OP_LAPLACIAN && items[k].op != SRMG_OP_HELMHOLTZ)
      return fail(ctx, SRMG_ERR_UNSUPPORTED, "item %d: unsupported discretisation %d", k, items[k].op);
    if (t->has_corners)
      return fail(ctx, SRMG_ERR_UNSUPPORTED, "item %d: batches need a StarStencil connectivity", k);
    for (int i = 0; i < 9; i++)
      if (items[k].bc[i] < -1 || items[k].bc[i] > 1)
        return fail(ctx, SRMG_ERR_BADARG, "item %d: boundary table entries must be -1, 0 or 1", k);
    nlev = std::max(nlev, t->htree.nlev);
    total += t->htree.max_blk;
  }
  if (total >= INT32_MAX / 8) return fail(ctx, SRMG_ERR_BADARG, "forest of %lld blocks is too large", (long long)total);
  HostTree f;
  f.nlev = nlev;
  f.max_blk = total;
  f.pairs.assign(nlev, {});
  f.nb.assign(nlev, {});
  f.bd.assign(nlev, {});
  f.rb.assign(nlev, {});
  f.ch.assign(nlev, {});
  std::vector<int> item_of((size_t)total + 1, 0);
  std::vector<int64_t> first(nitems), nblk(nitems);
  int64_t off = 0;
  for (int k = 0; k < nitems; k++) {
    const HostTree &t = items[k].tree->htree;
    first[k] = off;
    nblk[k] = t.max_blk;
    for (int64_t b = 1; b <= t.max_blk; b++) item_of[off + b] = k;
    for (int l = 0; l < t.nlev; l++) {
      for (srmg_pair p : t.pairs[l]) {
        p.blk += off;
        f.pairs[l].push_back(p);
      }
      for (srmg_neighbor e : t.nb[l]) {
        e.from += off;
        e.to += off;
        f.nb[l].push_back(e);
      }
      for (srmg_boundary e : t.bd[l]) {
        e.block += off;
        f.bd[l].push_back(e);
      }
      for (srmg_refbnd e : t.rb[l]) {
        e.fine += off;
        e.coarse += off;
        f.rb[l].push_back(e);
      }
      for (srmg_child e : t.ch[l]) {
        e.fine += off;
        e.coarse += off;
        f.ch[l].push_back(e);
      }
    }
    off += t.max_blk;
  }
  std::vector<int64_t> np(nlev), nn(nlev), nd(nlev), nr(nlev), nc(nlev);
  std::vector<const srmg_pair *> pp(nlev);
  std::vector<const srmg_neighbor *> pn(nlev);
  std::vector<const srmg_boundary *> pd(nlev);
  std::vector<const srmg_refbnd *> pr(nlev);
  std::vector<const srmg_child *> pc(nlev);
  for (int l = 0; l < nlev; l++) {
    np[l] = f.pairs[l].size();
    pp[l] = f.pairs[l].data();
    nn[l] = f.nb[l].size();
    pn[l] = f.nb[l].data();
    nd[l] = f.bd[l].size();
    pd[l] = f.bd[l].data();
    nr[l] = f.rb[l].size();
    pr[l] = f.rb[l].data();
    nc[l] = f.ch[l].size();
    pc[l] = f.ch[l].data();
  }
  if (ctx->graph_exec) {
    cudaGraphExecDestroy(ctx->graph_exec);
    ctx->graph_exec = nullptr;
    ctx->graph_key.clear();
  }
  RC(build_tree(ctx, nlev, np.data(), pp.data(), nn.data(), pn.data(), nd.data(), pd.data(), nr.data(), pr.data(),
                nc.data(), pc.data(), ctx->generation + 1, &item_of, nitems));
  ctx->htree = std::move(f);
  ctx->item_first = first;
  ctx->item_nblk = nblk;
  ctx->batch_items.assign(nitems, ItemSpec());
  for (int k = 0; k < nitems; k++) {
    ItemSpec &sp = ctx->batch_items[k];
    sp.s = items[k].s;
    sp.op = items[k].op;
    sp.k2 = items[k].k2;
    memcpy(sp.bc, items[k].bc, 9);
  }
  ctx->geom_forest = geom;
  return SRMG_OK;
}

extern "C" int srmg_batch_items(const srmg_ctx *ctx) {
  if (!ctx) return SRMG_ERR_BADARG;
  return ctx->has_tree ? ctx->nitems : 0;
}

extern "C" int64_t srmg_batch_offset(const srmg_ctx *ctx, int item) {
  if (!ctx || !ctx->has_tree || item < 0 || item >= (int)ctx->item_first.size()) return -1;
  return ctx->item_first[item];
}

extern "C" int64_t srmg_batch_nblk(const srmg_ctx *ctx, int item) {
  if (!ctx || !ctx->has_tree || item < 0 || item >= (int)ctx->item_nblk.size()) return -1;
  return ctx->item_nblk[item];
}

static int batch_check(srmg_ctx *ctx) {
  if (!ctx) return SRMG_ERR_BADARG;
  if (!ctx->has_tree || ctx->batch_items.empty() || (int)ctx->batch_items.size() != ctx->nitems)
    return fail(ctx, SRMG_ERR_NOTREE, "no batch: call srmg_batch_set first");
  cudaSetDevice(ctx->device);
  return SRMG_OK;
}

static int opts_of(srmg_ctx *ctx, const srmg_solve_opts *opts, srmg_solve_opts *o) {
  if (opts) *o = *opts; else srmg_solve_opts_default(o);
  if (!(o->tol > 0) || o->max_cycles < 0 || o->ndown < 0 || o->nup < 0 || o->ntop < 0)
    return fail(ctx, SRMG_ERR_BADARG, "srmg_batch_solve: bad options");
  if (o->mode != SRMG_MODE_FP64 && o->mode != SRMG_MODE_MIXED && o->mode != SRMG_MODE_FP64_DIRECT)
    return fail(ctx, SRMG_ERR_BADARG, "unknown solve mode %d", o->mode);
  return SRMG_OK;
}

static int stats_status(srmg_ctx *ctx, const srmg_stats *st) {
  for (int k = 0; k < ctx->nitems; k++)
    if (st[k].status) return fail(ctx, st[k].status, "item %d: residual is not finite after %d cycles", k, st[k].cycles);
  return SRMG_OK;
}

extern "C" int srmg_batch_solve_forest_dev(srmg_ctx *ctx, double *u, const double *b, const srmg_solve_opts *opts,
                                           srmg_stats *stats) {
  RC(batch_check(ctx));
  if (!u || !b || !stats) return fail(ctx, SRMG_ERR_BADARG, "srmg_batch_solve_forest_dev: null argument");
  RC(solve_items(ctx, u, b, ctx->max_blk, ctx->batch_items.data(), ctx->geom_forest, opts, stats));
  return stats_status(ctx, stats);
}

// Gather the items' fields into the forest layout, solve, scatter u back.  Host
// pointers when `host`; every copy is one cudaMemcpyAsync per item and field.
static int gather(srmg_ctx *ctx, double *fu, double *fb, double *const *u, const double *const *b, bool host) {
  const cudaMemcpyKind kind = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  for (int k = 0; k < ctx->nitems; k++) {
    const size_t off = (size_t)ctx->item_first[k] * kSS, bytes = (size_t)ctx->item_nblk[k] * kSS * sizeof(double);
    CK(cudaMemcpyAsync(fu + off, u[k], bytes, kind, ctx->stream));
    CK(cudaMemcpyAsync(fb + off, b[k], bytes, kind, ctx->stream));
  }
  return SRMG_OK;
}

static int scatter(srmg_ctx *ctx, double *const *u, const double *fu, bool host) {
  const cudaMemcpyKind kind = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  for (int k = 0; k < ctx->nitems; k++) {
    const size_t off = (size_t)ctx->item_first[k] * kSS, bytes = (size_t)ctx->item_nblk[k] * kSS * sizeof(double);
    CK(cudaMemcpyAsync(u[k], fu + off, bytes, kind, ctx->stream));
  }
  return SRMG_OK;
}

// Everything a captured sequence depends on: the callers' pointers, the options, the
// work buffers and the item tables.
static std::vector<const void *> graph_key_of(srmg_ctx *ctx, double *const *u, const double *const *b,
                                              const srmg_solve_opts &o) {
  std::vector<const void *> k;
  for (int i = 0; i < ctx->nitems; i++) {
    k.push_back(u[i]);
    k.push_back(b[i]);
  }
  const size_t nw = (sizeof o + sizeof(void *) - 1) / sizeof(void *);
  std::vector<const void *> ob(nw, nullptr);
  memcpy(ob.data(), &o, sizeof o);
  k.insert(k.end(), ob.begin(), ob.end());
  for (auto &x : ctx->f64) k.push_back(x.p);
  for (auto &x : ctx->f32) k.push_back(x.p);
  for (auto &x : ctx->forest) k.push_back(x.p);
  k.push_back(ctx->part.p);
  k.push_back(ctx->istat.p);
  k.push_back(ctx->sync.p);
  k.push_back(ctx->it_tab.p);
  k.push_back(ctx->h_items);
  k.push_back((const void *)ctx->stream);
  const size_t nt = (ctx->it_tab_host.size() + sizeof(void *) - 1) / sizeof(void *);
  std::vector<const void *> tb(nt, nullptr);
  memcpy(tb.data(), ctx->it_tab_host.data(), ctx->it_tab_host.size());
  k.insert(k.end(), tb.begin(), tb.end());
  k.push_back((const void *)(intptr_t)ctx->engine_ctas);
  k.push_back((const void *)(intptr_t)ctx->engine_threads);
  k.push_back((const void *)(intptr_t)ctx->local_max_blocks);
  k.push_back((const void *)(intptr_t)ctx->trace_on);
  return k;
}

static int batch_solve(srmg_ctx *ctx, double *const *u, const double *const *b, const srmg_solve_opts *opts,
                       srmg_stats *stats, bool host) {
  RC(batch_check(ctx));
  if (!u || !b || !stats) return fail(ctx, SRMG_ERR_BADARG, "srmg_batch_solve: null argument");
  for (int k = 0; k < ctx->nitems; k++)
    if (!u[k] || !b[k]) return fail(ctx, SRMG_ERR_BADARG, "srmg_batch_solve: null field of item %d", k);
  srmg_solve_opts o;
  RC(opts_of(ctx, opts, &o));
  const size_t bytes = (size_t)ctx->max_blk * kSS * sizeof(double);
  RC(ensure(ctx, ctx->forest[0], bytes));
  RC(ensure(ctx, ctx->forest[1], bytes));
  double *fu = (double *)ctx->forest[0].p, *fb = (double *)ctx->forest[1].p;
  const bool graph = ctx->use_graph && !host && engine_ok(ctx, &o, {fu, fb});
  if (!graph) {
    RC(gather(ctx, fu, fb, u, b, host));
    RC(solve_items(ctx, fu, fb, ctx->max_blk, ctx->batch_items.data(), ctx->geom_forest, &o, stats));
    RC(scatter(ctx, u, fu, host));
    CK(cudaStreamSynchronize(ctx->stream));
    return stats_status(ctx, stats);
  }
  // CUDA graph: gathers, the persistent solve, the result copy and the scatters are
  // captured once per key and replayed.
  ItemTabs tabs;
  RC(prepare_items(ctx, ctx->batch_items.data(), ctx->geom_forest, o.omega, o.mode != SRMG_MODE_FP64, 0, 0.0,
                   &tabs));
  RC(solve_reserve(ctx, ctx->max_blk, o.mode));
  RC(items_host_reserve(ctx));
  std::vector<const void *> key = graph_key_of(ctx, u, b, o);
  if (!ctx->graph_exec || key != ctx->graph_key) {
    // one eager run sizes every buffer, then the capture
    RC(gather(ctx, fu, fb, u, b, false));
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    RC(solve_enqueue(ctx, fu, fb, ctx->max_blk, tabs, ctx->geom_forest, &o));
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    RC(read_items(ctx));
    RC(scatter(ctx, u, fu, false));
    CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    items_stats(ctx, &o, stats);
    for (int k = 0; k < ctx->nitems; k++) stats[k].device_ms = ms;
    key = graph_key_of(ctx, u, b, o);
    if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
    ctx->graph_exec = nullptr;
    ctx->graph_key.clear();
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
    int rc = gather(ctx, fu, fb, u, b, false);
    if (!rc) rc = solve_enqueue(ctx, fu, fb, ctx->max_blk, tabs, ctx->geom_forest, &o);
    if (!rc) rc = items_d2h(ctx);
    if (!rc) rc = scatter(ctx, u, fu, false);
    const cudaError_t ec = cudaStreamEndCapture(ctx->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    CK(ec);
    const cudaError_t ei = cudaGraphInstantiate(&ctx->graph_exec, g, 0);
    cudaGraphDestroy(g);
    CK(ei);
    ctx->graph_key = key;
    return stats_status(ctx, stats);
  }
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  CK(cudaGraphLaunch(ctx->graph_exec, ctx->stream));
  ctx->launches += 1;
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  RC(engine_check(ctx));
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  items_stats(ctx, &o, stats);
  for (int k = 0; k < ctx->nitems; k++) stats[k].device_ms = ms;
  return stats_status(ctx, stats);
}

extern "C" int srmg_batch_solve_dev(srmg_ctx *ctx, double *const *u, const double *const *b,
                                    const srmg_solve_opts *opts, srmg_stats *stats) {
  return batch_solve(ctx, u, b, opts, stats, false);
}

extern "C" int srmg_batch_solve(srmg_ctx *ctx, double *const *u, const double *const *b, const srmg_solve_opts *opts,
                                srmg_stats *stats) {
  return batch_solve(ctx, u, b, opts, stats, true);
}
