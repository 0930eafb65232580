// srmg.cu -- C ABI of libsrmg: context, tree upload and validation, and the FP64
// reference-semantics multigrid (vcycle!/fmg!/resnorm!) on device fields.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <unordered_map>
#include <vector>

#include "srmg_ctx.h"
#include "srmg_internal.h"
#include "srmg_seq.cuh"

using namespace srmg;

// ------------------------------------------------------------------ error plumbing

int srmg::fail(srmg_ctx *c, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

int srmg::cuda_check(srmg_ctx *c, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return SRMG_OK;
  return fail(c, SRMG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

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

int srmg::ensure(srmg_ctx *ctx, DevBuf &b, size_t bytes) {
  if (b.bytes >= bytes) return SRMG_OK;
  if (b.p) {
    cudaStreamSynchronize(ctx->stream);
    cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
  }
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e != cudaSuccess) return fail(ctx, SRMG_ERR_NOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  b.bytes = bytes;
  return SRMG_OK;
}

// ------------------------------------------------------------------ context

extern "C" int srmg_create(srmg_ctx **out, int D, int M, int G, int device) {
  if (!out) return SRMG_ERR_BADARG;
  *out = nullptr;
  if ((D != 2 && D != 3) || M != kM || G != kG) return SRMG_ERR_UNSUPPORTED;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return SRMG_ERR_CUDA;
  srmg_ctx *ctx = new srmg_ctx();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess ||
      cudaMallocHost((void **)&ctx->h_small, 64 * sizeof(double)) != cudaSuccess) {
    delete ctx;
    return SRMG_ERR_CUDA;
  }
  ctx->stream = ctx->own_stream;
  ctx->D = D;
  if (ensure(ctx, ctx->small, 64 * sizeof(double))) {
    delete ctx;
    return SRMG_ERR_NOMEM;
  }
  *out = ctx;
  return SRMG_OK;
}

void srmg::drop_op_graphs(srmg_ctx *ctx) {
  for (auto &q : ctx->op_seqs)
    if (q.ops.p) cudaFree(q.ops.p);
  ctx->op_seqs.clear();
  for (auto &g : ctx->op_graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  ctx->op_graphs.clear();
}

void srmg::free_tree(srmg_ctx *ctx) {
  drop_op_graphs(ctx);
  if (ctx->d_tree) cudaFree(ctx->d_tree);
  ctx->d_tree = nullptr;
  ctx->lv.clear();
  ctx->lv3.clear();
  ctx->nblk_host.clear();
  ctx->nch_host.clear();
  ctx->has_tree = false;
  ctx->fbc_built = false;
  if (ctx->push_tab.p) cudaFree(ctx->push_tab.p);
  ctx->push_tab = DevBuf{};
  ctx->push_lv.clear();
  ctx->push_state = 0;
}

extern "C" void srmg_destroy(srmg_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  free_tree(ctx);
  for (auto &b : ctx->f64) if (b.p) cudaFree(b.p);
  for (auto &b : ctx->f32) if (b.p) cudaFree(b.p);
  if (ctx->part.p) cudaFree(ctx->part.p);
  if (ctx->small.p) cudaFree(ctx->small.p);
  for (auto &kv : ctx->coarse_cache) cudaFree(kv.second.p);
  if (ctx->it_tab.p) cudaFree(ctx->it_tab.p);
  if (ctx->istat.p) cudaFree(ctx->istat.p);
  if (ctx->h_items) cudaFreeHost(ctx->h_items);
  if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
  drop_op_graphs(ctx);
  for (auto &b : ctx->forest) if (b.p) cudaFree(b.p);
  for (auto &b : ctx->cnn_work) if (b.p) cudaFree(b.p);
  if (ctx->sync.p) cudaFree(ctx->sync.p);
  if (ctx->trace.p) cudaFree(ctx->trace.p);
  if (ctx->fbc.p) cudaFree(ctx->fbc.p);
  if (ctx->fbc_tabs.p) cudaFree(ctx->fbc_tabs.p);
  if (ctx->h_small) cudaFreeHost(ctx->h_small);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  for (auto &r : ctx->host_reg) cudaHostUnregister(r.first);
  delete ctx;
}

// Page-lock a caller's host range so that the host-array entry points copy it by DMA
// at full bandwidth (a pageable range is staged through a driver buffer).  The range
// stays registered until srmg_host_unregister or srmg_destroy; the caller must not free
// it before.
extern "C" int srmg_host_register(srmg_ctx *ctx, void *ptr, int64_t bytes) {
  if (!ctx) return SRMG_ERR_BADARG;
  if (!ptr || bytes <= 0) return fail(ctx, SRMG_ERR_BADARG, "srmg_host_register: null range");
  for (auto &r : ctx->host_reg)
    if (r.first == ptr) {
      if (r.second == (size_t)bytes) return SRMG_OK;
      return fail(ctx, SRMG_ERR_BADARG, "srmg_host_register: %p already registered with another size", ptr);
    }
  CK(cudaSetDevice(ctx->device));
  CK(cudaHostRegister(ptr, (size_t)bytes, cudaHostRegisterDefault));
  ctx->host_reg.emplace_back(ptr, (size_t)bytes);
  return SRMG_OK;
}

extern "C" int srmg_host_unregister(srmg_ctx *ctx, void *ptr) {
  if (!ctx) return SRMG_ERR_BADARG;
  for (size_t k = 0; k < ctx->host_reg.size(); k++)
    if (ctx->host_reg[k].first == ptr) {
      CK(cudaSetDevice(ctx->device));
      const cudaError_t e = cudaHostUnregister(ptr);
      ctx->host_reg.erase(ctx->host_reg.begin() + k);
      if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, SRMG_ERR_CUDA, "srmg_host_unregister: %s", cudaGetErrorString(e));
      }
      return SRMG_OK;
    }
  return fail(ctx, SRMG_ERR_BADARG, "srmg_host_unregister: %p was not registered", ptr);
}

extern "C" const char *srmg_last_error(const srmg_ctx *ctx) {
  return ctx ? ctx->err.c_str() : "null context";
}

extern "C" int srmg_set_stream(srmg_ctx *ctx, void *s) {
  if (!ctx) return SRMG_ERR_BADARG;
  if (ctx->async_pending)
    return fail(ctx, SRMG_ERR_BADARG, "an asynchronous solve is in flight on this context: call srmg_solve_wait first");
  ctx->stream = s ? (cudaStream_t)s : ctx->own_stream;
  return SRMG_OK;
}

extern "C" int srmg_synchronize(srmg_ctx *ctx) {
  if (!ctx) return SRMG_ERR_BADARG;
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->stream));
  return engine_check(ctx);
}

extern "C" int64_t srmg_launch_count(const srmg_ctx *ctx) { return ctx ? ctx->launches : -1; }
extern "C" uint64_t srmg_tree_generation(const srmg_ctx *ctx) { return ctx ? ctx->generation : 0; }

// ------------------------------------------------------------------ tree upload

static int face_of(const int64_t f[2]) {
  if (f[0] == -1 && f[1] == 0) return 0;
  if (f[0] == 1 && f[1] == 0) return 1;
  if (f[0] == 0 && f[1] == -1) return 2;
  if (f[0] == 0 && f[1] == 1) return 3;
  return -1;
}

// Corner index of a diagonal direction (both components +-1), else -1:
// q = (fr + 1) / 2 + 2 (fz + 1) / 2.
static int corner_of(const int64_t f[2]) {
  if ((f[0] != -1 && f[0] != 1) || (f[1] != -1 && f[1] != 1)) return -1;
  return (int)((f[0] + 1) / 2 + 2 * ((f[1] + 1) / 2));
}

// Validate and upload a tree (or a forest: item_of[blk] gives the item of every 1-based
// block id, each item's blocks contiguous within every level's list).
int srmg::build_tree(srmg_ctx *ctx, int nlev, const int64_t *npairs, const srmg_pair *const *pairs,
                     const int64_t *nnb, const srmg_neighbor *const *nb, const int64_t *nbd,
                     const srmg_boundary *const *bd, const int64_t *nrb, const srmg_refbnd *const *rb,
                     const int64_t *nch, const srmg_child *const *ch, uint64_t generation,
                     const std::vector<int> *item_of, int nitems) {
  if (!ctx) return SRMG_ERR_BADARG;
  if (ctx->D != 2) return fail(ctx, SRMG_ERR_BADARG, "a context created with D = 3 takes srmg_set_tree3");
  if (nlev < 1 || nlev > 30 || !npairs || !pairs || !nnb || !nb || !nbd || !bd || !nrb || !rb ||
      !nch || !ch)
    return fail(ctx, SRMG_ERR_BADARG, "srmg_set_tree: bad level count or null arrays");
  cudaSetDevice(ctx->device);

  // blk (1-based) -> (level, index within level)
  int64_t max_blk = 0, max_coord = 1;
  for (int l = 0; l < nlev; l++) {
    if (npairs[l] < 0 || (npairs[l] > 0 && !pairs[l]) || npairs[l] > (int64_t)INT32_MAX / 8)
      return fail(ctx, SRMG_ERR_BADTREE, "level %d: bad block count", l + 1);
    for (int64_t p = 0; p < npairs[l]; p++) {
      const srmg_pair &pr = pairs[l][p];
      if (pr.blk < 1 || pr.blk >= INT32_MAX)
        return fail(ctx, SRMG_ERR_BADTREE, "level %d: block index %lld out of range", l + 1,
                    (long long)pr.blk);
      if (pr.coord[0] < 1 || pr.coord[1] < 1 || pr.coord[0] > (1 << 24) || pr.coord[1] > (1 << 24))
        return fail(ctx, SRMG_ERR_BADTREE, "level %d: block coordinate out of range", l + 1);
      max_blk = std::max(max_blk, pr.blk);
      max_coord = std::max(max_coord, std::max(pr.coord[0], pr.coord[1]));
    }
  }
  std::vector<int> lev_of(max_blk + 1, 0), idx_of(max_blk + 1, -1);
  std::vector<int2> coord_of(max_blk + 1, make_int2(0, 0));
  for (int l = 0; l < nlev; l++)
    for (int64_t p = 0; p < npairs[l]; p++) {
      const srmg_pair &pr = pairs[l][p];
      if (lev_of[pr.blk] != 0)
        return fail(ctx, SRMG_ERR_BADTREE, "block %lld appears twice in the tree", (long long)pr.blk);
      lev_of[pr.blk] = l + 1;
      idx_of[pr.blk] = (int)p;
      coord_of[pr.blk] = make_int2((int)pr.coord[0], (int)pr.coord[1]);
    }
  auto at_level = [&](int64_t blk, int l) {
    return blk >= 1 && blk <= max_blk && lev_of[blk] == l;
  };

  std::vector<int4> binfo(max_blk + 1, make_int4(0, 0, 0, 0));
  std::vector<int4> bface(4 * (max_blk + 1), make_int4(FACE_NONE, 0, 0, -1));
  std::vector<int4> bkids(max_blk + 1, make_int4(-1, -1, -1, -1));
  std::vector<std::vector<int4>> hb(nlev), hf(nlev), hc(nlev), hcf(nlev);
  bool corners = false;
  for (int l = 0; l < nlev; l++) {
    const int lv = l + 1;
    hb[l].resize(npairs[l]);
    hf[l].assign(4 * npairs[l], make_int4(FACE_NONE, 0, 0, 0));
    hcf[l].assign(4 * npairs[l], make_int4(FACE_NONE, 0, 0, 0));
    for (int64_t p = 0; p < npairs[l]; p++) {
      const srmg_pair &pr = pairs[l][p];
      hb[l][p] = make_int4((int)(pr.blk - 1), (int)pr.coord[0], (int)pr.coord[1], 0);
    }
    auto set_face = [&](int64_t blk, int face, int4 v) -> int {
      int4 &slot = hf[l][4 * idx_of[blk] + face];
      if (slot.x != FACE_NONE)
        return fail(ctx, SRMG_ERR_BADTREE, "level %d: ghost face %d of block %lld written by two edges",
                    lv, face, (long long)blk);
      slot = v;
      return SRMG_OK;
    };
    // diagonal edges of a BoxStencil connectivity: the 2 x 2 corner ghosts
    auto set_corner = [&](int64_t blk, int q, int4 v) -> int {
      int4 &slot = hcf[l][4 * idx_of[blk] + q];
      if (slot.x != FACE_NONE)
        return fail(ctx, SRMG_ERR_BADTREE, "level %d: corner %d of block %lld written by two edges",
                    lv, q, (long long)blk);
      slot = v;
      corners = true;
      return SRMG_OK;
    };
    if (nnb[l] < 0 || (nnb[l] > 0 && !nb[l])) return fail(ctx, SRMG_ERR_BADTREE, "level %d: neighbours", lv);
    for (int64_t k = 0; k < nnb[l]; k++) {
      const srmg_neighbor &e = nb[l][k];
      const int64_t mf[2] = {-e.face[0], -e.face[1]};
      const int f = face_of(mf);
      if (!at_level(e.from, lv) || !at_level(e.to, lv))
        return fail(ctx, SRMG_ERR_BADTREE, "level %d: neighbour edge %lld->%lld not on this level", lv,
                    (long long)e.from, (long long)e.to);
      if (f < 0) {
        const int q = corner_of(mf);
        if (q < 0) return fail(ctx, SRMG_ERR_UNSUPPORTED, "level %d: neighbour face is not a box direction", lv);
        RC(set_corner(e.to, q, make_int4(FACE_NEIGHBOR, (int)(e.from - 1), 0, 0)));
        continue;
      }
      RC(set_face(e.to, f, make_int4(FACE_NEIGHBOR, (int)(e.from - 1), 0, 0)));
      {
        int4 &pf = bface[4 * (e.to - 1) + f];
        pf.x = FACE_NEIGHBOR;
        pf.y = (int)(e.from - 1);
        const int fp = face_of(e.face);
        if (bface[4 * (e.from - 1) + fp].w >= 0)
          return fail(ctx, SRMG_ERR_BADTREE, "level %d: block %lld has two neighbours across one face", lv,
                      (long long)e.from);
        bface[4 * (e.from - 1) + fp].w = (int)(e.to - 1);
      }
    }
    if (nbd[l] < 0 || (nbd[l] > 0 && !bd[l])) return fail(ctx, SRMG_ERR_BADTREE, "level %d: boundaries", lv);
    for (int64_t k = 0; k < nbd[l]; k++) {
      const srmg_boundary &e = bd[l][k];
      const int f = face_of(e.face);
      if (!at_level(e.block, lv) || e.level != lv)
        return fail(ctx, SRMG_ERR_BADTREE, "level %d: boundary edge of block %lld not on this level",
                    lv, (long long)e.block);
      if (f < 0) {
        // a diagonal step leaves the domain along bnd's nonzero components
        const int q = corner_of(e.face);
        if (q < 0 || (e.bnd[0] != 0 && e.bnd[0] != e.face[0]) || (e.bnd[1] != 0 && e.bnd[1] != e.face[1]) ||
            (e.bnd[0] == 0 && e.bnd[1] == 0))
          return fail(ctx, SRMG_ERR_UNSUPPORTED, "level %d: malformed boundary corner", lv);
        RC(set_corner(e.block, q, make_int4(FACE_BOUNDARY, 0, (int)e.bnd[0], (int)e.bnd[1])));
        continue;
      }
      if (e.bnd[0] != e.face[0] || e.bnd[1] != e.face[1])
        return fail(ctx, SRMG_ERR_UNSUPPORTED, "level %d: boundary edge is not a star face", lv);
      RC(set_face(e.block, f, make_int4(FACE_BOUNDARY, 0, 0, 0)));
      bface[4 * (e.block - 1) + f].x = FACE_BOUNDARY;
    }
    if (nrb[l] < 0 || (nrb[l] > 0 && !rb[l])) return fail(ctx, SRMG_ERR_BADTREE, "level %d: refboundaries", lv);
    for (int64_t k = 0; k < nrb[l]; k++) {
      const srmg_refbnd &e = rb[l][k];
      const int f = face_of(e.face);
      if (lv < 2 || !at_level(e.fine, lv) || !at_level(e.coarse, lv - 1) || e.subblock[0] < 1 ||
          e.subblock[0] > 2 || e.subblock[1] < 1 || e.subblock[1] > 2)
        return fail(ctx, SRMG_ERR_BADTREE, "level %d: malformed refinement boundary %lld/%lld", lv,
                    (long long)e.fine, (long long)e.coarse);
      if (f < 0) {
        const int q = corner_of(e.face);
        if (q < 0) return fail(ctx, SRMG_ERR_UNSUPPORTED, "level %d: refinement face is not a box direction", lv);
        RC(set_corner(e.fine, q, make_int4(FACE_REFBND, (int)(e.coarse - 1), (int)e.subblock[0],
                                           (int)e.subblock[1])));
        continue;
      }
      RC(set_face(e.fine, f, make_int4(FACE_REFBND, (int)(e.coarse - 1), (int)e.subblock[0],
                                       (int)e.subblock[1])));
      {
        int4 &pf = bface[4 * (e.fine - 1) + f];
        pf.x = FACE_REFBND;
        pf.y = (int)(e.coarse - 1);
        pf.z = (int)e.subblock[0] | ((int)e.subblock[1] << 8);
      }
    }
    if (nch[l] < 0 || (nch[l] > 0 && !ch[l])) return fail(ctx, SRMG_ERR_BADTREE, "level %d: children", lv);
    hc[l].resize(nch[l]);
    for (int64_t k = 0; k < nch[l]; k++) {
      const srmg_child &e = ch[l][k];
      if (lv < 2 || !at_level(e.fine, lv) || !at_level(e.coarse, lv - 1) || e.subblock[0] < 1 ||
          e.subblock[0] > 2 || e.subblock[1] < 1 || e.subblock[1] > 2)
        return fail(ctx, SRMG_ERR_BADTREE, "level %d: malformed child edge %lld/%lld", lv,
                    (long long)e.fine, (long long)e.coarse);
      hc[l][k] = make_int4((int)(e.fine - 1), (int)(e.coarse - 1), (int)e.subblock[0], (int)e.subblock[1]);
      int4 &cb = hb[l - 1][idx_of[e.coarse]];
      const int bit = 1 << ((int)(e.subblock[0] - 1) + 2 * (int)(e.subblock[1] - 1));
      if (cb.w & bit)
        return fail(ctx, SRMG_ERR_BADTREE, "level %d: two children cover one subblock of block %lld",
                    lv, (long long)e.coarse);
      cb.w |= bit;
      const int sub = (int)(e.subblock[0] - 1) + 2 * (int)(e.subblock[1] - 1);
      int4 &kd = bkids[e.coarse - 1];
      (sub == 0 ? kd.x : sub == 1 ? kd.y : sub == 2 ? kd.z : kd.w) = (int)(e.fine - 1);
    }
  }

  // items: per level, each item's blocks must form one contiguous run of the list
  if (nitems < 1 || (item_of && (int64_t)item_of->size() < max_blk + 1))
    return fail(ctx, SRMG_ERR_BADARG, "bad item table");
  std::vector<int2> lrange((size_t)nitems * nlev, make_int2(0, 0));
  for (int l = 0; l < nlev; l++) {
    int prev = -1;
    std::vector<char> seen(nitems, 0);
    for (size_t i = 0; i < hb[l].size(); i++) {
      int4 &b4 = hb[l][i];
      const int it = item_of ? (*item_of)[b4.x + 1] : 0;
      if (it < 0 || it >= nitems) return fail(ctx, SRMG_ERR_BADARG, "block %d: item out of range", b4.x + 1);
      if (it != prev) {
        if (seen[it]) return fail(ctx, SRMG_ERR_BADTREE, "level %d: blocks of item %d are not contiguous", l + 1, it);
        seen[it] = 1;
        lrange[(size_t)it * nlev + l] = make_int2((int)i, 0);
        prev = it;
      }
      lrange[(size_t)it * nlev + l].y++;
      b4.w |= it << 8;  // the item rides in bits 8.. of the child-mask word
    }
  }
  if (item_of)
    for (int l = 0; l < nlev; l++)
      for (const int4 &e : hc[l])
        if ((*item_of)[e.x + 1] != (*item_of)[e.y + 1])
          return fail(ctx, SRMG_ERR_BADTREE, "level %d: child edge between two items", l + 1);
  // norm chunks: up to kNormChunk consecutive blocks of one item on one level, ordered
  // by item, then level, then position, so that every item's chunks are contiguous
  std::vector<int4> chunks;
  std::vector<int2> itch(nitems);
  for (int it = 0; it < nitems; it++) {
    itch[it].x = (int)chunks.size();
    for (int l = 0; l < nlev; l++) {
      const int2 rg = lrange[(size_t)it * nlev + l];
      for (int q = 0; q < rg.y; q += kNormChunk)
        chunks.push_back(make_int4(l + 1, rg.x + q, std::min(kNormChunk, rg.y - q), it));
    }
    itch[it].y = (int)chunks.size() - itch[it].x;
  }
  // blocks holding at least one leaf cell, with their level (learned warm start)
  std::vector<int2> leafblk;
  for (int l = 0; l < nlev; l++)
    for (const int4 &b4 : hb[l])
      if ((b4.w & 15) != 15) leafblk.push_back(make_int2(b4.x, l + 1));
  for (int l = 0; l < nlev; l++)
    for (const int4 &b4 : hb[l]) binfo[b4.x] = make_int4(b4.y, b4.z, b4.w, l + 1);
  for (int64_t b = 0; b < max_blk; b++)
    for (int f = 0; f < 4; f++) {
      int4 &fc = bface[4 * b + f];
      if (fc.x == FACE_NEIGHBOR) {
        fc.z = binfo[fc.y].z & 15;  // the neighbour's child mask
        if (binfo[fc.y].z >> 8 != binfo[b].z >> 8)
          return fail(ctx, SRMG_ERR_BADTREE, "neighbour edge between two items");
      }
    }
  std::vector<std::vector<int4>> hr(nlev);
  for (int l = 0; l < nlev; l++) {
    hr[l].resize(5 * hb[l].size());
    for (size_t i = 0; i < hb[l].size(); i++) {
      hr[l][5 * i] = hb[l][i];
      for (int f = 0; f < 4; f++) hr[l][5 * i + 1 + f] = bface[4 * hb[l][i].x + f];
    }
  }

  // radial weight tables, 1-based global index i in [1, 16*max_coord]
  const int wn = (int)(kM * max_coord + 2);
  std::vector<double> wm(wn, 0.0), wp(wn, 0.0);
  std::vector<float> wm32(wn, 0.f), wp32(wn, 0.f);
  for (int i = 1; i < wn; i++) {
    wm[i] = (double)(2 * (int64_t)i - 2) / (double)(2 * (int64_t)i - 1);
    wp[i] = (double)(2 * (int64_t)i) / (double)(2 * (int64_t)i - 1);
    wm32[i] = (float)wm[i];
    wp32[i] = (float)wp[i];
  }

  // The same tables as rows per block coordinate c (geometry 1: the block's r
  // coordinate, geometry 2: its z coordinate): row c holds wm, then wp, at the 20 tile
  // positions k = 0..19 (global index i = k - 1 + 16 (c - 1)), zero where i falls
  // outside the table.  The engine copies one row per block with the block's tiles.
  const int nwrow = (int)max_coord + 1;
  std::vector<double> wrow(2 * kS * (size_t)nwrow, 0.0);
  std::vector<float> wrow32(2 * kS * (size_t)nwrow, 0.f);
  for (int c = 1; c < nwrow; c++)
    for (int k = 0; k < kS; k++) {
      const int64_t i = k - 1 + (int64_t)kM * (c - 1);
      if (i < 0 || i >= wn) continue;
      wrow[2 * kS * (size_t)c + k] = wm[i];
      wrow[2 * kS * (size_t)c + kS + k] = wp[i];
      wrow32[2 * kS * (size_t)c + k] = wm32[i];
      wrow32[2 * kS * (size_t)c + kS + k] = wp32[i];
    }

  // layout: per level blocks/faces/child, then coord_of, then weight tables
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  };
  std::vector<size_t> ob(nlev), of(nlev), oc(nlev), orr(nlev), ocf(nlev, 0);
  for (int l = 0; l < nlev; l++) {
    orr[l] = take(hr[l].size() * sizeof(int4));
    ob[l] = take(hb[l].size() * sizeof(int4));
    of[l] = take(hf[l].size() * sizeof(int4));
    oc[l] = take(hc[l].size() * sizeof(int4));
    if (corners) ocf[l] = take(hcf[l].size() * sizeof(int4));
  }
  const size_t ocoord = take((max_blk + 1) * sizeof(int2));
  const size_t owm = take(wn * sizeof(double)), owp = take(wn * sizeof(double));
  const size_t owm32 = take(wn * sizeof(float)), owp32 = take(wn * sizeof(float));
  const size_t owr = take(wrow.size() * sizeof(double)), owr32 = take(wrow32.size() * sizeof(float));
  const size_t oinfo = take((max_blk + 1) * sizeof(int4));
  const size_t ofaceb = take(4 * (max_blk + 1) * sizeof(int4));
  const size_t okids = take((max_blk + 1) * sizeof(int4));
  const size_t olr = take(lrange.size() * sizeof(int2));
  const size_t ochunk = take(std::max<size_t>(chunks.size(), 1) * sizeof(int4));
  const size_t oitch = take(itch.size() * sizeof(int2));
  const size_t oleaf = take(std::max<size_t>(leafblk.size(), 1) * sizeof(int2));
  std::vector<char> host(off, 0);
  for (int l = 0; l < nlev; l++) {
    memcpy(host.data() + orr[l], hr[l].data(), hr[l].size() * sizeof(int4));
    memcpy(host.data() + ob[l], hb[l].data(), hb[l].size() * sizeof(int4));
    memcpy(host.data() + of[l], hf[l].data(), hf[l].size() * sizeof(int4));
    memcpy(host.data() + oc[l], hc[l].data(), hc[l].size() * sizeof(int4));
    if (corners) memcpy(host.data() + ocf[l], hcf[l].data(), hcf[l].size() * sizeof(int4));
  }
  // coord_of indexed by 0-based block id
  std::vector<int2> c0(max_blk + 1, make_int2(0, 0));
  for (int64_t b = 1; b <= max_blk; b++) c0[b - 1] = coord_of[b];
  memcpy(host.data() + ocoord, c0.data(), c0.size() * sizeof(int2));
  memcpy(host.data() + owm, wm.data(), wn * sizeof(double));
  memcpy(host.data() + owp, wp.data(), wn * sizeof(double));
  memcpy(host.data() + owm32, wm32.data(), wn * sizeof(float));
  memcpy(host.data() + owp32, wp32.data(), wn * sizeof(float));
  memcpy(host.data() + owr, wrow.data(), wrow.size() * sizeof(double));
  memcpy(host.data() + owr32, wrow32.data(), wrow32.size() * sizeof(float));
  memcpy(host.data() + oinfo, binfo.data(), binfo.size() * sizeof(int4));
  memcpy(host.data() + ofaceb, bface.data(), bface.size() * sizeof(int4));
  memcpy(host.data() + okids, bkids.data(), bkids.size() * sizeof(int4));
  memcpy(host.data() + olr, lrange.data(), lrange.size() * sizeof(int2));
  memcpy(host.data() + ochunk, chunks.data(), chunks.size() * sizeof(int4));
  memcpy(host.data() + oitch, itch.data(), itch.size() * sizeof(int2));
  memcpy(host.data() + oleaf, leafblk.data(), leafblk.size() * sizeof(int2));

  CK(cudaStreamSynchronize(ctx->stream));
  free_tree(ctx);
  void *d = nullptr;
  if (cudaMalloc(&d, off) != cudaSuccess) return fail(ctx, SRMG_ERR_NOMEM, "tree allocation of %zu bytes", off);
  ctx->d_tree = d;
  // on the context's (non-blocking) stream, so that its later work is ordered after it
  CK(cudaMemcpyAsync(d, host.data(), off, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  char *base = (char *)d;
  ctx->nlev = nlev;
  ctx->lv.resize(nlev);
  ctx->nblk_host.resize(nlev);
  ctx->nch_host.resize(nlev);
  for (int l = 0; l < nlev; l++) {
    ctx->lv[l].nblk = (int)hb[l].size();
    ctx->lv[l].nch = (int)hc[l].size();
    ctx->lv[l].blocks = (int4 *)(base + ob[l]);
    ctx->lv[l].rec = (int4 *)(base + orr[l]);
    ctx->lv[l].faces = (int4 *)(base + of[l]);
    ctx->lv[l].child = (int4 *)(base + oc[l]);
    ctx->lv[l].cfaces = corners ? (int4 *)(base + ocf[l]) : nullptr;
    ctx->nblk_host[l] = ctx->lv[l].nblk;
    ctx->nch_host[l] = ctx->lv[l].nch;
  }
  ctx->d_coord_of = (int2 *)(base + ocoord);
  ctx->d_wm64 = (double *)(base + owm);
  ctx->d_wp64 = (double *)(base + owp);
  ctx->d_wm32 = (float *)(base + owm32);
  ctx->d_wp32 = (float *)(base + owp32);
  ctx->d_wrow64 = (double *)(base + owr);
  ctx->d_wrow32 = (float *)(base + owr32);
  ctx->has_corners = corners;
  ctx->refbnd_levels = 0;
  for (int l = 0; l < nlev; l++)
    if (nrb[l] > 0 && l + 1 < 32) ctx->refbnd_levels |= 1u << (l + 1);
  ctx->d_info = (int4 *)(base + oinfo);
  ctx->d_faceb = (int4 *)(base + ofaceb);
  ctx->d_kids = (int4 *)(base + okids);
  ctx->d_it_lrange = (int2 *)(base + olr);
  ctx->d_chunks = (int4 *)(base + ochunk);
  ctx->d_it_chunks = (int2 *)(base + oitch);
  ctx->nchunk = (int)chunks.size();
  ctx->d_leaf = (int2 *)(base + oleaf);
  ctx->nleaf = (int)leafblk.size();
  ctx->it_lrange_host = lrange;
  ctx->nitems = nitems;
  ctx->l1_blocks = hb[0];
  ctx->l1_faces = hf[0];
  ctx->l2_blocks = nlev >= 2 ? hb[1] : std::vector<int4>();
  ctx->l2_faces = nlev >= 2 ? hf[1] : std::vector<int4>();
  ctx->wtab_n = wn;
  ctx->max_blk = max_blk;
  ctx->generation = generation;
  ctx->has_tree = true;
  ctx->it_tab_host.clear();
  return SRMG_OK;
}

extern "C" int srmg_set_tree(srmg_ctx *ctx, int nlev, const int64_t *npairs,
                             const srmg_pair *const *pairs, const int64_t *nnb,
                             const srmg_neighbor *const *nb, const int64_t *nbd,
                             const srmg_boundary *const *bd, const int64_t *nrb,
                             const srmg_refbnd *const *rb, const int64_t *nch,
                             const srmg_child *const *ch, uint64_t generation) {
  if (ctx && ctx->async_pending)
    return fail(ctx, SRMG_ERR_BADARG, "an asynchronous solve is in flight on this context: call srmg_solve_wait first");
  RC(build_tree(ctx, nlev, npairs, pairs, nnb, nb, nbd, bd, nrb, rb, nch, ch, generation, nullptr, 1));
  // keep the arrays for forests built from this tree
  HostTree &h = ctx->htree;
  h.nlev = nlev;
  h.max_blk = ctx->max_blk;
  h.pairs.assign(nlev, {});
  h.nb.assign(nlev, {});
  h.bd.assign(nlev, {});
  h.rb.assign(nlev, {});
  h.ch.assign(nlev, {});
  for (int l = 0; l < nlev; l++) {
    h.pairs[l].assign(pairs[l], pairs[l] + npairs[l]);
    h.nb[l].assign(nb[l], nb[l] + nnb[l]);
    h.bd[l].assign(bd[l], bd[l] + nbd[l]);
    h.rb[l].assign(rb[l], rb[l] + nrb[l]);
    h.ch[l].assign(ch[l], ch[l] + nch[l]);
  }
  ctx->item_first.assign(1, 0);
  ctx->item_nblk.assign(1, ctx->max_blk);
  ctx->batch_items.clear();
  ctx->geom_forest = -1;
  return SRMG_OK;
}

// ------------------------------------------------------------------ argument checks

int srmg::check_call(srmg_ctx *ctx, int64_t nblk_alloc, int op, int geom, const int8_t *bc) {
  if (!ctx) return SRMG_ERR_BADARG;
  if (ctx->D != 2)
    return fail(ctx, SRMG_ERR_UNSUPPORTED, "three-dimensional trees support the multigrid entry points only");
  return check_call_any(ctx, nblk_alloc, op, geom, bc);
}

int srmg::check_call_any(srmg_ctx *ctx, int64_t nblk_alloc, int op, int geom, const int8_t *bc) {
  if (!ctx) return SRMG_ERR_BADARG;
  if (ctx->async_pending)
    return fail(ctx, SRMG_ERR_BADARG, "an asynchronous solve is in flight on this context: call srmg_solve_wait first");
  if (!ctx->has_tree) return fail(ctx, SRMG_ERR_NOTREE, "no tree: call srmg_set_tree first");
  if (nblk_alloc < ctx->max_blk)
    return fail(ctx, SRMG_ERR_BADARG, "field holds %lld blocks but the tree uses block %lld",
                (long long)nblk_alloc, (long long)ctx->max_blk);
  if (op != SRMG_OP_LAPLACIAN && op != SRMG_OP_HELMHOLTZ && op != SRMG_OP_LAPLACIAN4)
    return fail(ctx, SRMG_ERR_UNSUPPORTED, "unsupported discretisation %d", op);
  if (op == SRMG_OP_LAPLACIAN4 && !ctx->has_corners)
    return fail(ctx, SRMG_ERR_UNSUPPORTED, "the order-4 discretisation needs a BoxStencil connectivity");
  if (geom < 0 || geom > 2) return fail(ctx, SRMG_ERR_UNSUPPORTED, "unsupported geometry %d", geom);
  if (ctx->D == 3 && geom != 0)
    return fail(ctx, SRMG_ERR_UNSUPPORTED, "three-dimensional trees take the Cartesian geometry only");
  if (bc) {
    for (int i = 0; i < (ctx->D == 3 ? 27 : 9); i++)
      if (bc[i] < -1 || bc[i] > 1) return fail(ctx, SRMG_ERR_BADARG, "boundary table entries must be -1, 0 or 1");
  }
  cudaSetDevice(ctx->device);
  return SRMG_OK;
}

Signs srmg::make_signs(const int8_t *bc) {
  Signs s;
  for (int i = 0; i < 9; i++) s.v[i] = bc ? (double)bc[i] : 1.0;
  return s;
}

std::vector<int8_t> srmg::bc_of(const Signs &sg) {
  std::vector<int8_t> bc(9);
  for (int i = 0; i < 9; i++) bc[i] = (int8_t)sg.v[i];
  return bc;
}

// ------------------------------------------------------------------ launches

static inline int grid_for(int64_t work, int threads, int cap) {
  int64_t g = (work + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

constexpr int kGridCap = 148 * 16;

template <typename T>
WTab<T> wtab(srmg_ctx *ctx);
template <>
WTab<double> wtab<double>(srmg_ctx *ctx) { return WTab<double>{ctx->d_wm64, ctx->d_wp64}; }
template <>
WTab<float> wtab<float>(srmg_ctx *ctx) { return WTab<float>{ctx->d_wm32, ctx->d_wp32}; }

template <typename T>
OpParams<T> srmg::op_params(int op, int geom, double k2, double sl, double omega) {
  OpParams<T> p;
  p.op = op;
  p.geom = geom;
  p.s = (T)sl;
  const double centre = (op == SRMG_OP_HELMHOLTZ) ? (-4.0 - sl * k2) : -4.0;
  p.centre = (T)centre;
  const double c = (op == SRMG_OP_HELMHOLTZ) ? (-4 - sl * k2) : -4.0;  // diagelm (order 2)
  p.nwc = (T)(-(omega / c));
  p.omega = (T)omega;
  return p;
}
template OpParams<double> srmg::op_params<double>(int, int, double, double, double);
template OpParams<float> srmg::op_params<float>(int, int, double, double, double);

double srmg::level_scale(double s, int l) {
  const int64_t f = (int64_t)1 << (l - 1);
  return s / (double)(f * f);
}

// While a sequence is being recorded (ctx->seq_rec set, FP64 only) the launchers below
// append their operation instead of launching it.
template <typename T>
static bool seq_push(srmg_ctx *ctx, int kind, int i0, int i1, T *a, const T *b, const T *c, const LevelView &lv,
                     const OpParams<T> *p, const Signs *sg) {
  if (!ctx->seq_rec) return false;
  if (sizeof(T) != sizeof(double)) return false;  // only FP64 cycles are recorded
  SeqOp<T> op;
  memset(&op, 0, sizeof op);
  op.kind = kind;
  op.i0 = i0;
  op.i1 = i1;
  op.a = a;
  op.b = b;
  op.c = c;
  op.lv = lv;
  if (p) op.p = *p;
  if (sg) op.sg = *sg;
  const char *q = reinterpret_cast<const char *>(&op);
  ctx->seq_rec->insert(ctx->seq_rec->end(), q, q + sizeof op);
  ctx->launches++;
  return true;
}

template <typename T>
int srmg::L_fill_ghost(srmg_ctx *ctx, T *u, int l, const Signs &sg, int mask) {
  const DevLevel &L = ctx->lv[l - 1];
  if (L.nblk == 0) return SRMG_OK;
  const int threads = 256;
  const int gf = grid_for((int64_t)L.nblk * 4 * 32, threads, kGridCap);
  if (!L.cfaces) {
    // star faces only: the three passes touch disjoint cells and read none of each
    // other's results, so one launch does them all
    if (seq_push<T>(ctx, SEQ_FILL, mask, 0, u, nullptr, nullptr, L.view(l), nullptr, &sg)) return SRMG_OK;
    k_fill_ghost<T><<<gf, threads, 0, ctx->stream>>>(u, L.view(l), sg, mask);
    ctx->launches++;
    return SRMG_OK;
  }
  // BoxStencil tree: copy, boundary and interpolation are ordered passes (fill_ghost!,
  // src/connectivity.jl:155-159), each launch filling the faces and corners of its
  // passes.  Copy and boundary share one launch (a boundary corner evaluates the face
  // ghost it mirrors itself, fill_corner_cell); interpolation follows on its own.
  if ((mask & 3) == 3) {
    if (!seq_push<T>(ctx, SEQ_FILL, 3, 0, u, nullptr, nullptr, L.view(l), nullptr, &sg)) {
      k_fill_ghost<T><<<gf, threads, 0, ctx->stream>>>(u, L.view(l), sg, 3);
      ctx->launches++;
    }
    mask &= ~3;
  }
  for (int phase = 1; phase <= 4; phase <<= 1) {
    if (!(mask & phase)) continue;
    if (seq_push<T>(ctx, SEQ_FILL, phase, 0, u, nullptr, nullptr, L.view(l), nullptr, &sg)) continue;
    k_fill_ghost<T><<<gf, threads, 0, ctx->stream>>>(u, L.view(l), sg, phase);
    ctx->launches++;
  }
  return SRMG_OK;
}

// ------------------------------------------------------------------ Gauss-Seidel ghost pushes

// The push tables come from the fill itself.  The copy-and-boundary fill (mask 3) of
// every level runs twice on an identity field (each valid cell holds its index in the
// field + 1, each ghost 0): once with every boundary-table entry 1, once with entry k
// the k-th prime.  A ghost left 0 by the first run takes no valid cell's value (it
// mirrors a refinement ghost, or no pass writes it) and is never pushed; any other ghost
// names its source cell, and the ratio of the two runs names the boundary-table entries
// of the mirrors between them (at most two: a corner's and a face's).  A table is used
// only where pushing cannot race the sweep: no cell of the source's colour other than
// the source itself reads the ghost (the 5-point stencil for the red-black sweep, the
// 9-point one for the four-colour sweep).  Anything else -- a ghost that is not a signed
// copy of one valid cell of its own level -- leaves the tree on the fill launches.
// Identity field for building the push tables: every valid cell holds its own index in
// the field + 1 (exact in a double), every ghost 0; `copies` consecutive fields.
static __global__ void k_push_ident(double *__restrict__ a, int64_t n, int copies) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % kSS), x = c % kS, y = c / kS;
    const bool valid = x >= kG && x < kG + kM && y >= kG && y < kG + kM;
    for (int k = 0; k < copies; ++k) a[k * n + i] = valid ? (double)(i + 1) : 0.0;
  }
}

int srmg::ensure_gs_push(srmg_ctx *ctx, int op) {
  if (ctx->D == 3)
    return ctx->has_tree && (ctx->has_corners || op == SRMG_OP_LAPLACIAN4) ? d3_ensure_push(ctx) : SRMG_OK;
  if (ctx->push_state != 0 || !ctx->use_gs_push || !ctx->has_tree || ctx->D != 2 || ctx->seq_rec) return SRMG_OK;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(ctx->stream, &cap));
  if (cap != cudaStreamCaptureStatusNone) return SRMG_OK;
  ctx->push_state = -1;
  const int64_t nf = ctx->max_blk * kSS;
  if (nf <= 0 || nf >= ((int64_t)1 << 31)) return SRMG_OK;
  static const int kPrime[9] = {2, 3, 5, 7, 11, 13, 17, 19, 23};
  Signs ones, primes;
  for (int i = 0; i < 9; i++) {
    ones.v[i] = 1.0;
    primes.v[i] = kPrime[i];
  }
  std::vector<double> h((size_t)(2 * nf));
  {
    double *d = nullptr;
    CK(cudaMalloc(&d, (size_t)(2 * nf) * sizeof(double)));
    const int64_t l0 = ctx->launches;
    k_push_ident<<<grid_for(nf, 256, kGridCap), 256, 0, ctx->stream>>>(d, nf, 2);
    int rc = SRMG_OK;
    for (int l = 1; l <= ctx->nlev && rc == SRMG_OK; l++) {
      rc = L_fill_ghost<double>(ctx, d, l, ones, 3);
      if (rc == SRMG_OK) rc = L_fill_ghost<double>(ctx, d + nf, l, primes, 3);
    }
    ctx->launches = l0;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h.data(), d, (size_t)(2 * nf) * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d);
    RC(rc);
    CK(e);
  }
  std::vector<std::vector<int4>> blocks(ctx->nlev);
  std::vector<int> lvl_of((size_t)ctx->max_blk, 0), bi_of((size_t)ctx->max_blk, -1);
  for (int l = 1; l <= ctx->nlev; l++) {
    const DevLevel &L = ctx->lv[l - 1];
    blocks[l - 1].resize(L.nblk);
    if (L.nblk) CK(cudaMemcpy(blocks[l - 1].data(), L.blocks, L.nblk * sizeof(int4), cudaMemcpyDeviceToHost));
    for (int bi = 0; bi < L.nblk; bi++) {
      const int blk = blocks[l - 1][bi].x;
      if (blk < 0 || blk >= ctx->max_blk) return SRMG_OK;
      lvl_of[blk] = l;
      bi_of[blk] = bi;
    }
  }
  auto valid = [](int x, int y) { return x >= kG && x < kG + kM && y >= kG && y < kG + kM; };
  bool ok2 = true, ok4 = true;
  struct Ent { int key, dest, sg; };
  std::vector<std::vector<Ent>> ents(ctx->nlev);
  for (int l = 1; l <= ctx->nlev; l++)
    for (int bi = 0; bi < ctx->lv[l - 1].nblk; bi++) {
      const int blk = blocks[l - 1][bi].x;
      for (int g = 0; g < kSS; g++) {
        const int gx = g % kS, gy = g / kS;
        if (valid(gx, gy)) continue;
        const int64_t gi = (int64_t)blk * kSS + g;
        const double a = h[gi], a2 = h[nf + gi];
        if (a == 0.0) {
          if (a2 != 0.0) return SRMG_OK;
          continue;
        }
        if (!(a >= 1.0 && a <= (double)nf && a == std::floor(a))) return SRMG_OK;
        const int64_t src = (int64_t)a - 1;
        const int sblk = (int)(src / kSS), sc = (int)(src % kSS), sx = sc % kS, sy = sc / kS;
        if (!valid(sx, sy) || lvl_of[sblk] != l) return SRMG_OK;
        int s1 = 15, s2 = 15;
        bool found = a2 == a;
        for (int i = 0; i < 9 && !found; i++) {
          if (a2 == a * kPrime[i]) {
            s1 = i;
            found = true;
          }
          for (int j = i; j < 9 && !found; j++)
            if (a2 == a * (kPrime[i] * kPrime[j])) {
              s1 = i;
              s2 = j;
              found = true;
            }
        }
        if (!found) return SRMG_OK;
        for (int dy = -1; dy <= 1; dy++)
          for (int dx = -1; dx <= 1; dx++) {
            const int rx = gx + dx, ry = gy + dy;
            if (!valid(rx, ry) || (sblk == blk && rx == sx && ry == sy)) continue;
            if (((rx ^ sx) & 1) == 0 && ((ry ^ sy) & 1) == 0) ok4 = false;
            if (dx * dx + dy * dy == 1 && ((rx + ry + sx + sy) & 1) == 0) ok2 = false;
          }
        ents[l - 1].push_back({bi_of[sblk] * 256 + (sx - kG) + kM * (sy - kG), (int)gi, s1 | (s2 << 4)});
      }
    }
  if (!ok2 && !ok4) return SRMG_OK;
  // per level: offsets (nblk * 256 + 1 ints), then the entries sorted by source cell
  std::vector<size_t> at(ctx->nlev);
  size_t bytes = 0;
  for (int l = 1; l <= ctx->nlev; l++) {
    at[l - 1] = bytes;
    const int nb = ctx->lv[l - 1].nblk;
    if (!nb) continue;
    bytes += ((size_t)nb * 256 + 1) * sizeof(int);
    bytes = (bytes + 15) & ~(size_t)15;
    bytes += ents[l - 1].size() * sizeof(int2);
    bytes = (bytes + 15) & ~(size_t)15;
  }
  std::vector<char> stage(bytes);
  for (int l = 1; l <= ctx->nlev; l++) {
    const int nb = ctx->lv[l - 1].nblk;
    if (!nb) continue;
    int *off = reinterpret_cast<int *>(stage.data() + at[l - 1]);
    const size_t ent_at = (at[l - 1] + ((size_t)nb * 256 + 1) * sizeof(int) + 15) & ~(size_t)15;
    int2 *ent = reinterpret_cast<int2 *>(stage.data() + ent_at);
    std::fill(off, off + nb * 256 + 1, 0);
    for (const Ent &e : ents[l - 1]) off[e.key + 1]++;
    for (int k = 0; k < nb * 256; k++) off[k + 1] += off[k];
    std::vector<int> fillp(off, off + nb * 256);
    for (const Ent &e : ents[l - 1]) ent[fillp[e.key]++] = make_int2(e.dest, e.sg);
  }
  RC(ensure(ctx, ctx->push_tab, bytes));
  CK(cudaMemcpy(ctx->push_tab.p, stage.data(), bytes, cudaMemcpyHostToDevice));
  ctx->push_lv.assign(ctx->nlev, PushView{nullptr, nullptr});
  for (int l = 1; l <= ctx->nlev; l++) {
    const int nb = ctx->lv[l - 1].nblk;
    if (!nb) continue;
    char *base = static_cast<char *>(ctx->push_tab.p);
    const size_t ent_at = (at[l - 1] + ((size_t)nb * 256 + 1) * sizeof(int) + 15) & ~(size_t)15;
    ctx->push_lv[l - 1] = PushView{reinterpret_cast<const int *>(base + at[l - 1]),
                                   reinterpret_cast<const int2 *>(base + ent_at)};
  }
  ctx->push_ok2 = ok2;
  ctx->push_ok4 = ok4;
  ctx->push_state = 1;
  return SRMG_OK;
}

template <typename T>
int srmg::L_gs_colour(srmg_ctx *ctx, T *u, const T *b, int l, const OpParams<T> &p, int parity) {
  const DevLevel &L = ctx->lv[l - 1];
  if (L.nblk == 0) return SRMG_OK;
  const int threads = 128;
  if (p.op == SRMG_OP_LAPLACIAN4) {
    // FourColors{parity >> 1, parity & 1}
    if (seq_push<T>(ctx, SEQ_GS4, parity >> 1, parity & 1, u, b, nullptr, L.view(l), &p, nullptr)) return SRMG_OK;
    k_gs4<T><<<grid_for((int64_t)L.nblk * 64, threads, kGridCap), threads, 0, ctx->stream>>>(
        u, b, L.view(l), p, parity >> 1, parity & 1);
    ctx->launches++;
    return SRMG_OK;
  }
  if (seq_push<T>(ctx, SEQ_GS_COLOUR, parity, 0, u, b, nullptr, L.view(l), &p, nullptr)) return SRMG_OK;
  k_gs_colour<T><<<grid_for((int64_t)L.nblk * 128, threads, kGridCap), threads, 0, ctx->stream>>>(
      u, b, L.view(l), p, wtab<T>(ctx), parity);
  ctx->launches++;
  return SRMG_OK;
}

// One colour sweep that writes the copy and boundary ghosts of the cells it updates.
template <typename T>
static int L_gs_colour_push(srmg_ctx *ctx, T *u, const T *b, int l, const OpParams<T> &p, int parity,
                            const Signs &sg) {
  const DevLevel &L = ctx->lv[l - 1];
  const int threads = 128;
  unsigned sw = 0;  // entry + 1, two bits an entry (every entry is -1, 0 or 1 here)
  for (int i = 0; i < 9; i++) sw |= (unsigned)((int)sg.v[i] + 1) << (2 * i);
  if (p.op == SRMG_OP_LAPLACIAN4)
    k_gs4_push<T><<<grid_for((int64_t)L.nblk * 64, threads, kGridCap), threads, 0, ctx->stream>>>(
        u, b, L.view(l), p, parity >> 1, parity & 1, ctx->push_lv[l - 1], sw);
  else
    k_gs_colour_push<T><<<grid_for((int64_t)L.nblk * 128, threads, kGridCap), threads, 0, ctx->stream>>>(
        u, b, L.view(l), p, wtab<T>(ctx), parity, ctx->push_lv[l - 1], sw);
  ctx->launches++;
  return SRMG_OK;
}

// gauss_seidel_iter! (src/multigrid.jl:250-295): red-black (two colours) or, at order 4,
// four colours {0,0}, {0,1}, {1,0}, {1,1}, each followed by copy and boundary ghosts.
// With the push tables (ensure_gs_push) the first colour keeps its fill launch -- after
// it the ghosts are what the fill makes of the current cells, whatever they held before
// -- and every later colour writes the ghosts of the cells it updates itself, which is
// all that the fill after it would change: one launch a colour instead of two, the
// same values.
template <typename T>
int srmg::L_gs_iter(srmg_ctx *ctx, T *u, const T *b, int l, const OpParams<T> &p, int n,
                    const Signs &sg) {
  const bool four = p.op == SRMG_OP_LAPLACIAN4;
  if (ctx->push_state == 0) RC(ensure_gs_push(ctx, p.op));
  bool unit = true;
  for (int i = 0; i < 9; i++) unit = unit && (sg.v[i] == 1.0 || sg.v[i] == -1.0 || sg.v[i] == 0.0);
  const bool push = ctx->use_gs_push && ctx->push_state == 1 && !ctx->seq_rec && unit &&
                    (four ? ctx->push_ok4 : ctx->push_ok2) && ctx->lv[l - 1].nblk > 0;
  const int ncol = four ? 4 : 2;
  for (int i = 0; i < n; i++)
    for (int c = 0; c < ncol; c++) {
      if (push && (i > 0 || c > 0)) {
        RC(L_gs_colour_push<T>(ctx, u, b, l, p, c, sg));
        continue;
      }
      RC(L_gs_colour<T>(ctx, u, b, l, p, c));
      RC(L_fill_ghost<T>(ctx, u, l, sg, 3));
    }
  return SRMG_OK;
}

template <typename T>
int srmg::L_residual(srmg_ctx *ctx, T *r, const T *u, const T *b, int l, const OpParams<T> &p) {
  const DevLevel &L = ctx->lv[l - 1];
  if (L.nblk == 0) return SRMG_OK;
  if (seq_push<T>(ctx, SEQ_RESIDUAL, 0, 0, r, u, b, L.view(l), &p, nullptr)) return SRMG_OK;
  k_residual<T><<<grid_for((int64_t)L.nblk * 256, 256, kGridCap), 256, 0, ctx->stream>>>(
      r, u, b, L.view(l), p, wtab<T>(ctx));
  ctx->launches++;
  return SRMG_OK;
}

template <typename T>
int srmg::L_postrestrict(srmg_ctx *ctx, T *bf, const T *u, const T *r, int l, const OpParams<T> &pc) {
  const DevLevel &L = ctx->lv[l - 1];
  if (L.nch == 0) return SRMG_OK;
  if (seq_push<T>(ctx, SEQ_POSTRESTRICT, 0, 0, bf, u, r, L.view(l), &pc, nullptr)) return SRMG_OK;
  k_postrestrict<T><<<grid_for((int64_t)L.nch * 64, 256, kGridCap), 256, 0, ctx->stream>>>(
      bf, u, r, L.view(l), ctx->d_coord_of, pc, wtab<T>(ctx));
  ctx->launches++;
  return SRMG_OK;
}

template <typename T>
int srmg::L_restrict(srmg_ctx *ctx, T *u, int l) {
  const DevLevel &L = ctx->lv[l - 1];
  if (L.nch == 0) return SRMG_OK;
  if (seq_push<T>(ctx, SEQ_RESTRICT, 0, 0, u, nullptr, nullptr, L.view(l), nullptr, nullptr)) return SRMG_OK;
  k_restrict<T><<<grid_for((int64_t)L.nch * 64, 256, kGridCap), 256, 0, ctx->stream>>>(u, L.view(l));
  ctx->launches++;
  return SRMG_OK;
}

template <typename T>
int srmg::L_interp_add(srmg_ctx *ctx, T *u, const T *u1, int l) {
  const DevLevel &L = ctx->lv[l - 1];
  if (L.nch == 0) return SRMG_OK;
  if (seq_push<T>(ctx, SEQ_INTERP_ADD, 0, 0, u, u1, nullptr, L.view(l), nullptr, nullptr)) return SRMG_OK;
  k_interp_add<T><<<grid_for((int64_t)L.nch * 256, 256, kGridCap), 256, 0, ctx->stream>>>(
      u, u1, L.view(l));
  ctx->launches++;
  return SRMG_OK;
}

template <typename T>
int srmg::L_copy(srmg_ctx *ctx, T *dst, const T *src, int l) {
  const DevLevel &L = ctx->lv[l - 1];
  if (L.nblk == 0) return SRMG_OK;
  if (seq_push<T>(ctx, SEQ_COPY, 0, 0, dst, src, nullptr, L.view(l), nullptr, nullptr)) return SRMG_OK;
  k_copy_level<T><<<grid_for((int64_t)L.nblk * kSS, 256, kGridCap), 256, 0, ctx->stream>>>(
      dst, src, L.view(l));
  ctx->launches++;
  return SRMG_OK;
}

template <typename T>
int srmg::L_diff(srmg_ctx *ctx, T *dst, const T *a1, const T *a2, int l) {
  const DevLevel &L = ctx->lv[l - 1];
  if (L.nblk == 0) return SRMG_OK;
  if (seq_push<T>(ctx, SEQ_DIFF, 0, 0, dst, a1, a2, L.view(l), nullptr, nullptr)) return SRMG_OK;
  k_diff_level<T><<<grid_for((int64_t)L.nblk * kSS, 256, kGridCap), 256, 0, ctx->stream>>>(
      dst, a1, a2, L.view(l));
  ctx->launches++;
  return SRMG_OK;
}

// ------------------------------------------------------------------ V-cycle / FMG

template <typename T>
int srmg::vcycle_dev(srmg_ctx *ctx, T *u, T *b, T *r, T *u1, double s, int op, double k2, int geom,
                     const Signs &sg, int lmax, int ndown, int ntop, int nup, double omega) {
  if (lmax == 0) lmax = ctx->nlev;
  if (lmax < 1 || lmax > ctx->nlev) return fail(ctx, SRMG_ERR_BADARG, "lmax %d out of range", lmax);
  // The persistent engine runs the whole cycle in one launch; r carries the coarse
  // corrections there.  Sweep counts of zero keep the per-operation kernels.
  // Bulk copies need 16-byte aligned block tiles.
  const bool aligned = ((reinterpret_cast<uintptr_t>(u) | reinterpret_cast<uintptr_t>(b) |
                         reinterpret_cast<uintptr_t>(r) | reinterpret_cast<uintptr_t>(u1)) & 15) == 0;
  // The engine's ghost pushes cover the four star faces only; trees with corner ghosts
  // (BoxStencil connectivity) and the order-4 stencil use the per-operation kernels.
  // (a sequence being recorded holds per-operation records only)
  if (ctx->use_engine && aligned && !ctx->has_corners && op != SRMG_OP_LAPLACIAN4 && ndown >= 1 &&
      ntop >= 1 && nup >= 1 && ctx->nlev <= 30 && !ctx->seq_rec) {
    ItemTabs tabs;
    const std::vector<ItemSpec> specs = uniform_items(ctx, s, op, k2, bc_of(sg).data());
    RC(prepare_items(ctx, specs.data(), geom, omega, false, 0, 0.0, &tabs));
    return engine_vcycle<T>(ctx, u, b, u1, r, tabs, geom, lmax, ndown, ntop, nup);
  }
  for (int l = lmax; l >= 2; l--) {
    const double sl = level_scale(s, l);
    const OpParams<T> p = op_params<T>(op, geom, k2, sl, omega);
    const OpParams<T> pc = op_params<T>(op, geom, k2, 4 * sl, omega);
    RC(L_gs_iter<T>(ctx, u, b, l, p, ndown, sg));
    RC(L_restrict<T>(ctx, u, l));
    RC(L_fill_ghost<T>(ctx, u, l - 1, sg, 7));
    RC(L_copy<T>(ctx, u1, u, l - 1));
    RC(L_residual<T>(ctx, r, u, b, l, p));
    // fill_ghost!(r, l) and fill_ghost!(r, l-1) (src/multigrid.jl:80,83) are skipped:
    // r is scratch and no later operation reads r's ghost cells.
    RC(L_restrict<T>(ctx, r, l));
    RC(L_postrestrict<T>(ctx, b, u, r, l, pc));
  }
  {
    const OpParams<T> p = op_params<T>(op, geom, k2, s, omega);
    RC(L_gs_iter<T>(ctx, u, b, 1, p, ntop, sg));
  }
  for (int l = 2; l <= lmax; l++) {
    const double sl = level_scale(s, l);
    const OpParams<T> p = op_params<T>(op, geom, k2, sl, omega);
    RC(L_diff<T>(ctx, u1, u, u1, l - 1));
    RC(L_fill_ghost<T>(ctx, u1, l - 1, sg, 7));
    RC(L_interp_add<T>(ctx, u, u1, l));
    RC(L_fill_ghost<T>(ctx, u, l, sg, 7));
    RC(L_gs_iter<T>(ctx, u, b, l, p, nup, sg));
    RC(L_fill_ghost<T>(ctx, u, l, sg, 7));
  }
  return SRMG_OK;
}
template int srmg::vcycle_dev<double>(srmg_ctx *, double *, double *, double *, double *, double, int,
                                      double, int, const Signs &, int, int, int, int, double);
template int srmg::vcycle_dev<float>(srmg_ctx *, float *, float *, float *, float *, double, int,
                                     double, int, const Signs &, int, int, int, int, double);

static int finest_level(srmg_ctx *ctx) {
  int lmax = 0;
  for (int l = 1; l <= ctx->nlev; l++)
    if (ctx->nblk_host[l - 1] > 0) lmax = l;
  return lmax;
}

template <typename T>
static int fmg_dev_t(srmg_ctx *ctx, T *u, T *b, T *r, T *u1, double s, int op, double k2, int geom,
                     const Signs &sg, int ndown, int ntop, int nup, double omega) {
  const int lmax = finest_level(ctx);
  for (int l = lmax; l >= 2; l--) {
    const double sl = level_scale(s, l);
    const OpParams<T> p = op_params<T>(op, geom, k2, sl, omega);
    const OpParams<T> pc = op_params<T>(op, geom, k2, 4 * sl, omega);
    RC(L_restrict<T>(ctx, u, l));
    RC(L_fill_ghost<T>(ctx, u, l - 1, sg, 7));
    RC(L_residual<T>(ctx, r, u, b, l, p));
    RC(L_restrict<T>(ctx, r, l));
    RC(L_postrestrict<T>(ctx, b, u, r, l, pc));
  }
  for (int l = 1; l <= lmax; l++) {
    RC(L_copy<T>(ctx, u1, u, l));
    if (l > 1) {
      RC(L_diff<T>(ctx, u1, u, u1, l - 1));
      RC(L_fill_ghost<T>(ctx, u1, l - 1, sg, 7));
      RC(L_interp_add<T>(ctx, u, u1, l));
    }
    RC(L_fill_ghost<T>(ctx, u, l, sg, 7));
    RC(vcycle_dev<T>(ctx, u, b, r, u1, s, op, k2, geom, sg, l, ndown, ntop, nup, omega));
  }
  return SRMG_OK;
}

// ------------------------------------------------------------------ norms

// Leaf-weighted sum of squares of the residual (mode 0) or of b (mode 1) over all
// levels, reduced in a fixed order into ctx->small[slot] (sqrt applied).
template <typename T>
int srmg::leafnorm_dev(srmg_ctx *ctx, const T *u, const T *b, double s, int op, double k2, int geom,
                       int mode, int slot) {
  constexpr int NT = 256;
  int total_parts = 0;
  std::vector<int> grids(ctx->nlev);
  for (int l = 1; l <= ctx->nlev; l++) {
    const int n = ctx->nblk_host[l - 1];
    grids[l - 1] = n ? grid_for((int64_t)n * 256, NT, 148 * 4) : 0;
    total_parts += grids[l - 1];
  }
  RC(ensure(ctx, ctx->part, sizeof(double) * std::max(total_parts, 1)));
  double *part = (double *)ctx->part.p;
  int off = 0;
  for (int l = 1; l <= ctx->nlev; l++) {
    if (!grids[l - 1]) continue;
    const double sl = level_scale(s, l);
    const OpParams<T> p = op_params<T>(op, geom, k2, sl, 1.0);
    const double wl = 1.0 / (double)((int64_t)1 << (2 * (l - 1)));
    k_leafsq<T, NT><<<grids[l - 1], NT, 0, ctx->stream>>>(part + off, u, b, ctx->lv[l - 1].view(l), p,
                                                        wtab<T>(ctx), wl, mode);
    ctx->launches++;
    off += grids[l - 1];
  }
  double *out = (double *)ctx->small.p + slot;
  if (total_parts == 0) {
    CK(cudaMemsetAsync(out, 0, sizeof(double), ctx->stream));
    return SRMG_OK;
  }
  k_reduce_sqrt<1024><<<1, 1024, 0, ctx->stream>>>(out, part, total_parts);
  ctx->launches++;
  return SRMG_OK;
}
template int srmg::leafnorm_dev<double>(srmg_ctx *, const double *, const double *, double, int, double,
                                        int, int, int);
template int srmg::leafnorm_dev<float>(srmg_ctx *, const float *, const float *, double, int, double,
                                       int, int, int);

int srmg::read_small(srmg_ctx *ctx, int n) {
  CK(cudaMemcpyAsync(ctx->h_small, ctx->small.p, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return engine_check(ctx);
}

extern "C" int srmg_set_option(srmg_ctx *ctx, const char *key, int64_t value) {
  if (!ctx || !key) return SRMG_ERR_BADARG;
  if (ctx->async_pending)
    return fail(ctx, SRMG_ERR_BADARG, "an asynchronous solve is in flight on this context: call srmg_solve_wait first");
  if (!strcmp(key, "engine")) ctx->use_engine = value != 0;
  else if (!strcmp(key, "trace")) ctx->trace_on = value != 0;
  else if (!strcmp(key, "b_copy_back")) ctx->b_copy_back = value != 0;
  else if (!strcmp(key, "freebc_direct")) ctx->fbc_direct = value != 0;
  else if (!strcmp(key, "graph")) ctx->use_graph = value != 0;
  else if (!strcmp(key, "direct_level")) {
    if (value < 0 || value > 2) return fail(ctx, SRMG_ERR_BADARG, "direct_level must be 0, 1 or 2");
    ctx->direct_level = (int)value;
  } else if (!strcmp(key, "op_sequencer")) {
    ctx->use_op_seq = value != 0;
    if (!ctx->use_op_seq) drop_op_graphs(ctx);
  }
  else if (!strcmp(key, "gs_push")) {
    ctx->use_gs_push = value != 0;
    drop_op_graphs(ctx);
  }
  else if (!strcmp(key, "op_graphs")) {
    ctx->use_op_graphs = value != 0;
    if (!ctx->use_op_graphs) drop_op_graphs(ctx);
  }
  else if (!strcmp(key, "cnn_active_ppm")) {
    if (value < 0 || value > 1000000) return fail(ctx, SRMG_ERR_BADARG, "cnn_active_ppm out of range");
    ctx->cnn_active_ppm = (int)value;
  }
  else if (!strcmp(key, "local_max_blocks")) {
    if (value < 0 || value > 1024) return fail(ctx, SRMG_ERR_BADARG, "local_max_blocks out of range");
    ctx->local_max_blocks = (int)value;
  } else if (!strcmp(key, "engine_ctas")) {
    if (value < 0) return fail(ctx, SRMG_ERR_BADARG, "engine_ctas must be >= 0");
    if (value > 0) {
      int nsm = 0;
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
      if (value > nsm) return fail(ctx, SRMG_ERR_BADARG, "engine_ctas above the SM count (%d)", nsm);
    }
    ctx->engine_ctas = (int)value;
  } else if (!strcmp(key, "engine_threads")) {
    if (value != 0 && value != 768 && value != 1024)
      return fail(ctx, SRMG_ERR_BADARG, "engine_threads must be 0 (by tree size), 768 or 1024");
    ctx->engine_threads = (int)value;
  } else return fail(ctx, SRMG_ERR_BADARG, "unknown option '%s'", key);
  return SRMG_OK;
}

// ------------------------------------------------------------------ graphed per-operation V-cycles

namespace {
constexpr size_t kOpGraphs = 8;

template <typename V>
void put(std::vector<char> &k, const V &v) {
  const char *p = reinterpret_cast<const char *>(&v);
  k.insert(k.end(), p, p + sizeof(V));
}

int run_vcycles(srmg_ctx *ctx, double *u, double *b, double *r, double *u1, double s, int op, double k2, int geom,
                const int8_t *bc, int lmax, int ndown, int ntop, int nup, double omega, int ncycles) {
  if (ctx->D == 3) {
    for (int c = 0; c < ncycles; c++) RC(d3_vcycle(ctx, u, b, r, u1, s, op, k2, bc, lmax, ndown, ntop, nup, omega));
    return SRMG_OK;
  }
  const Signs sg = make_signs(bc);
  for (int c = 0; c < ncycles; c++)
    RC(vcycle_dev<double>(ctx, u, b, r, u1, s, op, k2, geom, sg, lmax, ndown, ntop, nup, omega));
  return SRMG_OK;
}
}  // namespace

// A per-operation V-cycle is a fixed sequence of several hundred small launches with no
// host work in between, so it is captured once into a CUDA graph and replayed: the
// kernels are the same, only their launch overhead changes.  The graph bakes in the
// field pointers, the operator, the sweep counts and the tree's device arrays, all of
// which are part of the key; a new tree drops every graph.
int srmg::vcycle_ops(srmg_ctx *ctx, double *u, double *b, double *r, double *u1, double s, int op, double k2,
                     int geom, const int8_t *bc, int lmax, int ndown, int ntop, int nup, double omega, int ncycles) {
  // a caller already capturing the stream records the launches into its own graph
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(ctx->stream, &cap));
  const bool seq = ctx->use_op_seq;
  if (!(ctx->use_op_graphs || seq) || ncycles <= 0 || cap != cudaStreamCaptureStatusNone)
    return run_vcycles(ctx, u, b, r, u1, s, op, k2, geom, bc, lmax, ndown, ntop, nup, omega, ncycles);
  RC(ensure_gs_push(ctx, op));  // before the key: a graph bakes in whether the sweeps push
  std::vector<char> key;
  for (const void *p : {(const void *)u, (const void *)b, (const void *)r, (const void *)u1, (const void *)ctx->d_tree,
                        (const void *)ctx->stream})
    put(key, p);
  for (double v : {s, k2, omega}) put(key, v);
  for (int v : {op, geom, lmax, ndown, ntop, nup, ncycles, ctx->D}) put(key, v);
  put(key, ctx->generation);
  put(key, (int)(ctx->use_gs_push && ctx->push_state == 1));
  const int nbc = ctx->D == 3 ? 27 : 9;
  for (int i = 0; i < nbc; i++) put(key, (int8_t)(bc ? bc[i] : 1));
  if (seq) {
    // the whole sequence as one cooperative launch of the sequencer: record it once per
    // key (the launchers append their operations instead of launching), keep it on the
    // device, launch it
    auto launch = [&](const srmg_ctx::OpSeq &q) {
      return ctx->D == 3 ? seq_launch3(ctx, q.ops.p, q.nops) : seq_launch(ctx, q.ops.p, q.nops);
    };
    for (auto &q : ctx->op_seqs)
      if (q.key == key) return launch(q);
    std::vector<char> rec;
    const int64_t l0 = ctx->launches;
    ctx->seq_rec = &rec;
    const int rc = run_vcycles(ctx, u, b, r, u1, s, op, k2, geom, bc, lmax, ndown, ntop, nup, omega, ncycles);
    ctx->seq_rec = nullptr;
    ctx->launches = l0;
    if (rc) return rc;
    if (ctx->op_seqs.size() >= kOpGraphs) {
      if (ctx->op_seqs.front().ops.p) cudaFree(ctx->op_seqs.front().ops.p);
      ctx->op_seqs.erase(ctx->op_seqs.begin());
    }
    srmg_ctx::OpSeq q;
    q.key = key;
    q.nops = (int)(rec.size() / (ctx->D == 3 ? seq3_op_bytes() : seq_op_bytes()));
    if (q.nops > 0) {
      RC(ensure(ctx, q.ops, rec.size()));
      // on the context's stream: the launch below is ordered after the copy (pageable
      // source, staged before the call returns)
      CK(cudaMemcpyAsync(q.ops.p, rec.data(), rec.size(), cudaMemcpyHostToDevice, ctx->stream));
    }
    ctx->op_seqs.push_back(q);
    return launch(q);
  }
  for (auto &g : ctx->op_graphs)
    if (g.key == key) {
      CK(cudaGraphLaunch(g.exec, ctx->stream));
      ctx->launches += g.launches;
      return SRMG_OK;
    }
  cudaGraph_t graph = nullptr;
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  const int64_t l0 = ctx->launches;
  const int rc = run_vcycles(ctx, u, b, r, u1, s, op, k2, geom, bc, lmax, ndown, ntop, nup, omega, ncycles);
  const cudaError_t ec = cudaStreamEndCapture(ctx->stream, &graph);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (ec != cudaSuccess) return cuda_check(ctx, ec, "cudaStreamEndCapture");
  cudaGraphExec_t exec = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ei != cudaSuccess) return cuda_check(ctx, ei, "cudaGraphInstantiate");
  if (ctx->op_graphs.size() >= kOpGraphs) {
    cudaGraphExecDestroy(ctx->op_graphs.front().exec);
    ctx->op_graphs.erase(ctx->op_graphs.begin());
  }
  ctx->op_graphs.push_back({key, exec, ctx->launches - l0});
  CK(cudaGraphLaunch(exec, ctx->stream));
  return SRMG_OK;
}

// ------------------------------------------------------------------ device entry points

extern "C" int srmg_vcycle_dev(srmg_ctx *ctx, double *u, double *b, double *r, double *u1,
                               int64_t nblk_alloc, double s, int op, double k2, int geom,
                               const int8_t bc[9], int lmax, int ndown, int ntop, int nup,
                               double omega, int ncycles) {
  RC(check_call_any(ctx, nblk_alloc, op, geom, bc));
  if (!u || !b || !r || !u1 || ndown < 0 || ntop < 0 || nup < 0 || ncycles < 0)
    return fail(ctx, SRMG_ERR_BADARG, "srmg_vcycle: bad arguments");
  // the per-operation path (3D trees, BoxStencil trees, order 4, or the engine switched
  // off) runs from a captured graph; the persistent engine is one launch already
  const bool aligned = ((reinterpret_cast<uintptr_t>(u) | reinterpret_cast<uintptr_t>(b) |
                         reinterpret_cast<uintptr_t>(r) | reinterpret_cast<uintptr_t>(u1)) & 15) == 0;
  const bool engine = ctx->D == 2 && ctx->use_engine && aligned && !ctx->has_corners && op != SRMG_OP_LAPLACIAN4 &&
                      ndown >= 1 && ntop >= 1 && nup >= 1 && ctx->nlev <= 30;
  if (!engine) {
    if (lmax < 0 || lmax > ctx->nlev) return fail(ctx, SRMG_ERR_BADARG, "lmax %d out of range", lmax);
    RC(vcycle_ops(ctx, u, b, r, u1, s, op, k2, geom, bc, lmax, ndown, ntop, nup, omega, ncycles));
    CK(cudaGetLastError());
    return SRMG_OK;
  }
  const Signs sg = make_signs(bc);
  for (int c = 0; c < ncycles; c++)
    RC(vcycle_dev<double>(ctx, u, b, r, u1, s, op, k2, geom, sg, lmax, ndown, ntop, nup, omega));
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_fmg_dev(srmg_ctx *ctx, double *u, double *b, double *r, double *u1,
                            int64_t nblk_alloc, double s, int op, double k2, int geom,
                            const int8_t bc[9], int ndown, int ntop, int nup, double omega) {
  RC(check_call_any(ctx, nblk_alloc, op, geom, bc));
  if (!u || !b || !r || !u1) return fail(ctx, SRMG_ERR_BADARG, "srmg_fmg: null field");
  if (ctx->D == 3) RC(d3_fmg(ctx, u, b, r, u1, s, op, k2, bc, ndown, ntop, nup, omega));
  else RC(fmg_dev_t<double>(ctx, u, b, r, u1, s, op, k2, geom, make_signs(bc), ndown, ntop, nup, omega));
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_resnorm_dev(srmg_ctx *ctx, double *r, const double *b, const double *u,
                                int64_t nblk_alloc, double s, int op, double k2, int geom,
                                const int8_t bc[9], double *out) {
  RC(check_call_any(ctx, nblk_alloc, op, geom, bc));
  (void)r;
  if (!b || !u || !out) return fail(ctx, SRMG_ERR_BADARG, "srmg_resnorm: null argument");
  if (ctx->D == 3) RC(d3_leafnorm(ctx, u, b, s, op, k2, 0, 0));
  else RC(leafnorm_dev<double>(ctx, u, b, s, op, k2, geom, 0, 0));
  RC(read_small(ctx, 1));
  *out = ctx->h_small[0];
  return SRMG_OK;
}

extern "C" int srmg_fill_ghost_dev(srmg_ctx *ctx, double *u, int64_t nblk_alloc, int level,
                                   const int8_t bc[9], int mask) {
  RC(check_call_any(ctx, nblk_alloc, 0, 0, bc));
  if (!u || level < 1 || level > ctx->nlev) return fail(ctx, SRMG_ERR_BADARG, "fill_ghost: bad level");
  if (mask & 8) {
    // InterpCopy refinement ghosts: one launch over the star faces only
    if (ctx->D == 3 || ctx->has_corners)
      return fail(ctx, SRMG_ERR_UNSUPPORTED, "fill_ghost: InterpCopy ghosts (mask bit 3) on 2D StarStencil trees only");
    if (!(mask & 4)) return fail(ctx, SRMG_ERR_BADARG, "fill_ghost: mask bit 3 needs bit 2");
  }
  if (ctx->D == 3) RC(d3_fill_ghost(ctx, u, level, bc, mask));
  else RC(L_fill_ghost<double>(ctx, u, level, make_signs(bc), mask));
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_gs_level_dev(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc,
                                 int level, double omega, double sl, int op, double k2, int geom,
                                 int parity) {
  RC(check_call_any(ctx, nblk_alloc, op, geom, nullptr));
  const int ncol = op == SRMG_OP_LAPLACIAN4 ? 4 : 2;
  if (!u || !b || level < 1 || level > ctx->nlev || parity < 0 || parity >= ncol)
    return fail(ctx, SRMG_ERR_BADARG, "gs_level: bad arguments");
  if (ctx->D == 3) {
    RC(d3_gs_level(ctx, u, b, level, omega, sl, op, k2, parity));
    CK(cudaGetLastError());
    return SRMG_OK;
  }
  RC(L_gs_colour<double>(ctx, u, b, level, op_params<double>(op, geom, k2, sl, omega), parity));
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_gs_iter_dev(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc,
                                int level, double omega, double sl, int n, int op, double k2,
                                int geom, const int8_t bc[9]) {
  RC(check_call_any(ctx, nblk_alloc, op, geom, bc));
  if (!u || !b || level < 1 || level > ctx->nlev || n < 0)
    return fail(ctx, SRMG_ERR_BADARG, "gs_iter: bad arguments");
  if (ctx->D == 3) {
    RC(d3_gs_iter(ctx, u, b, level, omega, sl, n, op, k2, bc));
    CK(cudaGetLastError());
    return SRMG_OK;
  }
  const bool aligned = ((reinterpret_cast<uintptr_t>(u) | reinterpret_cast<uintptr_t>(b)) & 15) == 0;
  if (ctx->use_engine && aligned && !ctx->has_corners && op != SRMG_OP_LAPLACIAN4) {
    ItemTabs tabs;
    const std::vector<ItemSpec> specs = uniform_items(ctx, sl, op, k2, bc);
    RC(prepare_items(ctx, specs.data(), geom, omega, false, level, sl, &tabs));
    RC(engine_smooth<double>(ctx, u, b, tabs, geom, level, n));
  } else
    RC(L_gs_iter<double>(ctx, u, b, level, op_params<double>(op, geom, k2, sl, omega), n, make_signs(bc)));
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_residual_level_dev(srmg_ctx *ctx, double *r, const double *u, const double *b,
                                       int64_t nblk_alloc, int level, double sl, int op, double k2,
                                       int geom) {
  RC(check_call_any(ctx, nblk_alloc, op, geom, nullptr));
  if (!r || !u || !b || level < 1 || level > ctx->nlev)
    return fail(ctx, SRMG_ERR_BADARG, "residual_level: bad arguments");
  if (ctx->D == 3) RC(d3_residual_level(ctx, r, u, b, level, sl, op, k2));
  else RC(L_residual<double>(ctx, r, u, b, level, op_params<double>(op, geom, k2, sl, 1.0)));
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_restrict_level_dev(srmg_ctx *ctx, double *u, int64_t nblk_alloc, int level) {
  RC(check_call_any(ctx, nblk_alloc, 0, 0, nullptr));
  if (!u || level < 1 || level > ctx->nlev) return fail(ctx, SRMG_ERR_BADARG, "restrict_level: bad level");
  if (ctx->D == 3) RC(d3_restrict_level(ctx, u, level));
  else RC(L_restrict<double>(ctx, u, level));
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_rhs_level_dev(srmg_ctx *ctx, double *q1, const double *q, int64_t nblk_alloc, int level,
                                  int op, int geom) {
  RC(check_call_any(ctx, nblk_alloc, op, geom, nullptr));
  if (!q1 || !q || level < 1 || level > ctx->nlev) return fail(ctx, SRMG_ERR_BADARG, "rhs_level: bad arguments");
  if (ctx->D == 3) {
    RC(d3_rhs_level(ctx, q1, q, level, op));
    CK(cudaGetLastError());
    return SRMG_OK;
  }
  const DevLevel &L = ctx->lv[level - 1];
  if (L.nblk > 0) {
    k_rhs<double><<<grid_for((int64_t)L.nblk * 256, 256, kGridCap), 256, 0, ctx->stream>>>(q1, q, L.view(level),
                                                                                         op, geom);
    ctx->launches++;
  }
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_interp_add_level_dev(srmg_ctx *ctx, double *u, const double *u1,
                                         int64_t nblk_alloc, int level) {
  RC(check_call_any(ctx, nblk_alloc, 0, 0, nullptr));
  if (!u || !u1 || level < 1 || level > ctx->nlev)
    return fail(ctx, SRMG_ERR_BADARG, "interp_add_level: bad level");
  if (ctx->D == 3) RC(d3_interp_add_level(ctx, u, u1, level));
  else RC(L_interp_add<double>(ctx, u, u1, level));
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_residual_postrestrict_level_dev(srmg_ctx *ctx, double *b, const double *u,
                                                    const double *r, int64_t nblk_alloc, int level,
                                                    double s, int op, double k2, int geom) {
  RC(check_call_any(ctx, nblk_alloc, op, geom, nullptr));
  if (!b || !u || !r || level < 1 || level > ctx->nlev)
    return fail(ctx, SRMG_ERR_BADARG, "postrestrict: bad arguments");
  if (ctx->D == 3) RC(d3_postrestrict_level(ctx, b, u, r, level, s, op, k2));
  else RC(L_postrestrict<double>(ctx, b, u, r, level, op_params<double>(op, geom, k2, s, 1.0)));
  CK(cudaGetLastError());
  return SRMG_OK;
}

// ------------------------------------------------------------------ host entry points

// Copy host fields into the context's device mirrors (slot i of f64).
int srmg::stage_in(srmg_ctx *ctx, int slot, const double *h, int64_t nblk_alloc, double **d) {
  const size_t bytes = (size_t)nblk_alloc * block_elems(ctx) * sizeof(double);
  RC(ensure(ctx, ctx->f64[slot], bytes));
  *d = (double *)ctx->f64[slot].p;
  if (h) CK(cudaMemcpyAsync(*d, h, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return SRMG_OK;
}

int srmg::stage_out(srmg_ctx *ctx, double *h, const double *d, int64_t nblk_alloc) {
  const size_t bytes = (size_t)nblk_alloc * block_elems(ctx) * sizeof(double);
  CK(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  return SRMG_OK;
}

extern "C" int srmg_vcycle(srmg_ctx *ctx, double *u, double *b, double *r, double *u1,
                           int64_t nblk_alloc, double s, int op, double k2, int geom,
                           const int8_t bc[9], int lmax, int ndown, int ntop, int nup, double omega,
                           int ncycles) {
  RC(check_call_any(ctx, nblk_alloc, op, geom, bc));
  if (!u || !b) return fail(ctx, SRMG_ERR_BADARG, "srmg_vcycle: null field");
  (void)r;
  (void)u1;
  double *du, *db, *dr, *du1;
  RC(stage_in(ctx, 0, u, nblk_alloc, &du));
  RC(stage_in(ctx, 1, b, nblk_alloc, &db));
  RC(stage_in(ctx, 2, nullptr, nblk_alloc, &dr));
  RC(stage_in(ctx, 3, nullptr, nblk_alloc, &du1));
  RC(srmg_vcycle_dev(ctx, du, db, dr, du1, nblk_alloc, s, op, k2, geom, bc, lmax, ndown, ntop, nup,
                     omega, ncycles));
  RC(stage_out(ctx, u, du, nblk_alloc));
  if (ctx->b_copy_back) RC(stage_out(ctx, b, db, nblk_alloc));
  CK(cudaStreamSynchronize(ctx->stream));
  return engine_check(ctx);
}

extern "C" int srmg_fmg(srmg_ctx *ctx, double *u, double *b, double *r, double *u1,
                        int64_t nblk_alloc, double s, int op, double k2, int geom,
                        const int8_t bc[9], int ndown, int ntop, int nup, double omega) {
  RC(check_call_any(ctx, nblk_alloc, op, geom, bc));
  if (!u || !b) return fail(ctx, SRMG_ERR_BADARG, "srmg_fmg: null field");
  (void)r;
  (void)u1;
  double *du, *db, *dr, *du1;
  RC(stage_in(ctx, 0, u, nblk_alloc, &du));
  RC(stage_in(ctx, 1, b, nblk_alloc, &db));
  RC(stage_in(ctx, 2, nullptr, nblk_alloc, &dr));
  RC(stage_in(ctx, 3, nullptr, nblk_alloc, &du1));
  RC(srmg_fmg_dev(ctx, du, db, dr, du1, nblk_alloc, s, op, k2, geom, bc, ndown, ntop, nup, omega));
  RC(stage_out(ctx, u, du, nblk_alloc));
  if (ctx->b_copy_back) RC(stage_out(ctx, b, db, nblk_alloc));
  CK(cudaStreamSynchronize(ctx->stream));
  return engine_check(ctx);
}

extern "C" int srmg_resnorm(srmg_ctx *ctx, double *r, const double *b, const double *u,
                            int64_t nblk_alloc, double s, int op, double k2, int geom,
                            const int8_t bc[9], double *out) {
  RC(check_call_any(ctx, nblk_alloc, op, geom, bc));
  if (!b || !u || !out) return fail(ctx, SRMG_ERR_BADARG, "srmg_resnorm: null argument");
  double *du, *db;
  RC(stage_in(ctx, 0, u, nblk_alloc, &du));
  RC(stage_in(ctx, 1, b, nblk_alloc, &db));
  RC(srmg_resnorm_dev(ctx, r, db, du, nblk_alloc, s, op, k2, geom, bc, out));
  return SRMG_OK;
}

extern "C" int srmg_rhs_level(srmg_ctx *ctx, double *q1, const double *q, int64_t nblk_alloc, int level, int op,
                              int geom) {
  RC(check_call_any(ctx, nblk_alloc, op, geom, nullptr));
  if (!q1 || !q) return fail(ctx, SRMG_ERR_BADARG, "srmg_rhs_level: null field");
  double *dq1, *dq;
  RC(stage_in(ctx, 0, q1, nblk_alloc, &dq1));
  RC(stage_in(ctx, 1, q, nblk_alloc, &dq));
  RC(srmg_rhs_level_dev(ctx, dq1, dq, nblk_alloc, level, op, geom));
  RC(stage_out(ctx, q1, dq1, nblk_alloc));
  CK(cudaStreamSynchronize(ctx->stream));
  return SRMG_OK;
}

extern "C" int srmg_fill_ghost(srmg_ctx *ctx, double *u, int64_t nblk_alloc, int level,
                               const int8_t bc[9]) {
  RC(check_call_any(ctx, nblk_alloc, 0, 0, bc));
  if (!u) return fail(ctx, SRMG_ERR_BADARG, "srmg_fill_ghost: null field");
  double *du;
  RC(stage_in(ctx, 0, u, nblk_alloc, &du));
  RC(srmg_fill_ghost_dev(ctx, du, nblk_alloc, level, bc, 7));
  RC(stage_out(ctx, u, du, nblk_alloc));
  CK(cudaStreamSynchronize(ctx->stream));
  return SRMG_OK;
}

// ------------------------------------------------------------------ explicit instantiations
#define SRMG_INST(T)                                                                         \
  template int srmg::L_fill_ghost<T>(srmg_ctx *, T *, int, const Signs &, int);              \
  template int srmg::L_gs_colour<T>(srmg_ctx *, T *, const T *, int, const OpParams<T> &, int); \
  template int srmg::L_gs_iter<T>(srmg_ctx *, T *, const T *, int, const OpParams<T> &, int,   \
                                  const Signs &);                                            \
  template int srmg::L_residual<T>(srmg_ctx *, T *, const T *, const T *, int, const OpParams<T> &); \
  template int srmg::L_postrestrict<T>(srmg_ctx *, T *, const T *, const T *, int,           \
                                       const OpParams<T> &);                                 \
  template int srmg::L_restrict<T>(srmg_ctx *, T *, int);                                    \
  template int srmg::L_interp_add<T>(srmg_ctx *, T *, const T *, int);                       \
  template int srmg::L_copy<T>(srmg_ctx *, T *, const T *, int);                             \
  template int srmg::L_diff<T>(srmg_ctx *, T *, const T *, const T *, int);
SRMG_INST(double)
SRMG_INST(float)
