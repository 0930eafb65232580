// srmg_items.cu -- per-item operator tables of the persistent engine and the FP64
// direct inverse of each item's coarsest level.
//
// An "item" is one independent problem of a context: a plain tree is one item; a forest
// assembled by srmg_batch_set holds one item per (tree, operator) pair.  The engine
// reads, per item, the operator values of every level (s_l = s 4^-(l-1), the stencil
// centre and -(omega / diagonal), src/laplacian.jl and src/helmholtz.jl), the boundary
// sign table (src/boundary.jl:28-38) and, in mixed mode, P = -s A_1^{-1}.
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

// Gauss-Jordan inverse with partial pivoting (n <= 1024).  Returns false if singular.
bool invert(std::vector<double> &a, int n) {
  std::vector<double> inv((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) inv[(size_t)i * n + i] = 1.0;
  for (int c = 0; c < n; c++) {
    int piv = c;
    double best = std::fabs(a[(size_t)c * n + c]);
    for (int r = c + 1; r < n; r++) {
      const double v = std::fabs(a[(size_t)r * n + c]);
      if (v > best) { best = v; piv = r; }
    }
    if (best < 1e-300) return false;
    if (piv != c)
      for (int k = 0; k < n; k++) {
        std::swap(a[(size_t)c * n + k], a[(size_t)piv * n + k]);
        std::swap(inv[(size_t)c * n + k], inv[(size_t)piv * n + k]);
      }
    const double d = 1.0 / a[(size_t)c * n + c];
    for (int k = 0; k < n; k++) {
      a[(size_t)c * n + k] *= d;
      inv[(size_t)c * n + k] *= d;
    }
    for (int r = 0; r < n; r++) {
      if (r == c) continue;
      const double f = a[(size_t)r * n + c];
      if (f == 0.0) continue;
      for (int k = 0; k < n; k++) {
        a[(size_t)r * n + k] -= f * a[(size_t)c * n + k];
        inv[(size_t)r * n + k] -= f * inv[(size_t)c * n + k];
      }
    }
  }
  a.swap(inv);
  return true;
}

// P = -s_t A_t^{-1} for one item on level t = lt (1 or 2): the level's operator over
// the item's blocks of that level, ghosts resolved through neighbour copies and boundary
// mirrors, assembled on the host, inverted and uploaded (cached by level, operator and
// structure).  *P stays null when the item's level has more than 4 blocks, a face with
// no ghost source on the level (a refinement boundary) or a singular operator.
int item_inverse(srmg_ctx *ctx, int item, const ItemSpec &sp, int geom, int lt, const double **P) {
  *P = nullptr;
  if (lt < 1 || lt > 2 || lt > ctx->nlev) return SRMG_OK;
  const std::vector<int4> &hb = lt == 1 ? ctx->l1_blocks : ctx->l2_blocks;
  const std::vector<int4> &hf = lt == 1 ? ctx->l1_faces : ctx->l2_faces;
  const int2 rg = ctx->it_lrange_host[(size_t)item * ctx->nlev + lt - 1];
  const int nb = rg.y;
  const int n = nb * 256;
  if (nb < 1 || nb > 4) return SRMG_OK;
  auto local = [&](int blk) {
    for (int i = 0; i < nb; i++)
      if (hb[rg.x + i].x == blk) return i;
    return -1;
  };
  const double s = level_scale(sp.s, lt);  // s_l = s / 4^(l-1)
  std::vector<double> key = {(double)lt, s, (double)sp.op, sp.k2, (double)geom, (double)nb};
  for (int i = 0; i < 9; i++) key.push_back(sp.bc[i]);
  for (int i = 0; i < nb; i++) {
    const int4 bk = hb[rg.x + i];
    key.push_back(bk.y);
    key.push_back(bk.z);
    for (int f = 0; f < 4; f++) {
      const int4 fi = hf[4 * (rg.x + i) + f];
      key.push_back(fi.x);
      key.push_back(fi.x == FACE_NEIGHBOR ? local(fi.y) : -1);
    }
  }
  auto hit = ctx->coarse_cache.find(key);
  if (hit != ctx->coarse_cache.end()) {
    *P = (const double *)hit->second.p;
    return SRMG_OK;
  }
  std::vector<double> A((size_t)n * n, 0.0);
  const double centre = (sp.op == SRMG_OP_HELMHOLTZ) ? (-4.0 - s * sp.k2) : -4.0;
  static const int sidx[4] = {3, 5, 1, 7};
  for (int bi = 0; bi < nb; bi++) {
    const int4 bk = hb[rg.x + bi];
    for (int y = 2; y < 18; y++)
      for (int x = 2; x < 18; x++) {
        const int row = bi * 256 + (y - 2) * 16 + (x - 2);
        double wzm = 1, wrm = 1, wrp = 1, wzp = 1;
        if (geom == SRMG_GEOM_CYL1) {
          const int64_t i = x - 1 + 16 * (int64_t)(bk.y - 1);
          wrm = (double)(2 * i - 2) / (double)(2 * i - 1);
          wrp = (double)(2 * i) / (double)(2 * i - 1);
        } else if (geom == SRMG_GEOM_CYL2) {
          const int64_t j = y - 1 + 16 * (int64_t)(bk.z - 1);
          wzm = (double)(2 * j - 2) / (double)(2 * j - 1);
          wzp = (double)(2 * j) / (double)(2 * j - 1);
        }
        A[(size_t)row * n + row] += centre;
        const int nx[4] = {x - 1, x + 1, x, x};
        const int ny[4] = {y, y, y - 1, y + 1};
        const double wv[4] = {wrm, wrp, wzm, wzp};
        for (int q = 0; q < 4; q++) {
          int cx = nx[q], cy = ny[q];
          double coef = wv[q];
          int cb = bi;
          if (cx < 2 || cx > 17 || cy < 2 || cy > 17) {
            const int f = q;  // the face crossed: 0 -r, 1 +r, 2 -z, 3 +z
            const int4 fi = hf[4 * (rg.x + bi) + f];
            if (fi.x == FACE_NEIGHBOR) {
              cb = local(fi.y);
              if (cb < 0) return SRMG_OK;  // neighbour outside the item: no direct solve
              if (f == 0) cx += 16; else if (f == 1) cx -= 16; else if (f == 2) cy += 16; else cy -= 16;
            } else if (fi.x == FACE_BOUNDARY) {
              coef *= (double)sp.bc[sidx[f]];
              if (f == 0) cx = 3 - cx; else if (f == 1) cx = 35 - cx;
              else if (f == 2) cy = 3 - cy; else cy = 35 - cy;
            } else {
              return SRMG_OK;  // no ghost source on this level
            }
          }
          const int col = cb * 256 + (cy - 2) * 16 + (cx - 2);
          A[(size_t)row * n + col] += coef;
        }
      }
  }
  if (!invert(A, n)) return SRMG_OK;
  for (auto &v : A) v *= -s;
  if (ctx->coarse_cache.size() >= 256) {
    CK(cudaStreamSynchronize(ctx->stream));
    for (auto &kv : ctx->coarse_cache) cudaFree(kv.second.p);
    ctx->coarse_cache.clear();
  }
  DevBuf buf;
  RC(ensure(ctx, buf, A.size() * sizeof(double)));
  // on the context's (non-blocking) stream, so that the solves that read it are ordered after it
  CK(cudaMemcpyAsync(buf.p, A.data(), A.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->coarse_cache[key] = buf;
  *P = (const double *)buf.p;
  return SRMG_OK;
}

size_t align8(size_t b) { return (b + 7) & ~size_t(7); }

}  // namespace

std::vector<ItemSpec> srmg::uniform_items(srmg_ctx *ctx, double s, int op, double k2, const int8_t *bc) {
  ItemSpec sp;
  sp.s = s;
  sp.op = op;
  sp.k2 = k2;
  for (int i = 0; i < 9; i++) sp.bc[i] = bc ? bc[i] : 1;
  return std::vector<ItemSpec>((size_t)ctx->nitems, sp);
}

int srmg::direct_top(srmg_ctx *ctx) {
  if (ctx->direct_level == 1 || ctx->nitems != 1 || ctx->D != 2 || ctx->nlev < 2) return 1;
  const int nb2 = ctx->nblk_host[1];
  return nb2 >= 1 && nb2 <= 4 ? 2 : 1;
}

int srmg::prepare_items(srmg_ctx *ctx, const ItemSpec *specs, int geom, double omega, bool want_P,
                        int smooth_level, double smooth_sl, ItemTabs *tabs, int top) {
  const int ni = ctx->nitems;
  const size_t o64 = 0;
  const size_t o32 = align8(o64 + sizeof(double) * kParStride * ni);
  const size_t osg = align8(o32 + sizeof(float) * kParStride * ni);
  const size_t oP = align8(osg + sizeof(int) * ni);
  const size_t total = oP + sizeof(double *) * ni;
  std::vector<char> host(total, 0);
  double *p64 = (double *)(host.data() + o64);
  float *p32 = (float *)(host.data() + o32);
  int *sg = (int *)(host.data() + osg);
  const double **pp = (const double **)(host.data() + oP);
  bool all_P = want_P;
  for (int k = 0; k < ni; k++) {
    const ItemSpec &sp = specs[k];
    for (int l = 1; l < 32; l++) {
      const double sl = (smooth_level > 0 && l == smooth_level) ? smooth_sl : level_scale(sp.s, l);
      const OpParams<double> q = op_params<double>(sp.op, geom, sp.k2, sl, omega);
      const OpParams<float> q32 = op_params<float>(sp.op, geom, sp.k2, sl, omega);
      p64[k * kParStride + l] = q.s;
      p64[k * kParStride + 32 + l] = q.centre;
      p64[k * kParStride + 64 + l] = q.nwc;
      p32[k * kParStride + l] = q32.s;
      p32[k * kParStride + 32 + l] = q32.centre;
      p32[k * kParStride + 64 + l] = q32.nwc;
    }
    sg[k] = 0;
    for (int i = 0; i < 9; i++) sg[k] |= (sp.bc[i] + 1) << (2 * i);
    pp[k] = nullptr;
  }
  if (all_P) {
    for (int k = 0; k < ni && all_P; k++) {
      RC(item_inverse(ctx, k, specs[k], geom, top, &pp[k]));
      if (!pp[k]) all_P = false;
    }
    if (!all_P && top == 2) {  // no usable level-2 inverse: the level-1 solve
      top = 1;
      all_P = true;
      for (int k = 0; k < ni && all_P; k++) {
        RC(item_inverse(ctx, k, specs[k], geom, top, &pp[k]));
        if (!pp[k]) all_P = false;
      }
    }
  }
  if (!all_P)
    for (int k = 0; k < ni; k++) pp[k] = nullptr;
  if (host != ctx->it_tab_host || !ctx->it_tab.p) {
    RC(ensure(ctx, ctx->it_tab, total));
    CK(cudaMemcpyAsync(ctx->it_tab.p, host.data(), total, cudaMemcpyHostToDevice, ctx->stream));
    ctx->it_tab_host.swap(host);
  }
  char *d = (char *)ctx->it_tab.p;
  tabs->par64 = (const double *)(d + o64);
  tabs->par32 = (const float *)(d + o32);
  tabs->sgbits = (const int *)(d + osg);
  tabs->P = all_P ? (const double *const *)(d + oP) : nullptr;
  tabs->P0 = all_P ? pp[0] : nullptr;
  tabs->n0 = all_P ? 256 * ctx->it_lrange_host[top - 1].y : 0;
  tabs->top = all_P ? top : 1;
  return SRMG_OK;
}

int srmg::items_host_reserve(srmg_ctx *ctx) {
  const size_t n = kItemRec * (size_t)ctx->nitems + 8;
  if (ctx->h_items_n >= n) return SRMG_OK;
  if (ctx->h_items) cudaFreeHost(ctx->h_items);
  ctx->h_items = nullptr;
  ctx->h_items_n = 0;
  if (cudaMallocHost((void **)&ctx->h_items, n * sizeof(double)) != cudaSuccess)
    return fail(ctx, SRMG_ERR_NOMEM, "pinned host buffer of %zu doubles", n);
  ctx->h_items_n = n;
  return SRMG_OK;
}

int srmg::items_d2h(srmg_ctx *ctx) {
  const size_t n = kItemRec * (size_t)ctx->nitems + 8;
  CK(cudaMemcpyAsync(ctx->h_items, ctx->istat.p, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  return SRMG_OK;
}

int srmg::read_items(srmg_ctx *ctx) {
  RC(items_host_reserve(ctx));
  RC(items_d2h(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  return engine_check(ctx);
}
