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

// Assemble the level-1 operator (ghosts resolved through copies and mirrors), invert
// it and upload P = -s A^{-1}.  Cached by (s, op, k2, geom, bc, tree generation).
int prepare_coarse(srmg_ctx *ctx, double s, int op, double k2, int geom, const int8_t *bc) {
  std::vector<double> key = {s, (double)op, k2, (double)geom, (double)ctx->generation};
  for (int i = 0; i < 9; i++) key.push_back(bc ? bc[i] : 1);
  if (ctx->coarse_key == key) return SRMG_OK;
  ctx->coarse_key = key;
  ctx->coarse_ok = false;
  const int nb = ctx->nblk_host[0];
  const int n = nb * 256;
  if (nb < 1 || n > 1024) return SRMG_OK;  // fall back to smoothing at the top
  std::vector<int4> blocks(nb), faces(4 * nb);
  CK(cudaMemcpy(blocks.data(), ctx->lv[0].blocks, nb * sizeof(int4), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(faces.data(), ctx->lv[0].faces, 4 * nb * sizeof(int4), cudaMemcpyDeviceToHost));
  std::vector<int> slot_of(ctx->max_blk + 1, -1);
  for (int i = 0; i < nb; i++) slot_of[blocks[i].x] = i;
  std::vector<double> A((size_t)n * n, 0.0);
  const double centre = (op == SRMG_OP_HELMHOLTZ) ? (-4.0 - s * k2) : -4.0;
  static const int sidx[4] = {3, 5, 1, 7};
  for (int bi = 0; bi < nb; bi++) {
    for (int y = 2; y < 18; y++)
      for (int x = 2; x < 18; x++) {
        const int row = bi * 256 + (y - 2) * 16 + (x - 2);
        double wzm = 1, wrm = 1, wrp = 1, wzp = 1;
        if (geom == 1) {
          const int64_t i = x - 1 + 16 * (int64_t)(blocks[bi].y - 1);
          wrm = (double)(2 * i - 2) / (double)(2 * i - 1);
          wrp = (double)(2 * i) / (double)(2 * i - 1);
        } else if (geom == 2) {
          const int64_t j = y - 1 + 16 * (int64_t)(blocks[bi].z - 1);
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
            const int4 fi = faces[4 * bi + f];
            if (fi.x == FACE_NEIGHBOR) {
              cb = slot_of[fi.y];
              if (cb < 0) return SRMG_OK;
              if (f == 0) cx += 16; else if (f == 1) cx -= 16; else if (f == 2) cy += 16; else cy -= 16;
            } else if (fi.x == FACE_BOUNDARY) {
              coef *= (bc ? (double)bc[sidx[f]] : 1.0);
              if (f == 0) cx = 3 - cx; else if (f == 1) cx = 35 - cx;
              else if (f == 2) cy = 3 - cy; else cy = 35 - cy;
            } else {
              return SRMG_OK;  // refinement boundary at level 1 cannot happen
            }
          }
          const int col = cb * 256 + (cy - 2) * 16 + (cx - 2);
          A[(size_t)row * n + col] += coef;
        }
      }
  }
  if (!invert(A, n)) return SRMG_OK;
  for (auto &v : A) v *= -s;
  RC(ensure(ctx, ctx->coarse_inv, A.size() * sizeof(double)));
  CK(cudaMemcpy(ctx->coarse_inv.p, A.data(), A.size() * sizeof(double), cudaMemcpyHostToDevice));
  ctx->coarse_n = n;
  ctx->coarse_ok = true;
  return SRMG_OK;
}

// FP32 V-cycle with the FP64 direct coarsest-level solve (when available), on the
// per-operation kernels (used when the persistent engine is switched off).  Same
// structure as the reference V-cycle; only the top changes.
int vcycle_mixed(srmg_ctx *ctx, float *e, float *b, float *r, float *u1, double s, int op, double k2,
                 int geom, const Signs &sg, int ndown, int ntop, int nup, double omega) {
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
  if (ctx->coarse_ok) {
    const int n = ctx->coarse_n;
    k_coarse_direct<<<(n + 7) / 8, 256, 0, ctx->stream>>>(e, b, (const double *)ctx->coarse_inv.p,
                                                          ctx->lv[0].view(1), n);
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
  o->inner_cycles = 1;
  o->warm_start = 0;
}

static int solve_fp64(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, double s, int op,
                      double k2, int geom, const int8_t *bc, const srmg_solve_opts *o,
                      srmg_stats *st) {
  const Signs sg = make_signs(bc);
  const size_t bytes = (size_t)nblk_alloc * kSS * sizeof(double);
  RC(ensure(ctx, ctx->f64[4], bytes));
  RC(ensure(ctx, ctx->f64[2], bytes));
  RC(ensure(ctx, ctx->f64[3], bytes));
  double *bw = (double *)ctx->f64[4].p, *r = (double *)ctx->f64[2].p, *u1 = (double *)ctx->f64[3].p;
  CK(cudaMemcpyAsync(bw, b, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  RC(leafnorm_dev<double>(ctx, u, b, s, op, k2, geom, 1, 1));
  const bool aligned = ((reinterpret_cast<uintptr_t>(u) | reinterpret_cast<uintptr_t>(bw) |
                         reinterpret_cast<uintptr_t>(r) | reinterpret_cast<uintptr_t>(u1)) & 15) == 0;
  if (ctx->use_engine && aligned && o->ndown >= 1 && o->ntop >= 1 && o->nup >= 1 && ctx->nlev <= 30) {
    // the whole tolerance loop in one persistent launch
    RC(read_small(ctx, 2));
    const double bn = ctx->h_small[1] > 0 ? ctx->h_small[1] : 1.0;
    st->bnorm = ctx->h_small[1];
    EngineRun run;
    run.max_cycles = std::max(1, o->max_cycles);
    run.tol_abs = o->tol * bn;
    RC(engine_vcycle<double>(ctx, u, bw, u1, r, s, op, k2, geom, sg, 0, o->ndown, o->ntop, o->nup, o->omega,
                             &run));
    RC(read_small(ctx, 12));
    const double *out = ctx->h_small + 8;
    st->rel_residual = out[0] / bn;
    st->initial_rel = out[3] / bn;
    st->cycles = (int)out[2];
    if (!std::isfinite(st->rel_residual))
      return fail(ctx, SRMG_ERR_DIVERGED, "residual is not finite after %d cycles", st->cycles);
    return SRMG_OK;
  }
  RC(leafnorm_dev<double>(ctx, u, bw, s, op, k2, geom, 0, 0));
  RC(read_small(ctx, 2));
  const double bn = ctx->h_small[1] > 0 ? ctx->h_small[1] : 1.0;
  st->bnorm = ctx->h_small[1];
  double rel = ctx->h_small[0] / bn;
  st->initial_rel = rel;
  int c = 0;
  while (rel > o->tol && c < o->max_cycles) {
    RC(vcycle_dev<double>(ctx, u, bw, r, u1, s, op, k2, geom, sg, 0, o->ndown, o->ntop, o->nup, o->omega));
    c++;
    RC(leafnorm_dev<double>(ctx, u, bw, s, op, k2, geom, 0, 0));
    RC(read_small(ctx, 1));
    const double nrel = ctx->h_small[0] / bn;
    if (!std::isfinite(nrel)) {
      st->cycles = c;
      st->rel_residual = nrel;
      return fail(ctx, SRMG_ERR_DIVERGED, "residual is not finite after %d cycles", c);
    }
    rel = nrel;
  }
  st->cycles = c;
  st->rel_residual = rel;
  return SRMG_OK;
}

// The whole mixed-precision solve in one persistent launch: every defect-correction
// step (FP64 update, composite consistency, FP64 defect and its leaf norm, FP32 V-cycle
// with the FP64 direct coarsest-level solve) runs on the device until the defect norm
// is <= tol * leafnorm(b).
static int solve_mixed_engine(srmg_ctx *ctx, double *u, const double *b, double s, int op, double k2,
                              int geom, const int8_t *bc, const srmg_solve_opts *o, srmg_stats *st,
                              float *e, float *be, float *r, float *u1, double bn) {
  const Signs sg = make_signs(bc);
  EngineRun run;
  run.coarse_P = ctx->coarse_ok ? (const double *)ctx->coarse_inv.p : nullptr;
  run.coarse_n = ctx->coarse_ok ? ctx->coarse_n : 0;
  run.u64 = u;
  run.b64 = b;
  run.apply_update = 0;
  run.max_cycles = std::max(1, o->max_cycles);
  run.tol_abs = o->tol * bn;
  RC(engine_vcycle<float>(ctx, e, be, u1, r, s, op, k2, geom, sg, 0, o->ndown, o->ntop, o->nup, o->omega,
                          &run));
  RC(read_small(ctx, 12));
  const double *out = ctx->h_small + 8;
  st->rel_residual = out[0] / bn;
  st->initial_rel = out[3] / bn;
  st->cycles = (int)out[2];
  st->outer = (int)out[2];
  if (!std::isfinite(st->rel_residual))
    return fail(ctx, SRMG_ERR_DIVERGED, "mixed solve: defect norm is not finite after %d steps", st->cycles);
  return SRMG_OK;
}

static int solve_mixed(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, double s, int op,
                       double k2, int geom, const int8_t *bc, const srmg_solve_opts *o,
                       srmg_stats *st) {
  const Signs sg = make_signs(bc);
  const size_t b32 = (size_t)nblk_alloc * kSS * sizeof(float);
  for (int i = 0; i < 4; i++) RC(ensure(ctx, ctx->f32[i], b32));
  float *e = (float *)ctx->f32[0].p, *be = (float *)ctx->f32[1].p, *r = (float *)ctx->f32[2].p,
        *u1 = (float *)ctx->f32[3].p;
  CK(cudaMemsetAsync(r, 0, b32, ctx->stream));
  CK(cudaMemsetAsync(u1, 0, b32, ctx->stream));
  RC(prepare_coarse(ctx, s, op, k2, geom, bc));
  RC(leafnorm_dev<double>(ctx, u, b, s, op, k2, geom, 1, 1));
  const bool aligned = ((reinterpret_cast<uintptr_t>(u) | reinterpret_cast<uintptr_t>(b)) & 15) == 0;
  if (ctx->use_engine && aligned && o->ndown >= 1 && o->nup >= 1 && o->ntop >= 1 && ctx->nlev <= 30) {
    RC(read_small(ctx, 2));
    const double bn = ctx->h_small[1] > 0 ? ctx->h_small[1] : 1.0;
    st->bnorm = ctx->h_small[1];
    return solve_mixed_engine(ctx, u, b, s, op, k2, geom, bc, o, st, e, be, r, u1, bn);
  }
  // per-operation kernels
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
      RC(vcycle_mixed(ctx, e, be, r, u1, s, op, k2, geom, sg, o->ndown, o->ntop, o->nup, o->omega));
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
      return fail(ctx, SRMG_ERR_DIVERGED, "mixed solve diverged after %d steps", outer);
    }
    prev = nrel;
    rel = nrel;
  }
  st->cycles = cycles;
  st->outer = outer;
  st->rel_residual = rel;
  return SRMG_OK;
}

extern "C" int srmg_solve_dev(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, double s,
                              int op, double k2, int geom, const int8_t bc[9],
                              const srmg_solve_opts *opts, srmg_stats *stats) {
  RC(check_call(ctx, nblk_alloc, op, geom, bc));
  if (!u || !b) return fail(ctx, SRMG_ERR_BADARG, "srmg_solve: null field");
  srmg_solve_opts o;
  if (opts) o = *opts; else srmg_solve_opts_default(&o);
  if (!(o.tol > 0) || o.max_cycles < 0 || o.ndown < 0 || o.nup < 0 || o.ntop < 0)
    return fail(ctx, SRMG_ERR_BADARG, "srmg_solve: bad options");
  srmg_stats st;
  memset(&st, 0, sizeof st);
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  int rc;
  if (o.mode == SRMG_MODE_FP64) rc = solve_fp64(ctx, u, b, nblk_alloc, s, op, k2, geom, bc, &o, &st);
  else if (o.mode == SRMG_MODE_MIXED) rc = solve_mixed(ctx, u, b, nblk_alloc, s, op, k2, geom, bc, &o, &st);
  else rc = fail(ctx, SRMG_ERR_BADARG, "unknown solve mode %d", o.mode);
  cudaEventRecord(ctx->ev1, ctx->stream);
  cudaEventSynchronize(ctx->ev1);
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  st.device_ms = ms;
  st.status = rc;
  if (stats) *stats = st;
  if (rc) return rc;
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_solve(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, double s, int op,
                          double k2, int geom, const int8_t bc[9], const srmg_solve_opts *opts,
                          srmg_stats *stats) {
  RC(check_call(ctx, nblk_alloc, op, geom, bc));
  if (!u || !b) return fail(ctx, SRMG_ERR_BADARG, "srmg_solve: null field");
  double *du, *db;
  RC(stage_in(ctx, 0, u, nblk_alloc, &du));
  RC(stage_in(ctx, 1, b, nblk_alloc, &db));
  RC(srmg_solve_dev(ctx, du, db, nblk_alloc, s, op, k2, geom, bc, opts, stats));
  RC(stage_out(ctx, u, du, nblk_alloc));
  CK(cudaStreamSynchronize(ctx->stream));
  return SRMG_OK;
}
