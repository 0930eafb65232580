// srmg_stage.cu -- the stage preparation and post-processing around the field solve,
// on the device, so that a time step need not bring u, b or the charge through the
// host between the streamer update and the solve:
//   * netcharge! (src/streamer.jl:369-373) for the NetIonization chemistry;
//   * restrict_full! (src/restrict.jl:43-47) of a field over the whole tree;
//   * electric_field! (src/multigrid.jl:421-449) with a constant background field.
// For order-2 discretisations rhs_level! (src/multigrid.jl:363-388) is the identity,
// so the net charge itself is the solve's right-hand side.
#include <cmath>

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

// VectorBlockField{2, 16, 2} storage (src/blockfield.jl:84-95): (S+1) x (S+1) x 2 values
// per block, column-major, component d at offset d * (S+1)^2.
constexpr int kSV = kS + 1;
constexpr int kSSV = kSV * kSV;

// q = dot(n, (-1, +1)) = (-1 n_e) + (1 n_ion) on the level's valid cells: the products by
// +-1 are exact, so q is n_ion - n_e rounded once, as the reference computes it.
__global__ void k_netcharge(double *__restrict__ q, const double *__restrict__ ne,
                            const double *__restrict__ nion, LevelView lv) {
  const int64_t total = (int64_t)lv.nblk * 256;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t >> 8), c = (int)(t & 255);
    const int64_t o = (int64_t)lv.blocks[bi].x * kSS + (2 + (c & 15)) + kS * (2 + (c >> 4));
    q[o] = __dadd_rn(-ne[o], nion[o]);
  }
}

// electric_field! on one level, one 256-thread CTA per block pass, thread (x, y) one
// valid cell.  The face value f[I, d] = (u[I - e_d] - u[I]) / h_l + e0[d] is written for
// the cell's lower face along each d, and by the last cell of a row also for the upper
// face (faces G+1 .. G+M+1 along d).  |E| at the cell uses the same two faces per d,
// recomputed with the same operations: sqrt((0 + s_1 s_1 / 4) + s_2 s_2 / 4),
// s_d = f[I, d] + f[I + e_d, d], every operation rounded on its own (no fused
// multiply-add), as in the reference.
__global__ void k_efield(double *__restrict__ e, double *__restrict__ eabs, const double *__restrict__ u,
                         LevelView lv, double hl, double e0r, double e0z) {
  const int x = 2 + (threadIdx.x & 15), y = 2 + (threadIdx.x >> 4);
  for (int bi = blockIdx.x; bi < lv.nblk; bi += gridDim.x) {
    const int64_t X = lv.blocks[bi].x;
    const double *ub = u + X * kSS;
    double *eb = e + X * (2 * kSSV);
    auto face = [&](int d, int fx, int fy) -> double {  // f[(fx, fy), d] in 0-based tile indices
      const double lo = d == 0 ? ub[(fx - 1) + kS * fy] : ub[fx + kS * (fy - 1)];
      return __dadd_rn(__ddiv_rn(__dsub_rn(lo, ub[fx + kS * fy]), hl), d == 0 ? e0r : e0z);
    };
    const double fr0 = face(0, x, y), fr1 = face(0, x + 1, y);
    const double fz0 = face(1, x, y), fz1 = face(1, x, y + 1);
    eb[x + kSV * y] = fr0;
    if (x == 17) eb[(x + 1) + kSV * y] = fr1;
    eb[kSSV + x + kSV * y] = fz0;
    if (y == 17) eb[kSSV + x + kSV * (y + 1)] = fz1;
    const double sr = __dadd_rn(fr0, fr1), sz = __dadd_rn(fz0, fz1);
    double f2 = __dadd_rn(0.0, __ddiv_rn(__dmul_rn(sr, sr), 4.0));
    f2 = __dadd_rn(f2, __ddiv_rn(__dmul_rn(sz, sz), 4.0));
    eabs[X * kSS + x + kS * y] = __dsqrt_rn(f2);
  }
}

int grid_cap(int64_t work, int threads, int cap) {
  const int64_t g = (work + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, cap));
}

}  // namespace

extern "C" int srmg_netcharge_dev(srmg_ctx *ctx, double *q, const double *ne, const double *nion,
                                  int64_t nblk_alloc) {
  RC(check_call(ctx, nblk_alloc, 0, 0, nullptr));
  if (!q || !ne || !nion) return fail(ctx, SRMG_ERR_BADARG, "srmg_netcharge: null field");
  for (int l = 1; l <= ctx->nlev; l++) {
    const int n = ctx->nblk_host[l - 1];
    if (!n) continue;
    k_netcharge<<<grid_cap((int64_t)n * 256, 256, 148 * 8), 256, 0, ctx->stream>>>(q, ne, nion,
                                                                                  ctx->lv[l - 1].view(l));
    ctx->launches++;
  }
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_restrict_full_dev(srmg_ctx *ctx, double *u, int64_t nblk_alloc) {
  RC(check_call(ctx, nblk_alloc, 0, 0, nullptr));
  if (!u) return fail(ctx, SRMG_ERR_BADARG, "srmg_restrict_full: null field");
  for (int l = ctx->nlev; l >= 2; l--) RC(srmg_restrict_level_dev(ctx, u, nblk_alloc, l));
  return SRMG_OK;
}

extern "C" int srmg_electric_field_dev(srmg_ctx *ctx, double *e, double *eabs, const double *u,
                                       int64_t nblk_alloc, double h, const double e0[2]) {
  RC(check_call(ctx, nblk_alloc, 0, 0, nullptr));
  if (!e || !eabs || !u || !e0) return fail(ctx, SRMG_ERR_BADARG, "srmg_electric_field: null argument");
  if (!(h > 0.0) || !std::isfinite(h)) return fail(ctx, SRMG_ERR_BADARG, "srmg_electric_field: h must be > 0");
  for (int l = 1; l <= ctx->nlev; l++) {
    const int n = ctx->nblk_host[l - 1];
    if (!n) continue;
    const double hl = h / (double)((int64_t)1 << (l - 1));  // h / (1 << (level - 1)), exact
    k_efield<<<std::min(n, 148 * 8), 256, 0, ctx->stream>>>(e, eabs, u, ctx->lv[l - 1].view(l), hl, e0[0],
                                                            e0[1]);
    ctx->launches++;
  }
  CK(cudaGetLastError());
  return SRMG_OK;
}

// Host-array variants (the ccall boundary): copies in, the device entry point, copies out.
extern "C" int srmg_netcharge(srmg_ctx *ctx, double *q, const double *ne, const double *nion, int64_t nblk_alloc) {
  RC(check_call(ctx, nblk_alloc, 0, 0, nullptr));
  if (!q || !ne || !nion) return fail(ctx, SRMG_ERR_BADARG, "srmg_netcharge: null field");
  double *dq, *dne, *dni;
  RC(stage_in(ctx, 0, q, nblk_alloc, &dq));
  RC(stage_in(ctx, 1, ne, nblk_alloc, &dne));
  RC(stage_in(ctx, 2, nion, nblk_alloc, &dni));
  RC(srmg_netcharge_dev(ctx, dq, dne, dni, nblk_alloc));
  RC(stage_out(ctx, q, dq, nblk_alloc));
  CK(cudaStreamSynchronize(ctx->stream));
  return SRMG_OK;
}

extern "C" int srmg_electric_field(srmg_ctx *ctx, double *e, double *eabs, const double *u, int64_t nblk_alloc,
                                   double h, const double e0[2]) {
  RC(check_call(ctx, nblk_alloc, 0, 0, nullptr));
  if (!e || !eabs || !u || !e0) return fail(ctx, SRMG_ERR_BADARG, "srmg_electric_field: null argument");
  double *du, *dabs;
  RC(stage_in(ctx, 0, u, nblk_alloc, &du));
  RC(stage_in(ctx, 1, eabs, nblk_alloc, &dabs));
  // the vector field (882 values per block) in the spare slot, copied in so that the
  // faces the reference does not write keep the caller's values
  const size_t vbytes = (size_t)nblk_alloc * 2 * kSSV * sizeof(double);
  RC(ensure(ctx, ctx->f64[2], vbytes));
  double *de = (double *)ctx->f64[2].p;
  CK(cudaMemcpyAsync(de, e, vbytes, cudaMemcpyHostToDevice, ctx->stream));
  RC(srmg_electric_field_dev(ctx, de, dabs, du, nblk_alloc, h, e0));
  CK(cudaMemcpyAsync(e, de, vbytes, cudaMemcpyDeviceToHost, ctx->stream));
  RC(stage_out(ctx, eabs, dabs, nblk_alloc));
  CK(cudaStreamSynchronize(ctx->stream));
  return SRMG_OK;
}
