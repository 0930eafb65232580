// srmg_streamer.cu -- the electron transport and chemistry inside derivs!
// (src/streamer.jl:292-366) and the SSPRK3 stage combinations of step!
// (src/streamer.jl:386-425), on the device, for the streamer runs that generate the
// learned warm start's training pairs:
//   * flux! with the Koren scheme (src/fluid.jl:44-94): per leaf block and per face of
//     validindices(e, d), the upwind value n_u + koren_limited(n_u - n_u2, n_d - n_u)
//     (src/fluid.jl:265-280) times the drift velocity -mu E, plus the diffusion flux, and
//     the block's largest stable time step (CFL, diffusion, Maxwell relaxation);
//   * restrict_flux! (src/connectivity.jl:327-360): at every refinement boundary the
//     coarse block's face flux is the mean of the two fine face fluxes it covers;
//   * chemderivs! for NetIonization (src/chemistry.jl:29-82) with the MinimalTransportModel
//     (src/transport.jl:9-35): ionisation before the (empty) photoionization, attachment
//     after it, for both species (electrons and net positive ions);
//   * fluxderivs! (src/fluid.jl:8-30): the flux divergence with the geometry factors of
//     src/geometry.jl:27-29, accumulated face by face in the reference's order;
//   * the three SSPRK3 combinations n + dn1 dt, n + (dn1 dt/4 + dn2 dt/4),
//     n + ((dn1 dt/6 + dn2 dt/6) + dn3 2dt/3).
// Every operation is rounded on its own (no fused multiply-add), as in the reference,
// so fluxes, time steps and stage combinations are bit-exact against a restatement with
// IEEE double arithmetic; the chemistry calls exp(), which may differ in the last bit.
//
// The vector fields (e, flux) use the VectorBlockField{2, 16, 2} storage
// (src/blockfield.jl:84-95): 21 x 21 values per component, component d at offset 441 d,
// 882 values per block; face (x, y) of component d (0-based local indices) is the face
// between cell (x, y) - e_d and cell (x, y).
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

constexpr int kSV = kS + 1;
constexpr int kSSV = kSV * kSV;
constexpr int kFacesPerDim = (kM + 1) * kM;  // 17 x 16 faces of validindices(e, d)

constexpr double kElemCharge = 1.6021766208e-19;  // src/constants.jl:55
constexpr double kEpsilon0 = 8.854187817620389e-12;  // src/constants.jl:56

__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

// koren_limited(a, b) = psi(a / b) b (src/fluid.jl:274-280).
__device__ __forceinline__ double koren_limited(double a, double b) {
  if (mul(a, b) < 0.0) return 0.0;
  if (fabs(a) > fabs(mul(4.0, b))) return b;
  if (fabs(mul(10.0, a)) > fabs(mul(4.0, b))) return add(dvd(b, 3.0), dvd(a, 6.0));
  return a;
}

// Leaf blocks (no child in any subblock: isleaf, src/tree.jl:105-115) among the blocks
// holding a leaf cell.
__device__ __forceinline__ bool leaf_block(const int4 *info, int X) { return (info[X].z & 15) == 0; }

// Non-negative doubles order like their bit patterns as unsigned integers.
__device__ __forceinline__ void atomic_min_nonneg(double *addr, double v) {
  atomicMin(reinterpret_cast<unsigned long long *>(addr), (unsigned long long)__double_as_longlong(v));
}

// flux! (Koren) on the leaf blocks: one 256-thread CTA per block pass, the 544 faces of
// the block strided over its threads.  ne needs 2 ghost layers, eabs 1.
__global__ void k_streamer_flux(double *__restrict__ flux, double *__restrict__ maxdt_blk,
                                double *__restrict__ maxdt_min, const double *__restrict__ ne,
                                const double *__restrict__ e, const double *__restrict__ eabs,
                                const int2 *__restrict__ leaf, int nleaf, const int4 *__restrict__ info,
                                double h1, srmg_transport tr) {
  __shared__ double s_min[8];
  const double maxwell = kEpsilon0 / kElemCharge;  // (co.epsilon_0 / co.elementary_charge)
  for (int k = blockIdx.x; k < nleaf; k += gridDim.x) {
    const int X = leaf[k].x;
    if (!leaf_block(info, X)) continue;  // uniform per CTA
    const double h = dvd(h1, (double)((int64_t)1 << (leaf[k].y - 1)));  // h /= 1 << (level - 1)
    const double *n = ne + (int64_t)X * kSS;
    const double *ea = eabs + (int64_t)X * kSS;
    const double *eb = e + (int64_t)X * 2 * kSSV;
    double *fb = flux + (int64_t)X * 2 * kSSV;
    double md = INFINITY;
    for (int q = threadIdx.x; q < 2 * kFacesPerDim; q += blockDim.x) {
      const int d = q >= kFacesPerDim;
      const int r = q - d * kFacesPerDim;
      // face I = (x, y) of component d; I1 = I - e_d
      const int x = d ? 2 + (r & 15) : 2 + r % 17;
      const int y = d ? 2 + (r >> 4) : 2 + r / 17;
      const int st = d ? kS : 1;  // e_d in tile offsets
      const int o = x + kS * y;
      const double ed = eb[d * kSSV + x + kSV * y];
      const double eabs1 = dvd(add(ea[o], ea[o - st]), 2.0);
      const double mu = tr.mu, diff = tr.D;  // mobility / diffusion of the minimal model, theta = 1
      const double v = mul(-ed, mu);
      const int sv = signbit(v) ? -1 : 1;
      // downstream, upstream and twice-upstream cells along d
      const int od = o + st * (sv == 1 ? 0 : -1);
      const int ou = o + st * (sv == 1 ? -1 : 0);
      const int ou2 = o + st * (sv == 1 ? -2 : 1);
      double F = mul(v, add(n[ou], koren_limited(sub(n[ou], n[ou2]), sub(n[od], n[ou]))));
      const double tmaxwell = dvd(mul(maxwell, eabs1), fabs(F));
      F = add(F, dvd(mul(diff, sub(n[o - st], n[o])), h));
      fb[d * kSSV + x + kSV * y] = F;
      md = fmin(md, fmin(fmin(dvd(h, fabs(v)), dvd(dvd(mul(h, h), diff), 4.0)), tmaxwell));
    }
    for (int off = 16; off > 0; off >>= 1) md = fmin(md, __shfl_xor_sync(0xffffffffu, md, off));
    if ((threadIdx.x & 31) == 0) s_min[threadIdx.x >> 5] = md;
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = s_min[0];
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmin(m, s_min[w]);
      if (maxdt_blk) maxdt_blk[X] = m;
      if (maxdt_min) atomic_min_nonneg(maxdt_min, m);
    }
    __syncthreads();
  }
}

// restrict_flux! over one level's refinement-boundary faces: thread (block, face, k)
// sets the coarse block's face k (0..7) of the half `subblock` covers to the mean of
// the two fine faces 2k, 2k + 1: f = ((0 + f_2k) + f_2k+1) / 2.
__global__ void k_restrict_flux(double *__restrict__ flux, LevelView lv) {
  const int64_t total = (int64_t)lv.nblk * 32;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t >> 5), f = (int)(t >> 3) & 3, k = (int)(t & 7);
    const int4 fi = lv.faces[4 * bi + f];
    if (fi.x != FACE_REFBND) continue;
    const int d = f >> 1;  // the face's dimension: 0 for -r/+r, 1 for -z/+z
    const int fine_n = (f & 1) ? 2 + kM : 2, coarse_n = (f & 1) ? 2 : 2 + kM;  // normal face index
    const int sb = d == 0 ? fi.w : fi.z;  // the tangential half
    const int ct = 2 + 8 * (sb - 1) + k, ft = 2 + 2 * k;
    const double *src = flux + (int64_t)lv.blocks[bi].x * 2 * kSSV + d * kSSV;
    double *dst = flux + (int64_t)fi.y * 2 * kSSV + d * kSSV;
    auto at = [&](int nrm, int tan) { return d == 0 ? nrm + kSV * tan : tan + kSV * nrm; };
    const double s = add(add(0.0, src[at(fine_n, ft)]), src[at(fine_n, ft + 1)]);
    dst[at(coarse_n, ct)] = dvd(s, 2.0);
  }
}

// chemderivs! (init, then add) and fluxderivs! on the valid cells of the leaf blocks:
// dni = pre + post; dne = (((pre + post) + lower-r) - upper-r) + lower-z) - upper-z,
// each face term (factor F) / h, factor = |1 + delta / (2 J - 1)| along the radial
// dimension (1 along the others and in Cartesian geometry).
__global__ void k_streamer_rates(double *__restrict__ dne, double *__restrict__ dni,
                                 const double *__restrict__ ne, const double *__restrict__ eabs,
                                 const double *__restrict__ flux, const int2 *__restrict__ leaf, int nleaf,
                                 const int4 *__restrict__ info, double h1, int geom, srmg_transport tr) {
  const int64_t total = (int64_t)nleaf * 256;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(t >> 8), c = (int)(t & 255);
    const int X = leaf[k].x;
    const int4 bi = info[X];
    if ((bi.z & 15) != 0) continue;
    const double h = dvd(h1, (double)((int64_t)1 << (leaf[k].y - 1)));
    const int x = 2 + (c & 15), y = 2 + (c >> 4);
    const int64_t o = (int64_t)X * kSS + x + kS * y;
    const double n1 = ne[o], E = eabs[o];
    // NetIonization, MinimalTransportModel: mobility mu, townsend ai exp(-Ei / E),
    // attachment aa exp(-Ea / E)
    const double pre = mul(mul(mul(tr.mu, E), n1), mul(tr.ai, exp(dvd(-tr.Ei, E))));
    const double post = mul(mul(mul(-tr.mu, E), n1), mul(tr.aa, exp(dvd(-tr.Ea, E))));
    const double chem = add(pre, post);
    dni[o] = chem;
    const double *fb = flux + (int64_t)X * 2 * kSSV;
    const int64_t Jr = gidx(bi.x, x), Jz = gidx(bi.y, y);
    auto fac = [&](int dim, int delta) -> double {  // factor(geom, J, delta e_dim)
      const bool radial = (geom == 1 && dim == 0) || (geom == 2 && dim == 1);
      if (geom == 0) return 1.0;
      const int64_t J = dim == 0 ? Jr : Jz;
      const double q = radial ? dvd((double)delta, (double)(2 * J - 1)) : 0.0;
      return fabs(add(1.0, q));
    };
    double v = chem;
    v = add(v, dvd(mul(fac(0, -1), fb[x + kSV * y]), h));
    v = sub(v, dvd(mul(fac(0, 1), fb[(x + 1) + kSV * y]), h));
    v = add(v, dvd(mul(fac(1, -1), fb[kSSV + x + kSV * y]), h));
    v = sub(v, dvd(mul(fac(1, 1), fb[kSSV + x + kSV * (y + 1)]), h));
    dne[o] = v;
  }
}

__global__ void k_init_min(double *m) { *m = INFINITY; }

// The SSPRK3 stage combinations of step! (src/streamer.jl:400-413), elementwise.
__global__ void k_ssprk3(double *__restrict__ out, const double *__restrict__ n, const double *__restrict__ d1,
                         const double *__restrict__ d2, const double *__restrict__ d3, int64_t count, double dt,
                         int stage) {
  const double dt1 = dvd(dt, 4.0), dt6 = dvd(dt, 6.0), dt23 = dvd(mul(2.0, dt), 3.0);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
    double inc;
    if (stage == 1) inc = mul(d1[i], dt);
    else if (stage == 2) inc = add(mul(d1[i], dt1), mul(d2[i], dt1));
    else inc = add(add(mul(d1[i], dt6), mul(d2[i], dt6)), mul(d3[i], dt23));
    out[i] = add(n[i], inc);
  }
}

int grid_of(int64_t work, int threads, int cap) {
  const int64_t g = (work + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, cap));
}

int check_transport(srmg_ctx *ctx, const srmg_transport *tr, const char *who) {
  if (!tr) return fail(ctx, SRMG_ERR_BADARG, "%s: null transport model", who);
  const double v[6] = {tr->mu, tr->D, tr->ai, tr->Ei, tr->aa, tr->Ea};
  for (double a : v)
    if (!std::isfinite(a)) return fail(ctx, SRMG_ERR_BADARG, "%s: transport values must be finite", who);
  if (!(tr->D > 0)) return fail(ctx, SRMG_ERR_BADARG, "%s: diffusion must be > 0", who);
  return SRMG_OK;
}

}  // namespace

extern "C" int srmg_streamer_flux_dev(srmg_ctx *ctx, double *flux, double *maxdt_blk, double *maxdt_min,
                                      const double *ne, const double *e, const double *eabs, int64_t nblk_alloc,
                                      double h, const srmg_transport *tr) {
  RC(check_call(ctx, nblk_alloc, 0, 0, nullptr));
  if (!flux || !ne || !e || !eabs) return fail(ctx, SRMG_ERR_BADARG, "srmg_streamer_flux_dev: null field");
  if (!(h > 0.0) || !std::isfinite(h)) return fail(ctx, SRMG_ERR_BADARG, "srmg_streamer_flux_dev: h must be > 0");
  RC(check_transport(ctx, tr, "srmg_streamer_flux_dev"));
  if (maxdt_min) {
    k_init_min<<<1, 1, 0, ctx->stream>>>(maxdt_min);
    ctx->launches++;
  }
  if (ctx->nleaf > 0) {
    k_streamer_flux<<<std::min(ctx->nleaf, 148 * 8), 256, 0, ctx->stream>>>(
        flux, maxdt_blk, maxdt_min, ne, e, eabs, ctx->d_leaf, ctx->nleaf, ctx->d_info, h, *tr);
    ctx->launches++;
  }
  for (int l = 2; l <= ctx->nlev; l++) {
    if (!((ctx->refbnd_levels >> l) & 1)) continue;
    const int n = ctx->nblk_host[l - 1];
    k_restrict_flux<<<grid_of((int64_t)n * 32, 256, 148 * 8), 256, 0, ctx->stream>>>(flux, ctx->lv[l - 1].view(l));
    ctx->launches++;
  }
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_streamer_rates_dev(srmg_ctx *ctx, double *dne, double *dni, const double *ne,
                                       const double *eabs, const double *flux, int64_t nblk_alloc, double h,
                                       int geom, const srmg_transport *tr) {
  RC(check_call(ctx, nblk_alloc, 0, 0, nullptr));
  if (!dne || !dni || !ne || !eabs || !flux) return fail(ctx, SRMG_ERR_BADARG, "srmg_streamer_rates_dev: null field");
  if (!(h > 0.0) || !std::isfinite(h)) return fail(ctx, SRMG_ERR_BADARG, "srmg_streamer_rates_dev: h must be > 0");
  if (geom < 0 || geom > 2) return fail(ctx, SRMG_ERR_BADARG, "srmg_streamer_rates_dev: geom must be 0, 1 or 2");
  RC(check_transport(ctx, tr, "srmg_streamer_rates_dev"));
  if (ctx->nleaf > 0) {
    k_streamer_rates<<<grid_of((int64_t)ctx->nleaf * 256, 256, 148 * 16), 256, 0, ctx->stream>>>(
        dne, dni, ne, eabs, flux, ctx->d_leaf, ctx->nleaf, ctx->d_info, h, geom, *tr);
    ctx->launches++;
  }
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_ssprk3_stage_dev(srmg_ctx *ctx, double *out, const double *n, const double *dn1,
                                     const double *dn2, const double *dn3, int64_t count, double dt, int stage) {
  if (!ctx) return SRMG_ERR_BADARG;
  if (stage < 1 || stage > 3) return fail(ctx, SRMG_ERR_BADARG, "srmg_ssprk3_stage_dev: stage must be 1, 2 or 3");
  if (!out || !n || !dn1 || (stage >= 2 && !dn2) || (stage == 3 && !dn3) || count < 0)
    return fail(ctx, SRMG_ERR_BADARG, "srmg_ssprk3_stage_dev: bad arguments");
  if (!std::isfinite(dt)) return fail(ctx, SRMG_ERR_BADARG, "srmg_ssprk3_stage_dev: dt must be finite");
  CK(cudaSetDevice(ctx->device));
  if (count > 0) {
    k_ssprk3<<<grid_of(count, 256, 148 * 16), 256, 0, ctx->stream>>>(out, n, dn1, dn2, dn3, count, dt, stage);
    ctx->launches++;
  }
  CK(cudaGetLastError());
  return SRMG_OK;
}
