// srmg_streamer.cu -- a minimal streamer stepper that produces the solve pairs the
// learned warm start trains on: electrons drift and diffuse in the field of the
// solved potential plus a uniform applied field, with Koren-limited upwind fluxes
// (src/fluid.jl:8-94: flux!, fluxderivs!), and ionisation/attachment feed two immobile
// ion species (the reference's NetIonization chemistry drifts only electrons,
// src/chemistry.jl:29-82; here positive and negative ions are both kept).
//
// Geometry: cylindrical (r = dim 1, z = dim 2), cell centres r_i = (i - 1/2) h.  The
// divergence of a face flux F is (r_{i+1/2} F_{i+1/2} - r_{i-1/2} F_{i-1/2}) / (r_i h)
// + (F_{j+1/2} - F_{j-1/2}) / h; the axis face has r = 0.  Every block needs its 2-cell
// ghost halo of n_e and of phi filled (the face at a block edge reads 2 cells on each
// side).  Rates are computed on the valid cells of every leaf-holding block.
#include <cmath>
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

constexpr double kE = 1.6021766208e-19;      // elementary charge (src/constants.jl:55)
constexpr double kEps0 = 8.854187817620389e-12;  // (src/constants.jl:56)

// Koren limiter psi(r) = max(0, min(2r, (1 + 2r)/3, 2)) on the slope ratio r.
__device__ __forceinline__ double koren(double r) { return fmax(0.0, fmin(fmin(2.0 * r, (1.0 + 2.0 * r) / 3.0), 2.0)); }

// Face value of n upwind of a face between cells a (left) and b (right), velocity v:
// second-order reconstruction limited by Koren (n0 = left of a, n3 = right of b).
__device__ __forceinline__ double face_value(double v, double n0, double na, double nb, double n3) {
  if (v >= 0.0) {
    const double d = nb - na;
    const double r = d != 0.0 ? (na - n0) / d : 0.0;
    return na + 0.5 * koren(r) * d;
  }
  const double d = na - nb;
  const double r = d != 0.0 ? (nb - n3) / d : 0.0;
  return nb + 0.5 * koren(r) * d;
}

__device__ __forceinline__ void atomic_max_pos(double *addr, double v) {
  // non-negative doubles order like their bit patterns as signed integers
  atomicMax(reinterpret_cast<unsigned long long *>(addr), (unsigned long long)__double_as_longlong(v));
}

struct Phys {
  double mu, D;        // electron mobility (m^2/Vs) and diffusion (m^2/s)
  double E0;           // applied field along +z (V/m)
  double alpha_A, alpha_B;  // ionisation alpha = A exp(-B/|E|) (1/m, V/m)
  double eta;          // attachment (1/m)
};

// Rates on the valid cells of the leaf-holding blocks; maxima of |v| and n_e into mx.
__global__ void k_streamer_rates(const double *__restrict__ ne, const double *__restrict__ phi, const int2 *leaf,
                                 int nleaf, const int4 *__restrict__ info, double h1, Phys P,
                                 double *__restrict__ dne, double *__restrict__ dnp, double *__restrict__ dnn,
                                 double *__restrict__ mx) {
  const int64_t total = (int64_t)nleaf * 256;
  double vmax = 0.0, nmax = 0.0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(t >> 8), c = (int)(t & 255);
    const int2 lb = leaf[k];
    const int4 bi = info[lb.x];
    const double h = h1 / (double)((int64_t)1 << (lb.y - 1));
    const int x = 2 + (c & 15), y = 2 + (c >> 4);
    const int64_t base = (int64_t)lb.x * kSS;
    const double *n = ne + base, *f = phi + base;
    auto N = [&](int a, int b) { return n[a + kS * b]; };
    auto F = [&](int a, int b) { return f[a + kS * b]; };
    // global 1-based r index of this cell; face radii r_{i-1/2} = (i - 1) h, r_{i+1/2} = i h
    const int64_t ig = x - 1 + 16 * (int64_t)(bi.x - 1);
    const double rc = ((double)ig - 0.5) * h, rm = (double)(ig - 1) * h, rp = (double)ig * h;
    // fields at the four faces (E = -grad phi, plus the applied field on z faces)
    const double Erm = -(F(x, y) - F(x - 1, y)) / h, Erp = -(F(x + 1, y) - F(x, y)) / h;
    const double Ezm = -(F(x, y) - F(x, y - 1)) / h + P.E0, Ezp = -(F(x, y + 1) - F(x, y)) / h + P.E0;
    const double vrm = -P.mu * Erm, vrp = -P.mu * Erp, vzm = -P.mu * Ezm, vzp = -P.mu * Ezp;
    const double Frm = vrm * face_value(vrm, N(x - 2, y), N(x - 1, y), N(x, y), N(x + 1, y)) -
                       P.D * (N(x, y) - N(x - 1, y)) / h;
    const double Frp = vrp * face_value(vrp, N(x - 1, y), N(x, y), N(x + 1, y), N(x + 2, y)) -
                       P.D * (N(x + 1, y) - N(x, y)) / h;
    const double Fzm = vzm * face_value(vzm, N(x, y - 2), N(x, y - 1), N(x, y), N(x, y + 1)) -
                       P.D * (N(x, y) - N(x, y - 1)) / h;
    const double Fzp = vzp * face_value(vzp, N(x, y - 1), N(x, y), N(x, y + 1), N(x, y + 2)) -
                       P.D * (N(x, y + 1) - N(x, y)) / h;
    const double div = (rp * Frp - rm * Frm) / (rc * h) + (Fzp - Fzm) / h;
    // cell-centred field magnitude for the sources
    const double Er = 0.5 * (Erm + Erp), Ez = 0.5 * (Ezm + Ezp);
    const double Em = sqrt(Er * Er + Ez * Ez);
    const double ion = P.alpha_A * exp(-P.alpha_B / fmax(Em, 1.0)) * P.mu * Em * N(x, y);
    const double att = P.eta * P.mu * Em * N(x, y);
    const int64_t o = base + x + kS * y;
    dne[o] = -div + ion - att;
    dnp[o] = ion;
    dnn[o] = att;
    vmax = fmax(vmax, fmax(fmax(fabs(vrm), fabs(vrp)), fmax(fabs(vzm), fabs(vzp))));
    nmax = fmax(nmax, N(x, y));
  }
  for (int off = 16; off > 0; off >>= 1) {
    vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, off));
    nmax = fmax(nmax, __shfl_xor_sync(0xffffffffu, nmax, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_pos(mx, vmax);
    atomic_max_pos(mx + 1, nmax);
  }
}

__global__ void k_streamer_update(double *__restrict__ ne, double *__restrict__ np, double *__restrict__ nn,
                                  const double *__restrict__ dne, const double *__restrict__ dnp,
                                  const double *__restrict__ dnn, const int2 *leaf, int nleaf, double dt) {
  const int64_t total = (int64_t)nleaf * 256;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(t >> 8), c = (int)(t & 255);
    const int64_t o = (int64_t)leaf[k].x * kSS + (2 + (c & 15)) + kS * (2 + (c >> 4));
    ne[o] = fmax(0.0, ne[o] + dt * dne[o]);
    np[o] = np[o] + dt * dnp[o];
    nn[o] = nn[o] + dt * dnn[o];
  }
}

}  // namespace

// One forward-Euler step of the densities (n_e, n_+, n_-) on the leaf-holding blocks.
// n_e and phi must have their ghosts filled.  dt = min(dt_max, cfl * h_min / max|v|,
// cfl * h_min^2 / (4 D), cfl * eps0 / (e mu max n_e)) is returned in *dt_out.  work:
// 3 device fields of nblk_alloc blocks (rates), 2 doubles (maxima).
extern "C" int srmg_streamer_step_dev(srmg_ctx *ctx, double *ne, double *npos, double *nneg, const double *phi,
                                      int64_t nblk_alloc, double h1, double E0, double mu, double D,
                                      double alpha_A, double alpha_B, double eta, double cfl, double dt_max,
                                      double *work, double *dt_out) {
  RC(check_call(ctx, nblk_alloc, 0, 0, nullptr));
  if (!ne || !npos || !nneg || !phi || !work || !dt_out || !(h1 > 0) || !(cfl > 0) || !(dt_max > 0))
    return fail(ctx, SRMG_ERR_BADARG, "srmg_streamer_step_dev: bad arguments");
  const int64_t nval = nblk_alloc * (int64_t)kSS;
  double *dne = work, *dnp = work + nval, *dnn = work + 2 * nval, *mx = work + 3 * nval;
  CK(cudaMemsetAsync(mx, 0, 2 * sizeof(double), ctx->stream));
  Phys P{mu, D, E0, alpha_A, alpha_B, eta};
  const int n = ctx->nleaf;
  const int grid = (int)std::min<int64_t>(4096, ((int64_t)n * 256 + 255) / 256);
  k_streamer_rates<<<grid, 256, 0, ctx->stream>>>(ne, phi, ctx->d_leaf, n, ctx->d_info, h1, P, dne, dnp, dnn, mx);
  CK(cudaGetLastError());
  double hmx[2];
  CK(cudaMemcpyAsync(hmx, mx, sizeof hmx, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  int lmax = 1;
  for (int l = 1; l <= ctx->nlev; l++)
    if (ctx->nblk_host[l - 1] > 0) lmax = l;
  const double hmin = h1 / (double)((int64_t)1 << (lmax - 1));
  double dt = dt_max;
  if (hmx[0] > 0) dt = std::min(dt, cfl * hmin / hmx[0]);
  if (D > 0) dt = std::min(dt, cfl * hmin * hmin / (4.0 * D));
  if (hmx[1] > 0) dt = std::min(dt, cfl * kEps0 / (kE * mu * hmx[1]));
  k_streamer_update<<<grid, 256, 0, ctx->stream>>>(ne, npos, nneg, dne, dnp, dnn, ctx->d_leaf, n, dt);
  CK(cudaGetLastError());
  *dt_out = dt;
  return SRMG_OK;
}
