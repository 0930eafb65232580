// srmg3.cu -- the multigrid field solve on three-dimensional block trees (D = 3,
// CartesianGeometry: the only geometry with 3D stencils in the reference,
// src/laplacian.jl:274-340, src/helmholtz.jl:74-100).
//
// A 3D context (srmg_create with D = 3) holds an octree uploaded by srmg_set_tree3 and
// runs the per-operation path in FP64: every generic entry point (vcycle, fmg,
// resnorm, the ghost fills, the per-level operations, rhs_level, FP64 solve) checks
// the context's dimension and lands here.  Blocks are 20^3 doubles (16^3 valid cells
// and 2 ghost layers), dimension 1 fastest; Julia passes pointer(u.u) as in 2D.
//
// Device tree, per level: blocks {blk, c1, c2, c3} (0-based id, 1-based coords), the
// child mask per block (bit (s1-1) + 2(s2-1) + 4(s3-1) set when that octant has a
// child), a pull table of 27 faces per block indexed by the ghost direction
// (f1+1) + 3(f2+1) + 9(f3+1) (entry 13 unused): {type, source block, packed vector},
// the packed vector holding a boundary's bnd or a refinement face's subblock as
// 2-bit fields (component + 1), and the child edges {fine, coarse, packed subblock}.
//
// Operation order follows the dimension-generic reference code written out for
// D = 3 (Base.Cartesian loops, first index innermost): ghost copies, mirrors and
// interpolation (weights 1/4, src/interp.jl:7-11) and restriction (8 cells, / 8) are
// bit-exact; stencils are accumulated in the reference's order without contraction.
#include <cmath>
#include <algorithm>
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

constexpr int S = kS, S2 = kS * kS, S3 = kS * kS * kS;

struct Signs27 { double v[27]; };

__device__ __forceinline__ int o3(int x, int y, int z) { return x + S * y + S2 * z; }
__device__ __forceinline__ int unpack(int packed, int d) { return ((packed >> (2 * d)) & 3) - 1; }

// ---- ghost fills (src/connectivity.jl:155-258), one thread per ghost cell -----------
// `phase` is a mask: 1 copies from neighbours, 2 mirrors at the domain boundary, 4
// interpolates from the parent.  fill_ghost! runs them in that order; on BoxStencil{3}
// trees an edge or corner boundary ghost can mirror a face or edge ghost that the copy
// pass writes (its bnd is zero along the directions where it is not on the domain
// boundary), so there copy and boundary share one launch -- such a ghost takes the
// neighbour's valid cell the copy would write -- and interpolation, which rewrites
// ghosts the boundary pass reads as they were, follows in a second.  On StarStencil{3}
// trees only face ghosts are filled, each reads valid cells of its own level or cells
// of the parent level, and no ghost reads another: one launch does all three passes.
// The ghost cells of a 20^3 block, enumerated: the four z-planes z = 0, 1, 18, 19 whole
// (4 x 400 cells), then for each of the 16 valid z the rows y = 0, 1, 18, 19 whole
// (4 x 20) and, on the 16 valid rows, the columns x = 0, 1, 18, 19 -- 3904 cells.
constexpr int kGhost3 = 4 * S2 + kM * (4 * S + kM * 4);
__device__ __forceinline__ int ghost_side(int i) { return i < 2 ? i : kS - 4 + i; }  // 0, 1, 18, 19
__device__ __forceinline__ void ghost_cell(int g, int &x, int &y, int &z) {
  if (g < 4 * S2) {
    z = ghost_side(g / S2);
    x = g % S;
    y = (g / S) % S;
    return;
  }
  g -= 4 * S2;
  z = kG + g / (4 * S + 4 * kM);
  const int r = g % (4 * S + 4 * kM);
  if (r < 4 * S) {
    y = ghost_side(r / S);
    x = r % S;
  } else {
    y = kG + (r - 4 * S) / 4;
    x = ghost_side((r - 4 * S) % 4);
  }
}

__device__ __forceinline__ void d3_fill(double *__restrict__ u, Level3View L, const Signs27 &sg, int phase) {
  const int64_t total = (int64_t)L.nblk * kGhost3;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t / kGhost3);
    int x, y, z;
    ghost_cell((int)(t % kGhost3), x, y, z);
    const int c = o3(x, y, z);
    const int f1 = x < kG ? -1 : x >= kG + kM ? 1 : 0;
    const int f2 = y < kG ? -1 : y >= kG + kM ? 1 : 0;
    const int f3 = z < kG ? -1 : z >= kG + kM ? 1 : 0;
    const int4 fi = L.faces[27 * bi + (f1 + 1) + 3 * (f2 + 1) + 9 * (f3 + 1)];
    const int type = fi.x;
    if ((type == FACE_NEIGHBOR && !(phase & 1)) || (type == FACE_BOUNDARY && !(phase & 2)) ||
        (type == FACE_REFBND && !(phase & 4)) || type == FACE_NONE)
      continue;
    double *ub = u + (int64_t)L.blocks[bi].x * S3;
    if (type == FACE_NEIGHBOR) {
      const double *src = u + (int64_t)fi.y * S3;
      ub[c] = src[o3(x - kM * f1, y - kM * f2, z - kM * f3)];
    } else if (type == FACE_BOUNDARY) {
      const int b1 = unpack(fi.z, 0), b2 = unpack(fi.z, 1), b3 = unpack(fi.z, 2);
      auto mir = [](int i, int b) { return b < 0 ? 2 * kG - 1 - i : b > 0 ? 2 * (kG + kM) - 1 - i : i; };
      const int mx = mir(x, b1), my = mir(y, b2), mz = mir(z, b3);
      // the mirrored cell is still a ghost along the directions where bnd is zero; when
      // this launch also runs the copy pass and that ghost is a neighbour copy, take the
      // neighbour's valid cell itself (the copy pass's own operation) instead of the
      // ghost the copy writes
      const int g1 = b1 ? 0 : f1, g2 = b2 ? 0 : f2, g3 = b3 ? 0 : f3;
      double src;
      const int4 gi = (phase & 1) && (g1 || g2 || g3) ? L.faces[27 * bi + (g1 + 1) + 3 * (g2 + 1) + 9 * (g3 + 1)]
                                                       : make_int4(FACE_NONE, 0, 0, 0);
      if (gi.x == FACE_NEIGHBOR)
        src = u[(int64_t)gi.y * S3 + o3(mx - kM * g1, my - kM * g2, mz - kM * g3)];
      else
        src = ub[o3(mx, my, mz)];
      ub[c] = __dmul_rn(sg.v[(1 + b1) + 3 * (1 + b2) + 9 * (1 + b3)], src);
    } else {
      // interp! from the parent's subblockbnd cell: along a face dimension the parent's
      // last (ghost below) or first (ghost above) subblock cell, else the subblock cell
      // over this one; i_d is the child offset
      const double *cb = u + (int64_t)fi.y * S3;
      const int p[3] = {x, y, z}, f[3] = {f1, f2, f3};
      int js[3], ii[3];
      for (int d = 0; d < 3; ++d) {
        const int sb = unpack(fi.z, d) + 1;
        if (f[d] < 0) { js[d] = 1 + 8 * sb; ii[d] = p[d]; }
        else if (f[d] > 0) { js[d] = 2 + 8 * (sb - 1); ii[d] = p[d] - (kG + kM); }
        else { js[d] = 2 + 8 * (sb - 1) + ((p[d] - kG) >> 1); ii[d] = (p[d] - kG) & 1; }
      }
      const int o = o3(js[0], js[1], js[2]);
      double v = __dmul_rn(0.25, cb[o]);
      v = __dadd_rn(v, __dmul_rn(0.25, cb[o + (2 * ii[0] - 1)]));
      v = __dadd_rn(v, __dmul_rn(0.25, cb[o + S * (2 * ii[1] - 1)]));
      v = __dadd_rn(v, __dmul_rn(0.25, cb[o + S2 * (2 * ii[2] - 1)]));
      ub[c] = v;
    }
  }
}

// ---- stencils: @stencil over the 3x3x3 literal, slab (third offset) slowest ---------
__device__ __forceinline__ double lhs3(const double *ub, int o, int op, double centre) {
  if (op == 2) {  // order 4: faces 2, edges 1, centre -24, corners absent; / 6
    double v = 0.0;
#pragma unroll
    for (int d3 = -1; d3 <= 1; ++d3)
#pragma unroll
      for (int d2 = -1; d2 <= 1; ++d2)
#pragma unroll
        for (int d1 = -1; d1 <= 1; ++d1) {
          const int nz = (d1 != 0) + (d2 != 0) + (d3 != 0);
          if (nz == 3) continue;
          const double c = nz == 0 ? -24.0 : nz == 1 ? 2.0 : 1.0;
          v = __dadd_rn(v, __dmul_rn(c, ub[o + d1 + S * d2 + S2 * d3]));
        }
    return v / 6.0;
  }
  double v = 0.0;  // order 2: (0,0,-1), (0,-1,0), (-1,0,0), centre, (1,0,0), (0,1,0), (0,0,1)
  v = __dadd_rn(v, ub[o - S2]);
  v = __dadd_rn(v, ub[o - S]);
  v = __dadd_rn(v, ub[o - 1]);
  v = __dadd_rn(v, __dmul_rn(centre, ub[o]));
  v = __dadd_rn(v, ub[o + 1]);
  v = __dadd_rn(v, ub[o + S]);
  v = __dadd_rn(v, ub[o + S2]);
  return v;
}

struct Op3 { int op; double s, centre, diag, omega; };

// RedBlack{P} (src/multigrid.jl:153-180): x steps by 2, parity P xor (y+1 & 1) xor (z+1 & 1)
// in 1-based terms; two fused multiply-adds as the reference's muladds.
__device__ __forceinline__ void d3_gs_rb(double *__restrict__ u, const double *__restrict__ b, Level3View L, Op3 p, int parity) {
  const int64_t total = (int64_t)L.nblk * (kM * kM * kM / 2);
  const double nwc = -(p.omega / p.diag);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t / 2048), c = (int)(t % 2048);
    const int z = kG + c / 128, y = kG + (c / 8) % 16, k = c % 8;
    const int pp = parity ^ ((y + 1) & 1) ^ ((z + 1) & 1);
    const int x = kG + 2 * k + pp;
    const int64_t base = (int64_t)L.blocks[bi].x * S3;
    const int o = o3(x, y, z);
    const double Lu = lhs3(u + base, o, p.op, p.centre);
    const double v = fma(p.s, b[base + o], Lu);
    u[base + o] = fma(nwc, v, u[base + o]);
  }
}

// d3_gs_rb on a StarStencil{3} tree, also writing the face ghosts that copy or mirror
// each updated cell -- the neighbour's facing ghost (fill_ghost_copy!) and the block's own
// mirror ghost with its sign (fill_ghost_bnd!), the operations of d3_fill's passes 1 and 2
// -- so that no fill launch follows the sweep.  The sweep reads only cells and ghosts of
// the other colour, and each ghost it writes copies a cell of its own colour or mirrors
// an unchanged cell of the other colour, so no thread reads a value another one writes.
__device__ __forceinline__ void d3_gs_rb_push(double *__restrict__ u, const double *__restrict__ b, Level3View L,
                                              Op3 p, int parity, const Signs27 &sg) {
  const int64_t total = (int64_t)L.nblk * (kM * kM * kM / 2);
  const double nwc = -(p.omega / p.diag);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t / 2048), c = (int)(t % 2048);
    const int z = kG + c / 128, y = kG + (c / 8) % 16, k = c % 8;
    const int pp = parity ^ ((y + 1) & 1) ^ ((z + 1) & 1);
    const int x = kG + 2 * k + pp;
    const int64_t base = (int64_t)L.blocks[bi].x * S3;
    const int o = o3(x, y, z);
    const double Lu = lhs3(u + base, o, p.op, p.centre);
    const double v = fma(p.s, b[base + o], Lu);
    const double nu = fma(nwc, v, u[base + o]);
    u[base + o] = nu;
    const int q[3] = {x, y, z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int f = q[d] < kG + 2 ? -1 : q[d] >= kG + kM - 2 ? 1 : 0;
      if (!f) continue;
      const int4 fi = L.faces[27 * bi + 13 + f * (d == 0 ? 1 : d == 1 ? 3 : 9)];
      int g[3] = {x, y, z};
      if (fi.x == FACE_NEIGHBOR) {
        g[d] -= kM * f;  // the neighbour's facing ghost
        u[(int64_t)fi.y * S3 + o3(g[0], g[1], g[2])] = nu;
      } else if (fi.x == FACE_BOUNDARY) {
        const int b1 = unpack(fi.z, 0), b2 = unpack(fi.z, 1), b3 = unpack(fi.z, 2);
        const int bb[3] = {b1, b2, b3};
        const double sgn = sg.v[(1 + b1) + 3 * (1 + b2) + 9 * (1 + b3)];
        auto mirror = [&](int *m) {
#pragma unroll
          for (int e = 0; e < 3; ++e)
            if (bb[e]) m[e] = bb[e] < 0 ? 2 * kG - 1 - m[e] : 2 * (kG + kM) - 1 - m[e];
        };
        mirror(g);
        u[base + o3(g[0], g[1], g[2])] = __dmul_rn(sgn, nu);
        // one layer in from the face: also the first-layer mirror of the other colour's
        // edge cell beside this one (unchanged by this sweep), which that cell's own
        // sweep reads next -- the value the fill after this sweep would give it
        if (q[d] == (f < 0 ? kG + 1 : kG + kM - 2)) {
          int m[3] = {x, y, z};
          m[d] += f;
          const double w = u[base + o3(m[0], m[1], m[2])];
          mirror(m);
          u[base + o3(m[0], m[1], m[2])] = __dmul_rn(sgn, w);
        }
      }
    }
  }
}

// FourColors{P1,P2} (src/multigrid.jl:206-232) for D = 3: cells (x + p1, y + p2, z) on
// the even grid of the first two dimensions, p_a = (P_a + z + 1) mod 2 (1-based z);
// u -= omega (Lu + s b) / c, unfused.
__device__ __forceinline__ void d3_gs4(double *__restrict__ u, const double *__restrict__ b, Level3View L, Op3 p, int P1, int P2) {
  const int64_t total = (int64_t)L.nblk * 1024;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t / 1024), c = (int)(t % 1024);
    const int z = kG + c / 64;
    const int p1 = (P1 + z + 1) & 1, p2 = (P2 + z + 1) & 1;
    const int x = kG + 2 * (c % 8) + p1, y = kG + 2 * ((c / 8) % 8) + p2;
    const int64_t base = (int64_t)L.blocks[bi].x * S3;
    const int o = o3(x, y, z);
    const double Lu = lhs3(u + base, o, p.op, p.centre);
    const double upd = __dmul_rn(p.omega, __dadd_rn(Lu, __dmul_rn(p.s, b[base + o]))) / p.diag;
    u[base + o] = u[base + o] - upd;
  }
}

__device__ __forceinline__ void d3_residual(double *__restrict__ r, const double *__restrict__ u, const double *__restrict__ b,
                            Level3View L, Op3 p) {
  const int64_t total = (int64_t)L.nblk * 4096;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t / 4096), c = (int)(t % 4096);
    const int o = o3(kG + c % 16, kG + (c / 16) % 16, kG + c / 256);
    const int64_t base = (int64_t)L.blocks[bi].x * S3;
    r[base + o] = -(b[base + o] + lhs3(u + base, o, p.op, p.centre) / p.s);
  }
}

// residual_subblock! on the coarse subblock of every child edge of this level
__device__ __forceinline__ void d3_postrestrict(double *__restrict__ bf, const double *__restrict__ u, const double *__restrict__ r,
                                Level3View L, Op3 pc) {
  const int64_t total = (int64_t)L.nch * 512;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int e = (int)(t / 512), c = (int)(t % 512);
    const int4 ch = L.child[e];
    const int x = kG + 8 * unpack(ch.z, 0) + c % 8;
    const int y = kG + 8 * unpack(ch.z, 1) + (c / 8) % 8;
    const int z = kG + 8 * unpack(ch.z, 2) + c / 64;
    const int o = o3(x, y, z);
    const int64_t base = (int64_t)ch.y * S3;
    bf[base + o] = -(r[base + o] + lhs3(u + base, o, pc.op, pc.centre) / pc.s);
  }
}

// restrict! (src/restrict.jl:5-25): f = 0; f += the 8 fine cells (first offset
// innermost); coarse = f / 8
__device__ __forceinline__ void d3_restrict(double *__restrict__ u, Level3View L) {
  const int64_t total = (int64_t)L.nch * 512;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int e = (int)(t / 512), c = (int)(t % 512);
    const int4 ch = L.child[e];
    const int kx = c % 8, ky = (c / 8) % 8, kz = c / 64;
    const double *fb = u + (int64_t)ch.x * S3 + o3(kG + 2 * kx, kG + 2 * ky, kG + 2 * kz);
    double f = 0.0;
#pragma unroll
    for (int i3 = 0; i3 <= 1; ++i3)
#pragma unroll
      for (int i2 = 0; i2 <= 1; ++i2)
#pragma unroll
        for (int i1 = 0; i1 <= 1; ++i1) f = __dadd_rn(f, fb[i1 + S * i2 + S2 * i3]);
    u[(int64_t)ch.y * S3 + o3(kG + 8 * unpack(ch.z, 0) + kx, kG + 8 * unpack(ch.z, 1) + ky,
                              kG + 8 * unpack(ch.z, 2) + kz)] = f / 8.0;
  }
}

// interp_add_level! (src/interp.jl:107-115): u_fine += P(u1 over the parent's subblock)
__device__ __forceinline__ void d3_interp_add(double *__restrict__ u, const double *__restrict__ u1, Level3View L) {
  const int64_t total = (int64_t)L.nch * 4096;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int e = (int)(t / 4096), c = (int)(t % 4096);
    const int4 ch = L.child[e];
    const int dx = c % 16, dy = (c / 16) % 16, dz = c / 256;
    const int o = o3(kG + 8 * unpack(ch.z, 0) + (dx >> 1), kG + 8 * unpack(ch.z, 1) + (dy >> 1),
                     kG + 8 * unpack(ch.z, 2) + (dz >> 1));
    const double *cb = u1 + (int64_t)ch.y * S3;
    double v = __dmul_rn(0.25, cb[o]);
    v = __dadd_rn(v, __dmul_rn(0.25, cb[o + (2 * (dx & 1) - 1)]));
    v = __dadd_rn(v, __dmul_rn(0.25, cb[o + S * (2 * (dy & 1) - 1)]));
    v = __dadd_rn(v, __dmul_rn(0.25, cb[o + S2 * (2 * (dz & 1) - 1)]));
    double *d = u + (int64_t)ch.x * S3 + o3(kG + dx, kG + dy, kG + dz);
    *d = __dadd_rn(v, *d);
  }
}

__device__ __forceinline__ void d3_copy(double *__restrict__ dst, const double *__restrict__ a1, const double *__restrict__ a2,
                        Level3View L) {
  const int64_t total = (int64_t)L.nblk * S3;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t o = (int64_t)L.blocks[t / S3].x * S3 + t % S3;
    dst[o] = a2 ? a1[o] - a2[o] : a1[o];
  }
}

// The per-operation kernels: each one body, launched alone or run by the sequencer.
__global__ void k3_fill(double *__restrict__ u, Level3View L, Signs27 sg, int phase) { d3_fill(u, L, sg, phase); }
__global__ void k3_gs_rb(double *__restrict__ u, const double *__restrict__ b, Level3View L, Op3 p, int parity) { d3_gs_rb(u, b, L, p, parity); }
__global__ void k3_gs_rb_push(double *__restrict__ u, const double *__restrict__ b, Level3View L, Op3 p, int parity,
                              Signs27 sg) {
  d3_gs_rb_push(u, b, L, p, parity, sg);
}
__global__ void k3_gs4(double *__restrict__ u, const double *__restrict__ b, Level3View L, Op3 p, int P1, int P2) { d3_gs4(u, b, L, p, P1, P2); }
__global__ void k3_residual(double *__restrict__ r, const double *__restrict__ u, const double *__restrict__ b,
                            Level3View L, Op3 p) { d3_residual(r, u, b, L, p); }
__global__ void k3_postrestrict(double *__restrict__ bf, const double *__restrict__ u, const double *__restrict__ r,
                                Level3View L, Op3 pc) { d3_postrestrict(bf, u, r, L, pc); }
__global__ void k3_restrict(double *__restrict__ u, Level3View L) { d3_restrict(u, L); }
__global__ void k3_interp_add(double *__restrict__ u, const double *__restrict__ u1, Level3View L) { d3_interp_add(u, u1, L); }
__global__ void k3_copy(double *__restrict__ dst, const double *__restrict__ a1, const double *__restrict__ a2,
                        Level3View L) { d3_copy(dst, a1, a2, L); }

// Table-driven ghost pushes of a colour sweep (octrees other than StarStencil{3} at
// order 2): off[bi*4096 + cell] .. off[bi*4096 + cell + 1] index ent = {the ghost's
// index in the field, up to three boundary-table entries of the mirrors on the way,
// 5 bits each, 31 = none}; the boundary table comes packed, two bits an entry (entry
// + 1: the pushes run only where every entry is -1, 0 or 1, so the products are exact
// in any order).  Tables built from the fill itself (ensure_push3).
__device__ __forceinline__ void push3(double *__restrict__ u, const PushView &pv, unsigned long long sg, int bi,
                                      int x, int y, int z, double v) {
  const int c = bi * 4096 + (x - kG) + kM * (y - kG) + kM * kM * (z - kG);
  const int e1 = pv.off[c + 1];
  for (int e = pv.off[c]; e < e1; ++e) {
    const int2 d = pv.ent[e];
    double w = v;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int i = (d.y >> (5 * k)) & 31;
      if (i < 27) w = __dmul_rn((double)((int)((sg >> (2 * i)) & 3ull) - 1), w);
    }
    u[d.x] = w;
  }
}

// d3_gs_rb / d3_gs4 with the table pushes after each update.
__global__ void k3_gs_rb_tpush(double *__restrict__ u, const double *__restrict__ b, Level3View L, Op3 p, int parity,
                               PushView pv, unsigned long long sg) {
  const int64_t total = (int64_t)L.nblk * (kM * kM * kM / 2);
  const double nwc = -(p.omega / p.diag);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t / 2048), c = (int)(t % 2048);
    const int z = kG + c / 128, y = kG + (c / 8) % 16, k = c % 8;
    const int pp = parity ^ ((y + 1) & 1) ^ ((z + 1) & 1);
    const int x = kG + 2 * k + pp;
    const int64_t base = (int64_t)L.blocks[bi].x * S3;
    const int o = o3(x, y, z);
    const double Lu = lhs3(u + base, o, p.op, p.centre);
    const double v = fma(p.s, b[base + o], Lu);
    const double nv = fma(nwc, v, u[base + o]);
    u[base + o] = nv;
    push3(u, pv, sg, bi, x, y, z, nv);
  }
}

__global__ void k3_gs4_push(double *__restrict__ u, const double *__restrict__ b, Level3View L, Op3 p, int P1, int P2,
                            PushView pv, unsigned long long sg) {
  const int64_t total = (int64_t)L.nblk * 1024;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t / 1024), c = (int)(t % 1024);
    const int z = kG + c / 64;
    const int p1 = (P1 + z + 1) & 1, p2 = (P2 + z + 1) & 1;
    const int x = kG + 2 * (c % 8) + p1, y = kG + 2 * ((c / 8) % 8) + p2;
    const int64_t base = (int64_t)L.blocks[bi].x * S3;
    const int o = o3(x, y, z);
    const double Lu = lhs3(u + base, o, p.op, p.centre);
    const double upd = __dmul_rn(p.omega, __dadd_rn(Lu, __dmul_rn(p.s, b[base + o]))) / p.diag;
    const double nv = u[base + o] - upd;
    u[base + o] = nv;
    push3(u, pv, sg, bi, x, y, z, nv);
  }
}

// Identity field for the push tables: valid cells hold their index in the field + 1,
// ghosts 0; `copies` consecutive fields.
__global__ void k3_push_ident(double *__restrict__ a, int64_t n, int copies) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % S3), x = c % S, y = (c / S) % S, z = c / S2;
    const bool valid = x >= kG && x < kG + kM && y >= kG && y < kG + kM && z >= kG && z < kG + kM;
    for (int k = 0; k < copies; ++k) a[k * n + i] = valid ? (double)(i + 1) : 0.0;
  }
}

// ---- the sequencer (3D): a recorded per-operation V-cycle in one cooperative launch --
// The records are the launches the per-operation path would make, in order; a grid
// barrier (release/acquire on a counter, bounded wait) separates consecutive records,
// so every operation sees its predecessors' writes as a separate launch would, and the
// results are those of the launches.
enum Seq3Kind { S3_FILL = 1, S3_GS_RB, S3_GS4, S3_RESIDUAL, S3_POSTRESTRICT, S3_RESTRICT, S3_INTERP_ADD, S3_COPY, S3_GS_RB_PUSH };
struct SeqOp3 {
  int kind, i0, i1, pad;
  double *a;
  const double *b;
  const double *c;
  Level3View lv;
  Op3 p;
  Signs27 sg;
};

constexpr int kSeq3Threads = 512;
constexpr int kSeq3PerSM = 1;  // resident CTAs per SM

__global__ void __launch_bounds__(kSeq3Threads, kSeq3PerSM)
    k3_sequencer(const SeqOp3 *__restrict__ ops, int nops, unsigned *bar, int *err, long long timeout_ns) {
  unsigned epoch = 0;
  for (int i = 0; i < nops; ++i) {
    const SeqOp3 &op = ops[i];
    switch (op.kind) {
      case S3_FILL: d3_fill(op.a, op.lv, op.sg, op.i0); break;
      case S3_GS_RB: d3_gs_rb(op.a, op.b, op.lv, op.p, op.i0); break;
      case S3_GS_RB_PUSH: d3_gs_rb_push(op.a, op.b, op.lv, op.p, op.i0, op.sg); break;
      case S3_GS4: d3_gs4(op.a, op.b, op.lv, op.p, op.i0, op.i1); break;
      case S3_RESIDUAL: d3_residual(op.a, op.b, op.c, op.lv, op.p); break;
      case S3_POSTRESTRICT: d3_postrestrict(op.a, op.b, op.c, op.lv, op.p); break;
      case S3_RESTRICT: d3_restrict(op.a, op.lv); break;
      case S3_INTERP_ADD: d3_interp_add(op.a, op.b, op.lv); break;
      case S3_COPY: d3_copy(op.a, op.b, op.c, op.lv); break;
      default:
        if (threadIdx.x == 0) atomicCAS(err, 0, 4);
        return;
    }
    if (i + 1 < nops && !grid_barrier(bar, err, epoch, timeout_ns)) return;
  }
}

// While a sequence is being recorded (ctx->seq_rec set) the launchers below append
// their operation instead of launching it.
bool seq3_push(srmg_ctx *ctx, int kind, int i0, int i1, double *a, const double *b, const double *c,
               const Level3View &lv, const Op3 *p, const Signs27 *sg) {
  if (!ctx->seq_rec) return false;
  SeqOp3 op;
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

// rhs! (src/multigrid.jl:363-388): identity at order 2, the 7-point right-hand side
// (centre 6) / 12 at order 4 (src/laplacian.jl:322-337)
__global__ void k3_rhs(double *__restrict__ q1, const double *__restrict__ q, Level3View L, int op) {
  const int64_t total = (int64_t)L.nblk * 4096;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t / 4096), c = (int)(t % 4096);
    const int o = o3(kG + c % 16, kG + (c / 16) % 16, kG + c / 256);
    const int64_t base = (int64_t)L.blocks[bi].x * S3;
    const double *qb = q + base;
    if (op != 2) {
      q1[base + o] = qb[o];
      continue;
    }
    double v = 0.0;
    v = __dadd_rn(v, qb[o - S2]);
    v = __dadd_rn(v, qb[o - S]);
    v = __dadd_rn(v, qb[o - 1]);
    v = __dadd_rn(v, __dmul_rn(6.0, qb[o]));
    v = __dadd_rn(v, qb[o + 1]);
    v = __dadd_rn(v, qb[o + S]);
    v = __dadd_rn(v, qb[o + S2]);
    q1[base + o] = v / 12.0;
  }
}

// Sum over the level's leaf cells of w_l f^2 (f = residual, or b itself), one partial per
// CTA; a leaf cell of level l carries 8^-(l-1), what resnorm!'s restriction of squares
// gives it (src/multigrid.jl:391-417).
template <int NT>
__global__ void __launch_bounds__(NT) k3_leafsq(double *__restrict__ part, const double *__restrict__ u,
                                                const double *__restrict__ b, Level3View L, Op3 p, double wl,
                                                int mode) {
  double acc = 0.0;
  const int64_t total = (int64_t)L.nblk * 4096;
  for (int64_t t = blockIdx.x * (int64_t)NT + threadIdx.x; t < total; t += (int64_t)gridDim.x * NT) {
    const int bi = (int)(t / 4096), c = (int)(t % 4096);
    const int cx = c % 16, cy = (c / 16) % 16, cz = c / 256;
    const int oct = (cx >> 3) + 2 * (cy >> 3) + 4 * (cz >> 3);
    if ((L.mask[bi] >> oct) & 1) continue;
    const int o = o3(kG + cx, kG + cy, kG + cz);
    const int64_t base = (int64_t)L.blocks[bi].x * S3;
    const double v = mode == 0 ? -(b[base + o] + lhs3(u + base, o, p.op, p.centre) / p.s) : b[base + o];
    acc = fma(v, v, acc);
  }
  __shared__ double sh[NT / 32];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < NT / 32 ? sh[threadIdx.x] : 0.0;
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if (threadIdx.x == 0) part[blockIdx.x] = v * wl;
  }
}

int grid3(int64_t work, int threads) {
  const int64_t g = (work + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 16));
}

Signs27 signs27(const int8_t *bc) {
  Signs27 s;
  for (int i = 0; i < 27; ++i) s.v[i] = bc ? (double)bc[i] : 1.0;
  return s;
}

Op3 op3(int op, double k2, double sl, double omega) {
  Op3 p;
  p.op = op;
  p.s = sl;
  p.centre = op == SRMG_OP_HELMHOLTZ ? -6.0 - sl * k2 : -6.0;
  p.diag = op == SRMG_OP_LAPLACIAN4 ? -4.0 : p.centre;  // diagelm (src/laplacian.jl:299,339)
  p.omega = omega;
  return p;
}

Level3View view(srmg_ctx *ctx, int l) { return ctx->lv3[l - 1].view(); }

int fill(srmg_ctx *ctx, double *u, int l, const Signs27 &sg, int mask) {
  const int n = ctx->nblk_host[l - 1];
  if (!n) return SRMG_OK;
  if (!ctx->has_corners) {
    if (seq3_push(ctx, S3_FILL, mask, 0, u, nullptr, nullptr, view(ctx, l), nullptr, &sg)) return SRMG_OK;
    k3_fill<<<grid3((int64_t)n * kGhost3, 256), 256, 0, ctx->stream>>>(u, view(ctx, l), sg, mask);
    ctx->launches++;
    return SRMG_OK;
  }
  if ((mask & 3) == 3 && ctx->merge_fill) {
    if (!seq3_push(ctx, S3_FILL, 3, 0, u, nullptr, nullptr, view(ctx, l), nullptr, &sg)) {
      k3_fill<<<grid3((int64_t)n * kGhost3, 256), 256, 0, ctx->stream>>>(u, view(ctx, l), sg, 3);
      ctx->launches++;
    }
    mask &= ~3;
  }
  for (int phase = 1; phase <= 4; phase <<= 1) {
    if (!(mask & phase)) continue;
    if (seq3_push(ctx, S3_FILL, phase, 0, u, nullptr, nullptr, view(ctx, l), nullptr, &sg)) continue;
    k3_fill<<<grid3((int64_t)n * kGhost3, 256), 256, 0, ctx->stream>>>(u, view(ctx, l), sg, phase);
    ctx->launches++;
  }
  return SRMG_OK;
}

// The push tables of an octree, read off its copy-and-boundary fill (mask 3) run on an
// identity field: once with every boundary entry 1 (each ghost then holds its source
// cell's index + 1, or 0 if it takes no valid cell's value) and once with entry k the
// k-th prime (the ratio names the entries of the mirrors on the way, at most three).
// The tables are used for a colouring only if no cell of the source's colour other
// than the source reads a pushed ghost: the 6 face neighbours for red-black, the 18
// face and edge neighbours of the order-4 stencil for four colours.  Anything the tables
// cannot express leaves the tree on the fill launches (push_state -1).
int ensure_push3(srmg_ctx *ctx) {
  if (ctx->push_state != 0 || !ctx->use_gs_push || !ctx->has_tree || ctx->seq_rec) return SRMG_OK;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(ctx->stream, &cap));
  if (cap != cudaStreamCaptureStatusNone) return SRMG_OK;
  ctx->push_state = -1;
  const int64_t nf = ctx->max_blk * S3;
  if (nf <= 0 || nf >= ((int64_t)1 << 31)) return SRMG_OK;
  static const int kPrime[27] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43,
                                 47, 53, 59, 61, 67, 71, 73, 79, 83, 89, 97, 101, 103};
  Signs27 ones, primes;
  for (int i = 0; i < 27; i++) {
    ones.v[i] = 1.0;
    primes.v[i] = kPrime[i];
  }
  std::vector<double> h((size_t)(2 * nf));
  {
    double *d = nullptr;
    CK(cudaMalloc(&d, (size_t)(2 * nf) * sizeof(double)));
    const int64_t l0 = ctx->launches;
    k3_push_ident<<<grid3(nf, 256), 256, 0, ctx->stream>>>(d, nf, 2);
    int rc = SRMG_OK;
    for (int l = 1; l <= ctx->nlev && rc == SRMG_OK; l++) {
      rc = fill(ctx, d, l, ones, 3);
      if (rc == SRMG_OK) rc = fill(ctx, d + nf, l, primes, 3);
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
    const Dev3Level &L = ctx->lv3[l - 1];
    blocks[l - 1].resize(L.nblk);
    if (L.nblk) CK(cudaMemcpy(blocks[l - 1].data(), L.blocks, L.nblk * sizeof(int4), cudaMemcpyDeviceToHost));
    for (int bi = 0; bi < L.nblk; bi++) {
      const int blk = blocks[l - 1][bi].x;
      if (blk < 0 || blk >= ctx->max_blk) return SRMG_OK;
      lvl_of[blk] = l;
      bi_of[blk] = bi;
    }
  }
  auto valid = [](int x, int y, int z) {
    return x >= kG && x < kG + kM && y >= kG && y < kG + kM && z >= kG && z < kG + kM;
  };
  bool ok2 = true, ok4 = true;
  struct Ent { int key, dest, sg; };
  std::vector<std::vector<Ent>> ents(ctx->nlev);
  for (int l = 1; l <= ctx->nlev; l++)
    for (int bi = 0; bi < ctx->lv3[l - 1].nblk; bi++) {
      const int blk = blocks[l - 1][bi].x;
      for (int g = 0; g < S3; g++) {
        const int gx = g % S, gy = (g / S) % S, gz = g / S2;
        if (valid(gx, gy, gz)) continue;
        const int64_t gi = (int64_t)blk * S3 + g;
        const double a = h[gi], a2 = h[nf + gi];
        if (a == 0.0) {
          if (a2 != 0.0) return SRMG_OK;
          continue;
        }
        if (!(a >= 1.0 && a <= (double)nf && a == std::floor(a))) return SRMG_OK;
        const int64_t src = (int64_t)a - 1;
        const int sblk = (int)(src / S3), sc = (int)(src % S3);
        const int sx = sc % S, sy = (sc / S) % S, sz = sc / S2;
        if (!valid(sx, sy, sz) || lvl_of[sblk] != l) return SRMG_OK;
        // the ratio of the two runs, factored into at most three primes
        const double q = a2 / a;
        if (!(q >= 1.0 && q == std::floor(q) && a2 == a * q)) return SRMG_OK;
        int64_t rest = (int64_t)q;
        int idx[3] = {31, 31, 31}, nidx = 0;
        for (int i = 0; i < 27 && rest > 1; i++)
          while (rest % kPrime[i] == 0 && rest > 1) {
            if (nidx == 3) return SRMG_OK;
            idx[nidx++] = i;
            rest /= kPrime[i];
          }
        if (rest != 1) return SRMG_OK;
        for (int dz = -1; dz <= 1; dz++)
          for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
              const int nz = (dx != 0) + (dy != 0) + (dz != 0);
              if (nz == 0 || nz == 3) continue;
              const int rx = gx + dx, ry = gy + dy, rz = gz + dz;
              if (!valid(rx, ry, rz) || (sblk == blk && rx == sx && ry == sy && rz == sz)) continue;
              if (((rx + rz + sx + sz) & 1) == 0 && ((ry + rz + sy + sz) & 1) == 0) ok4 = false;
              if (nz == 1 && ((rx + ry + rz + sx + sy + sz) & 1) == 0) ok2 = false;
            }
        ents[l - 1].push_back({bi_of[sblk] * 4096 + (sx - kG) + kM * (sy - kG) + kM * kM * (sz - kG), (int)gi,
                               idx[0] | (idx[1] << 5) | (idx[2] << 10)});
      }
    }
  if (!ok2 && !ok4) return SRMG_OK;
  std::vector<size_t> at(ctx->nlev), ent_at(ctx->nlev);
  size_t bytes = 0;
  for (int l = 1; l <= ctx->nlev; l++) {
    const int nb = ctx->lv3[l - 1].nblk;
    at[l - 1] = ent_at[l - 1] = bytes;
    if (!nb) continue;
    bytes += ((size_t)nb * 4096 + 1) * sizeof(int);
    bytes = (bytes + 15) & ~(size_t)15;
    ent_at[l - 1] = bytes;
    bytes += ents[l - 1].size() * sizeof(int2);
    bytes = (bytes + 15) & ~(size_t)15;
  }
  std::vector<char> stage(bytes);
  for (int l = 1; l <= ctx->nlev; l++) {
    const int nb = ctx->lv3[l - 1].nblk;
    if (!nb) continue;
    int *off = reinterpret_cast<int *>(stage.data() + at[l - 1]);
    int2 *ent = reinterpret_cast<int2 *>(stage.data() + ent_at[l - 1]);
    std::fill(off, off + nb * 4096 + 1, 0);
    for (const Ent &e : ents[l - 1]) off[e.key + 1]++;
    for (int k = 0; k < nb * 4096; k++) off[k + 1] += off[k];
    std::vector<int> fillp(off, off + nb * 4096);
    for (const Ent &e : ents[l - 1]) ent[fillp[e.key]++] = make_int2(e.dest, e.sg);
  }
  RC(ensure(ctx, ctx->push_tab, bytes));
  CK(cudaMemcpy(ctx->push_tab.p, stage.data(), bytes, cudaMemcpyHostToDevice));
  ctx->push_lv.assign(ctx->nlev, PushView{nullptr, nullptr});
  char *base = static_cast<char *>(ctx->push_tab.p);
  for (int l = 1; l <= ctx->nlev; l++)
    if (ctx->lv3[l - 1].nblk)
      ctx->push_lv[l - 1] = PushView{reinterpret_cast<const int *>(base + at[l - 1]),
                                     reinterpret_cast<const int2 *>(base + ent_at[l - 1])};
  ctx->push_ok2 = ok2;
  ctx->push_ok4 = ok4;
  ctx->push_state = 1;
  return SRMG_OK;
}

int gs_colour(srmg_ctx *ctx, double *u, const double *b, int l, const Op3 &p, int colour) {
  const int n = ctx->nblk_host[l - 1];
  if (!n) return SRMG_OK;
  if (p.op == SRMG_OP_LAPLACIAN4 &&
      seq3_push(ctx, S3_GS4, colour >> 1, colour & 1, u, b, nullptr, view(ctx, l), &p, nullptr))
    return SRMG_OK;
  if (p.op != SRMG_OP_LAPLACIAN4 && seq3_push(ctx, S3_GS_RB, colour, 0, u, b, nullptr, view(ctx, l), &p, nullptr))
    return SRMG_OK;
  if (p.op == SRMG_OP_LAPLACIAN4)
    k3_gs4<<<grid3((int64_t)n * 1024, 256), 256, 0, ctx->stream>>>(u, b, view(ctx, l), p, colour >> 1, colour & 1);
  else
    k3_gs_rb<<<grid3((int64_t)n * 2048, 256), 256, 0, ctx->stream>>>(u, b, view(ctx, l), p, colour);
  ctx->launches++;
  return SRMG_OK;
}

// Whether gs_iter's sweeps write their own copy and mirror ghosts (d3_gs_rb_push).
bool gs_pushes(const srmg_ctx *ctx, const Op3 &p) { return !ctx->has_corners && p.op != SRMG_OP_LAPLACIAN4; }

// gauss_seidel_iter! (src/multigrid.jl:250-295): each colour followed by copy and
// boundary ghosts -- on StarStencil{3} trees at order 2 written by the sweep itself
// (d3_gs_rb_push), one launch a colour instead of two
int gs_iter(srmg_ctx *ctx, double *u, const double *b, int l, const Op3 &p, int n, const Signs27 &sg) {
  const int ncol = p.op == SRMG_OP_LAPLACIAN4 ? 4 : 2;
  const bool push = gs_pushes(ctx, p);
  const int nb = ctx->nblk_host[l - 1];
  // elsewhere the table pushes (ensure_push3): the first colour keeps its fill launch,
  // which makes the ghosts what the fill makes of the current cells; every later colour
  // writes the ghosts of the cells it updates, all that the fill after it would change
  bool tpush = false;
  unsigned long long sw = 0;
  if (!push && ctx->use_gs_push && nb > 0) {
    if (ctx->push_state == 0) RC(ensure_push3(ctx));
    bool unit = true;
    for (int i = 0; i < 27; i++) unit = unit && (sg.v[i] == 1.0 || sg.v[i] == -1.0 || sg.v[i] == 0.0);
    tpush = ctx->push_state == 1 && !ctx->seq_rec && unit &&
            (p.op == SRMG_OP_LAPLACIAN4 ? ctx->push_ok4 : ctx->push_ok2);
    for (int i = 0; tpush && i < 27; i++) sw |= (unsigned long long)((int)sg.v[i] + 1) << (2 * i);
  }
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < ncol; ++c) {
      if (push) {
        if (!nb || seq3_push(ctx, S3_GS_RB_PUSH, c, 0, u, b, nullptr, view(ctx, l), &p, &sg)) continue;
        k3_gs_rb_push<<<grid3((int64_t)nb * 2048, 256), 256, 0, ctx->stream>>>(u, b, view(ctx, l), p, c, sg);
        ctx->launches++;
        continue;
      }
      if (tpush && (i > 0 || c > 0)) {
        if (p.op == SRMG_OP_LAPLACIAN4)
          k3_gs4_push<<<grid3((int64_t)nb * 1024, 256), 256, 0, ctx->stream>>>(u, b, view(ctx, l), p, c >> 1, c & 1,
                                                                               ctx->push_lv[l - 1], sw);
        else
          k3_gs_rb_tpush<<<grid3((int64_t)nb * 2048, 256), 256, 0, ctx->stream>>>(u, b, view(ctx, l), p, c,
                                                                                  ctx->push_lv[l - 1], sw);
        ctx->launches++;
        continue;
      }
      RC(gs_colour(ctx, u, b, l, p, c));
      RC(fill(ctx, u, l, sg, 3));
    }
  return SRMG_OK;
}

int residual(srmg_ctx *ctx, double *r, const double *u, const double *b, int l, const Op3 &p) {
  const int n = ctx->nblk_host[l - 1];
  if (!n) return SRMG_OK;
  if (seq3_push(ctx, S3_RESIDUAL, 0, 0, r, u, b, view(ctx, l), &p, nullptr)) return SRMG_OK;
  k3_residual<<<grid3((int64_t)n * 4096, 256), 256, 0, ctx->stream>>>(r, u, b, view(ctx, l), p);
  ctx->launches++;
  return SRMG_OK;
}

int postrestrict(srmg_ctx *ctx, double *bf, const double *u, const double *r, int l, const Op3 &pc) {
  const int n = ctx->nch_host[l - 1];
  if (!n) return SRMG_OK;
  if (seq3_push(ctx, S3_POSTRESTRICT, 0, 0, bf, u, r, view(ctx, l), &pc, nullptr)) return SRMG_OK;
  k3_postrestrict<<<grid3((int64_t)n * 512, 256), 256, 0, ctx->stream>>>(bf, u, r, view(ctx, l), pc);
  ctx->launches++;
  return SRMG_OK;
}

int restrict_l(srmg_ctx *ctx, double *u, int l) {
  const int n = ctx->nch_host[l - 1];
  if (!n) return SRMG_OK;
  if (seq3_push(ctx, S3_RESTRICT, 0, 0, u, nullptr, nullptr, view(ctx, l), nullptr, nullptr)) return SRMG_OK;
  k3_restrict<<<grid3((int64_t)n * 512, 256), 256, 0, ctx->stream>>>(u, view(ctx, l));
  ctx->launches++;
  return SRMG_OK;
}

int interp_add(srmg_ctx *ctx, double *u, const double *u1, int l) {
  const int n = ctx->nch_host[l - 1];
  if (!n) return SRMG_OK;
  if (seq3_push(ctx, S3_INTERP_ADD, 0, 0, u, u1, nullptr, view(ctx, l), nullptr, nullptr)) return SRMG_OK;
  k3_interp_add<<<grid3((int64_t)n * 4096, 256), 256, 0, ctx->stream>>>(u, u1, view(ctx, l));
  ctx->launches++;
  return SRMG_OK;
}

int copy_l(srmg_ctx *ctx, double *dst, const double *a1, const double *a2, int l) {
  const int n = ctx->nblk_host[l - 1];
  if (!n) return SRMG_OK;
  if (seq3_push(ctx, S3_COPY, 0, 0, dst, a1, a2, view(ctx, l), nullptr, nullptr)) return SRMG_OK;
  k3_copy<<<grid3((int64_t)n * S3, 256), 256, 0, ctx->stream>>>(dst, a1, a2, view(ctx, l));
  ctx->launches++;
  return SRMG_OK;
}

int vcycle(srmg_ctx *ctx, double *u, double *b, double *r, double *u1, double s, int op, double k2,
           const Signs27 &sg, int lmax, int ndown, int ntop, int nup, double omega) {
  if (lmax == 0) lmax = ctx->nlev;
  if (lmax < 1 || lmax > ctx->nlev) return fail(ctx, SRMG_ERR_BADARG, "lmax %d out of range", lmax);
  for (int l = lmax; l >= 2; --l) {
    const double sl = level_scale(s, l);
    const Op3 p = op3(op, k2, sl, omega), pc = op3(op, k2, 4 * sl, omega);
    RC(gs_iter(ctx, u, b, l, p, ndown, sg));
    RC(restrict_l(ctx, u, l));
    RC(fill(ctx, u, l - 1, sg, 7));
    RC(copy_l(ctx, u1, u, nullptr, l - 1));
    RC(residual(ctx, r, u, b, l, p));
    // r's ghost fills (src/multigrid.jl:80,83) are not read by any later operation
    RC(restrict_l(ctx, r, l));
    RC(postrestrict(ctx, b, u, r, l, pc));
  }
  RC(gs_iter(ctx, u, b, 1, op3(op, k2, s, omega), ntop, sg));
  for (int l = 2; l <= lmax; ++l) {
    const Op3 p = op3(op, k2, level_scale(s, l), omega);
    RC(copy_l(ctx, u1, u, u1, l - 1));
    RC(fill(ctx, u1, l - 1, sg, 7));
    RC(interp_add(ctx, u, u1, l));
    RC(fill(ctx, u, l, sg, 7));
    RC(gs_iter(ctx, u, b, l, p, nup, sg));
    // after sweeps that write their own copy and mirror ghosts this fill would change
    // nothing: those ghosts are current, and the refinement ghosts interpolate level
    // l - 1, which has not changed since the fill above
    if (!gs_pushes(ctx, p)) RC(fill(ctx, u, l, sg, 7));
  }
  return SRMG_OK;
}

int leafnorm(srmg_ctx *ctx, const double *u, const double *b, double s, int op, double k2, int mode, int slot) {
  constexpr int NT = 256;
  int total = 0;
  std::vector<int> grids(ctx->nlev);
  for (int l = 1; l <= ctx->nlev; ++l) {
    const int n = ctx->nblk_host[l - 1];
    grids[l - 1] = n ? std::min(grid3((int64_t)n * 4096, NT), 148 * 4) : 0;
    total += grids[l - 1];
  }
  RC(ensure(ctx, ctx->part, sizeof(double) * std::max(total, 1)));
  double *part = (double *)ctx->part.p;
  int off = 0;
  for (int l = 1; l <= ctx->nlev; ++l) {
    if (!grids[l - 1]) continue;
    const double wl = 1.0 / (double)((int64_t)1 << (3 * (l - 1)));
    k3_leafsq<NT><<<grids[l - 1], NT, 0, ctx->stream>>>(part + off, u, b, view(ctx, l),
                                                       op3(op, k2, level_scale(s, l), 1.0), wl, mode);
    ctx->launches++;
    off += grids[l - 1];
  }
  double *out = (double *)ctx->small.p + slot;
  if (total == 0) {
    CK(cudaMemsetAsync(out, 0, sizeof(double), ctx->stream));
    return SRMG_OK;
  }
  k_reduce_sqrt<1024><<<1, 1024, 0, ctx->stream>>>(out, part, total);
  ctx->launches++;
  return SRMG_OK;
}

int corner_code(const int64_t f[3]) {
  for (int d = 0; d < 3; ++d)
    if (f[d] < -1 || f[d] > 1) return -1;
  if (!f[0] && !f[1] && !f[2]) return -1;
  return (int)((f[0] + 1) + 3 * (f[1] + 1) + 9 * (f[2] + 1));
}

int pack3(const int64_t v[3], int add) {
  return (int)((v[0] + add) | ((v[1] + add) << 2) | ((v[2] + add) << 4));
}

}  // namespace

// the D = 3 part of ensure_gs_push: octrees whose sweeps do not push by rule
int srmg::d3_ensure_push(srmg_ctx *ctx) { return ensure_push3(ctx); }

// ------------------------------------------------------------------ tree upload

extern "C" int srmg_set_tree3(srmg_ctx *ctx, int nlev, const int64_t *npairs, const srmg_pair3 *const *pairs,
                              const int64_t *nnb, const srmg_neighbor3 *const *nb, const int64_t *nbd,
                              const srmg_boundary3 *const *bd, const int64_t *nrb, const srmg_refbnd3 *const *rb,
                              const int64_t *nch, const srmg_child3 *const *ch, uint64_t generation) {
  if (ctx && ctx->async_pending)
    return fail(ctx, SRMG_ERR_BADARG, "an asynchronous solve is in flight on this context: call srmg_solve_wait first");
  if (!ctx) return SRMG_ERR_BADARG;
  if (ctx->D != 3) return fail(ctx, SRMG_ERR_BADARG, "srmg_set_tree3 needs a context created with D = 3");
  if (nlev < 1 || nlev > 20 || !npairs || !pairs || !nnb || !nb || !nbd || !bd || !nrb || !rb || !nch || !ch)
    return fail(ctx, SRMG_ERR_BADARG, "srmg_set_tree3: bad level count or null arrays");
  cudaSetDevice(ctx->device);
  int64_t max_blk = 0;
  for (int l = 0; l < nlev; ++l) {
    if (npairs[l] < 0 || (npairs[l] > 0 && !pairs[l]) || npairs[l] > (int64_t)INT32_MAX / 32)
      return fail(ctx, SRMG_ERR_BADTREE, "level %d: bad block count", l + 1);
    for (int64_t p = 0; p < npairs[l]; ++p) {
      const srmg_pair3 &pr = pairs[l][p];
      if (pr.blk < 1 || pr.blk >= INT32_MAX / 2)
        return fail(ctx, SRMG_ERR_BADTREE, "level %d: block index out of range", l + 1);
      for (int d = 0; d < 3; ++d)
        if (pr.coord[d] < 1 || pr.coord[d] > (1 << 22))
          return fail(ctx, SRMG_ERR_BADTREE, "level %d: block coordinate out of range", l + 1);
      max_blk = std::max(max_blk, pr.blk);
    }
  }
  std::vector<int> lev_of(max_blk + 1, 0), idx_of(max_blk + 1, -1);
  for (int l = 0; l < nlev; ++l)
    for (int64_t p = 0; p < npairs[l]; ++p) {
      const int64_t b = pairs[l][p].blk;
      if (lev_of[b]) return fail(ctx, SRMG_ERR_BADTREE, "block %lld appears twice in the tree", (long long)b);
      lev_of[b] = l + 1;
      idx_of[b] = (int)p;
    }
  auto at = [&](int64_t b, int l) { return b >= 1 && b <= max_blk && lev_of[b] == l; };
  std::vector<std::vector<int4>> hb(nlev), hf(nlev), hc(nlev);
  std::vector<std::vector<int>> hm(nlev);
  bool corners = false;
  bool merge_fill = true;
  for (int l = 0; l < nlev; ++l) {
    const int lv = l + 1;
    hb[l].resize(npairs[l]);
    hm[l].assign(npairs[l], 0);
    hf[l].assign(27 * npairs[l], make_int4(FACE_NONE, 0, 0, 0));
    for (int64_t p = 0; p < npairs[l]; ++p) {
      const srmg_pair3 &pr = pairs[l][p];
      hb[l][p] = make_int4((int)(pr.blk - 1), (int)pr.coord[0], (int)pr.coord[1], (int)pr.coord[2]);
    }
    auto set = [&](int64_t blk, int code, int4 v) -> int {
      int4 &slot = hf[l][27 * idx_of[blk] + code];
      if (slot.x != FACE_NONE)
        return fail(ctx, SRMG_ERR_BADTREE, "level %d: ghost direction %d of block %lld written twice", lv, code,
                    (long long)blk);
      slot = v;
      const int nz = (code % 3 != 1) + ((code / 3) % 3 != 1) + (code / 9 != 1);
      if (nz > 1) corners = true;
      return SRMG_OK;
    };
    if (nnb[l] < 0 || (nnb[l] > 0 && !nb[l])) return fail(ctx, SRMG_ERR_BADTREE, "level %d: neighbours", lv);
    for (int64_t k = 0; k < nnb[l]; ++k) {
      const srmg_neighbor3 &e = nb[l][k];
      const int64_t mf[3] = {-e.face[0], -e.face[1], -e.face[2]};
      const int code = corner_code(mf);
      if (code < 0 || !at(e.from, lv) || !at(e.to, lv))
        return fail(ctx, SRMG_ERR_BADTREE, "level %d: malformed neighbour edge", lv);
      RC(set(e.to, code, make_int4(FACE_NEIGHBOR, (int)(e.from - 1), 0, 0)));
    }
    if (nbd[l] < 0 || (nbd[l] > 0 && !bd[l])) return fail(ctx, SRMG_ERR_BADTREE, "level %d: boundaries", lv);
    for (int64_t k = 0; k < nbd[l]; ++k) {
      const srmg_boundary3 &e = bd[l][k];
      const int code = corner_code(e.face);
      bool ok = code >= 0 && at(e.block, lv) && e.level == lv && (e.bnd[0] || e.bnd[1] || e.bnd[2]);
      for (int d = 0; d < 3 && ok; ++d) ok = e.bnd[d] == 0 || e.bnd[d] == e.face[d];
      if (!ok) return fail(ctx, SRMG_ERR_BADTREE, "level %d: malformed boundary edge", lv);
      RC(set(e.block, code, make_int4(FACE_BOUNDARY, 0, pack3(e.bnd, 1), 0)));
    }
    if (nrb[l] < 0 || (nrb[l] > 0 && !rb[l])) return fail(ctx, SRMG_ERR_BADTREE, "level %d: refboundaries", lv);
    for (int64_t k = 0; k < nrb[l]; ++k) {
      const srmg_refbnd3 &e = rb[l][k];
      const int code = corner_code(e.face);
      bool ok = code >= 0 && lv >= 2 && at(e.fine, lv) && at(e.coarse, lv - 1);
      for (int d = 0; d < 3 && ok; ++d) ok = e.subblock[d] == 1 || e.subblock[d] == 2;
      if (!ok) return fail(ctx, SRMG_ERR_BADTREE, "level %d: malformed refinement boundary", lv);
      RC(set(e.fine, code, make_int4(FACE_REFBND, (int)(e.coarse - 1), pack3(e.subblock, 0), 0)));
    }
    // a boundary ghost mirrors, along the directions where its bnd is zero, a ghost that
    // must not itself be a boundary ghost for copy and boundary to share a launch
    for (size_t k = 0; k < hf[l].size(); ++k) {
      const int4 v = hf[l][k];
      if (v.x != FACE_BOUNDARY) continue;
      const int code = (int)(k % 27);
      const int f[3] = {code % 3 - 1, (code / 3) % 3 - 1, code / 9 - 1};
      int g[3];
      for (int d = 0; d < 3; ++d) g[d] = ((v.z >> (2 * d)) & 3) - 1 ? 0 : f[d];
      if (!g[0] && !g[1] && !g[2]) continue;
      if (hf[l][k - code + (g[0] + 1) + 3 * (g[1] + 1) + 9 * (g[2] + 1)].x == FACE_BOUNDARY) merge_fill = false;
    }
    if (nch[l] < 0 || (nch[l] > 0 && !ch[l])) return fail(ctx, SRMG_ERR_BADTREE, "level %d: children", lv);
    hc[l].resize(nch[l]);
    for (int64_t k = 0; k < nch[l]; ++k) {
      const srmg_child3 &e = ch[l][k];
      bool ok = lv >= 2 && at(e.fine, lv) && at(e.coarse, lv - 1);
      for (int d = 0; d < 3 && ok; ++d) ok = e.subblock[d] == 1 || e.subblock[d] == 2;
      if (!ok) return fail(ctx, SRMG_ERR_BADTREE, "level %d: malformed child edge", lv);
      hc[l][k] = make_int4((int)(e.fine - 1), (int)(e.coarse - 1), pack3(e.subblock, 0), 0);
      const int bit = 1 << ((int)(e.subblock[0] - 1) + 2 * (int)(e.subblock[1] - 1) + 4 * (int)(e.subblock[2] - 1));
      int &m = hm[l - 1][idx_of[e.coarse]];
      if (m & bit) return fail(ctx, SRMG_ERR_BADTREE, "level %d: two children cover one octant", lv);
      m |= bit;
    }
  }
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  };
  std::vector<size_t> ob(nlev), om(nlev), of(nlev), oc(nlev);
  for (int l = 0; l < nlev; ++l) {
    ob[l] = take(hb[l].size() * sizeof(int4));
    om[l] = take(hm[l].size() * sizeof(int));
    of[l] = take(hf[l].size() * sizeof(int4));
    oc[l] = take(hc[l].size() * sizeof(int4));
  }
  std::vector<char> host(std::max<size_t>(off, 256), 0);
  for (int l = 0; l < nlev; ++l) {
    memcpy(host.data() + ob[l], hb[l].data(), hb[l].size() * sizeof(int4));
    memcpy(host.data() + om[l], hm[l].data(), hm[l].size() * sizeof(int));
    memcpy(host.data() + of[l], hf[l].data(), hf[l].size() * sizeof(int4));
    memcpy(host.data() + oc[l], hc[l].data(), hc[l].size() * sizeof(int4));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  free_tree(ctx);
  void *d = nullptr;
  if (cudaMalloc(&d, host.size()) != cudaSuccess)
    return fail(ctx, SRMG_ERR_NOMEM, "tree allocation of %zu bytes", host.size());
  ctx->d_tree = d;
  CK(cudaMemcpyAsync(d, host.data(), host.size(), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  char *base = (char *)d;
  ctx->nlev = nlev;
  ctx->lv3.assign(nlev, Dev3Level{});
  ctx->nblk_host.resize(nlev);
  ctx->nch_host.resize(nlev);
  for (int l = 0; l < nlev; ++l) {
    Dev3Level &L = ctx->lv3[l];
    L.nblk = (int)hb[l].size();
    L.nch = (int)hc[l].size();
    L.blocks = (int4 *)(base + ob[l]);
    L.mask = (int *)(base + om[l]);
    L.faces = (int4 *)(base + of[l]);
    L.child = (int4 *)(base + oc[l]);
    ctx->nblk_host[l] = L.nblk;
    ctx->nch_host[l] = L.nch;
  }
  ctx->lv.clear();
  ctx->max_blk = max_blk;
  ctx->generation = generation;
  ctx->has_corners = corners;
  ctx->merge_fill = merge_fill;
  ctx->nitems = 1;
  ctx->has_tree = true;
  return SRMG_OK;
}

// ------------------------------------------------------------------ entry-point bodies

int srmg::d3_fill_ghost(srmg_ctx *ctx, double *u, int level, const int8_t *bc, int mask) {
  if (level < 1 || level > ctx->nlev) return fail(ctx, SRMG_ERR_BADARG, "fill_ghost: bad level");
  return fill(ctx, u, level, signs27(bc), mask);
}

int srmg::d3_gs_level(srmg_ctx *ctx, double *u, const double *b, int level, double omega, double sl, int op,
                      double k2, int colour) {
  const int ncol = op == SRMG_OP_LAPLACIAN4 ? 4 : 2;
  if (level < 1 || level > ctx->nlev || colour < 0 || colour >= ncol)
    return fail(ctx, SRMG_ERR_BADARG, "gs_level: bad arguments");
  return gs_colour(ctx, u, b, level, op3(op, k2, sl, omega), colour);
}

int srmg::d3_gs_iter(srmg_ctx *ctx, double *u, const double *b, int level, double omega, double sl, int n, int op,
                     double k2, const int8_t *bc) {
  if (level < 1 || level > ctx->nlev || n < 0) return fail(ctx, SRMG_ERR_BADARG, "gs_iter: bad arguments");
  return gs_iter(ctx, u, b, level, op3(op, k2, sl, omega), n, signs27(bc));
}

int srmg::d3_residual_level(srmg_ctx *ctx, double *r, const double *u, const double *b, int level, double sl,
                            int op, double k2) {
  if (level < 1 || level > ctx->nlev) return fail(ctx, SRMG_ERR_BADARG, "residual_level: bad level");
  return residual(ctx, r, u, b, level, op3(op, k2, sl, 1.0));
}

int srmg::d3_restrict_level(srmg_ctx *ctx, double *u, int level) {
  if (level < 1 || level > ctx->nlev) return fail(ctx, SRMG_ERR_BADARG, "restrict_level: bad level");
  return restrict_l(ctx, u, level);
}

int srmg::d3_interp_add_level(srmg_ctx *ctx, double *u, const double *u1, int level) {
  if (level < 1 || level > ctx->nlev) return fail(ctx, SRMG_ERR_BADARG, "interp_add_level: bad level");
  return interp_add(ctx, u, u1, level);
}

int srmg::d3_postrestrict_level(srmg_ctx *ctx, double *b, const double *u, const double *r, int level, double s,
                                int op, double k2) {
  if (level < 1 || level > ctx->nlev) return fail(ctx, SRMG_ERR_BADARG, "postrestrict: bad level");
  return postrestrict(ctx, b, u, r, level, op3(op, k2, s, 1.0));
}

int srmg::d3_rhs_level(srmg_ctx *ctx, double *q1, const double *q, int level, int op) {
  if (level < 1 || level > ctx->nlev) return fail(ctx, SRMG_ERR_BADARG, "rhs_level: bad level");
  const int n = ctx->nblk_host[level - 1];
  if (n) {
    k3_rhs<<<grid3((int64_t)n * 4096, 256), 256, 0, ctx->stream>>>(q1, q, view(ctx, level), op);
    ctx->launches++;
  }
  return SRMG_OK;
}

int srmg::d3_vcycle(srmg_ctx *ctx, double *u, double *b, double *r, double *u1, double s, int op, double k2,
                    const int8_t *bc, int lmax, int ndown, int ntop, int nup, double omega) {
  return vcycle(ctx, u, b, r, u1, s, op, k2, signs27(bc), lmax, ndown, ntop, nup, omega);
}

int srmg::d3_fmg(srmg_ctx *ctx, double *u, double *b, double *r, double *u1, double s, int op, double k2,
                 const int8_t *bc, int ndown, int ntop, int nup, double omega) {
  const Signs27 sg = signs27(bc);
  int lmax = 0;
  for (int l = 1; l <= ctx->nlev; ++l)
    if (ctx->nblk_host[l - 1] > 0) lmax = l;
  for (int l = lmax; l >= 2; --l) {
    const double sl = level_scale(s, l);
    RC(restrict_l(ctx, u, l));
    RC(fill(ctx, u, l - 1, sg, 7));
    RC(residual(ctx, r, u, b, l, op3(op, k2, sl, omega)));
    RC(restrict_l(ctx, r, l));
    RC(postrestrict(ctx, b, u, r, l, op3(op, k2, 4 * sl, omega)));
  }
  for (int l = 1; l <= lmax; ++l) {
    RC(copy_l(ctx, u1, u, nullptr, l));
    if (l > 1) {
      RC(copy_l(ctx, u1, u, u1, l - 1));
      RC(fill(ctx, u1, l - 1, sg, 7));
      RC(interp_add(ctx, u, u1, l));
    }
    RC(fill(ctx, u, l, sg, 7));
    RC(vcycle(ctx, u, b, r, u1, s, op, k2, sg, l, ndown, ntop, nup, omega));
  }
  return SRMG_OK;
}

int srmg::d3_leafnorm(srmg_ctx *ctx, const double *u, const double *b, double s, int op, double k2, int mode,
                      int slot) {
  return leafnorm(ctx, u, b, s, op, k2, mode, slot);
}

// FP64 tolerance loop on the per-operation V-cycle (srmg_solve for D = 3).
int srmg::d3_solve(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, double s, int op, double k2,
                   const int8_t *bc, const srmg_solve_opts *o, srmg_stats *st) {
  if (o->mode != SRMG_MODE_FP64)
    return fail(ctx, SRMG_ERR_UNSUPPORTED, "three-dimensional solves run in FP64 mode");
  if (!(o->tol > 0) || o->max_cycles < 0 || o->ndown < 0 || o->nup < 0 || o->ntop < 0)
    return fail(ctx, SRMG_ERR_BADARG, "srmg_solve: bad options");
  memset(st, 0, sizeof(*st));
  const size_t bytes = (size_t)nblk_alloc * S3 * sizeof(double);
  for (int i : {2, 3, 4}) RC(ensure(ctx, ctx->f64[i], bytes));
  double *r = (double *)ctx->f64[2].p, *u1 = (double *)ctx->f64[3].p, *bw = (double *)ctx->f64[4].p;
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  CK(cudaMemcpyAsync(bw, b, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  RC(leafnorm(ctx, u, b, s, op, k2, 1, 1));
  RC(leafnorm(ctx, u, bw, s, op, k2, 0, 0));
  RC(read_small(ctx, 2));
  const double bn = ctx->h_small[1] > 0 ? ctx->h_small[1] : 1.0;
  st->bnorm = ctx->h_small[1];
  double rel = ctx->h_small[0] / bn;
  st->initial_rel = rel;
  int c = 0;
  while (rel > o->tol && c < o->max_cycles) {
    RC(vcycle_ops(ctx, u, bw, r, u1, s, op, k2, 0, bc, 0, o->ndown, o->ntop, o->nup, o->omega, 1));
    ++c;
    RC(leafnorm(ctx, u, bw, s, op, k2, 0, 0));
    RC(read_small(ctx, 1));
    rel = ctx->h_small[0] / bn;
    if (!std::isfinite(rel)) {
      st->status = SRMG_ERR_DIVERGED;
      break;
    }
  }
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  CK(cudaEventSynchronize(ctx->ev1));
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  st->device_ms = ms;
  st->cycles = c;
  st->rel_residual = rel;
  if (st->status) return fail(ctx, st->status, "residual is not finite after %d cycles", c);
  return SRMG_OK;
}

// One launch of the 3D sequencer over `nops` records at d_ops (device memory), on the
// context's stream.  The barrier counter and error word are the persistent engine's
// (zeroed here, read by engine_check).
int srmg::seq_launch3(srmg_ctx *ctx, const void *d_ops, int nops) {
  if (nops <= 0) return SRMG_OK;
  const void *fn = (const void *)k3_sequencer;
  if (ctx->num_sms == 0) CK(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->device));
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kSeq3Threads, 0));
  if (per_sm < 1) return fail(ctx, SRMG_ERR_CUDA, "sequencer kernel cannot be resident (occupancy 0)");
  RC(ensure(ctx, ctx->sync, 256 + sizeof(int) * (size_t)ctx->nitems));
  CK(cudaMemsetAsync(ctx->sync.p, 0, 256, ctx->stream));
  const SeqOp3 *ops = (const SeqOp3 *)d_ops;
  unsigned *bar = (unsigned *)ctx->sync.p;
  int *err = (int *)((char *)ctx->sync.p + 128);
  long long timeout = 2000000000LL;  // 2 s per barrier wait
  void *args[] = {&ops, &nops, &bar, &err, &timeout};
  CK(cudaLaunchCooperativeKernel(fn, dim3(ctx->num_sms * std::min(per_sm, kSeq3PerSM)), dim3(kSeq3Threads), args, 0, ctx->stream));
  ctx->launches++;
  return SRMG_OK;
}

size_t srmg::seq3_op_bytes() { return sizeof(SeqOp3); }
