// srmg_kernels.cuh -- per-operation CUDA kernels for the FAS multigrid on a block tree.
//
// Block geometry is fixed at compile time: M = 16 valid cells per side, G = 2 ghost
// layers, S = 20, one block = S*S elements, dim 1 (r, "x") fastest.  All local indices
// here are 0-based: valid cells are x, y in [2, 17]; element (x, y) of block blk is at
// blk*400 + x + 20*y.  Block ids are 0-based on the device.
//
// Each kernel restates one reference routine and keeps its floating-point operation
// order where the result must be bit-exact (ghost copies, mirrors, linear
// interpolation, restriction, and the stencils of the smoother and the residual);
// __dadd_rn/__dmul_rn stop the compiler from contracting those into FMAs, and fma()
// stands where the reference calls muladd.  The same bodies run as separate kernels
// and inside the sequencer's single launch, with identical results.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace srmg {

constexpr int kM = 16;
constexpr int kG = 2;
constexpr int kS = kM + 2 * kG;
constexpr int kSS = kS * kS;
// Per-item operator table of the persistent engine: s_l [32], stencil centre_l [32] and
// -(omega / diagonal)_l [32], indexed by level l.
constexpr int kParStride = 96;
// Blocks per norm chunk: the leaf norms are summed per chunk of up to this many
// consecutive blocks of one item and level, then per item over its chunks.
constexpr int kNormChunk = 4;
// Per-item result record of a device solve loop: {norm, |b|, initial norm, V-cycles run,
// defect-correction steps run (mixed mode; 0 in FP64 mode)}.
constexpr int kItemRec = 5;

// Face numbering (the four StarStencil directions): 0 = -r, 1 = +r, 2 = -z, 3 = +z.
enum FaceType : int { FACE_NONE = 0, FACE_NEIGHBOR = 1, FACE_BOUNDARY = 2, FACE_REFBND = 3 };

// Per-level device view of the tree.
struct LevelView {
  const int4 *blocks;   // [nblk] {blk, coord_r, coord_z, child_mask}; coords 1-based
  const int4 *faces;    // [nblk*4] {type, src_blk, sb_r, sb_z}
  const int4 *child;    // [nch] {fine_blk, coarse_blk, sb_r, sb_z} (fine at this level)
  int nblk;
  int nch;
  int level;
  // BoxStencil trees only (else null): [nblk*4] corner faces, corner q at direction
  // (2 (q & 1) - 1, 2 (q >> 1) - 1); {type, src_blk, a, b} with (a, b) the subblock of a
  // refinement corner or the boundary's bnd vector (components -1, 0, +1) of a
  // boundary corner.
  const int4 *cfaces;
};

// Operator parameters for one level.
template <typename T>
struct OpParams {
  int op;        // 0 Laplacian, 1 Helmholtz, 2 compact order-4 Laplacian
  int geom;      // 0 Cartesian, 1 cylindrical r = dim 1, 2 cylindrical r = dim 2
  T s;           // level scale s_l
  T centre;      // -4 or -4 - s_l*k2 (stencil centre, src/helmholtz.jl:43-45)
  T nwc;         // -(omega / diagelm)  (src/multigrid.jl:177)
  T omega;       // the relaxation factor itself (order 4 divides by a per-cell diagonal)
};

struct Signs { double v[9]; };  // boundary-condition table as doubles, column-major

// Radial weights (2i-2)/(2i-1), 2i/(2i-1) tabulated by 1-based global index
// (src/laplacian.jl:104-106).
template <typename T>
struct WTab { const T *wm; const T *wp; };

__device__ __forceinline__ int face_sign_index(int f) {
  // bnd == face for a star stencil; index (1 + bnd1) + 3 (1 + bnd2)
  return f == 0 ? 3 : f == 1 ? 5 : f == 2 ? 1 : 7;
}

template <typename T> __device__ __forceinline__ T dadd(T a, T b);
template <> __device__ __forceinline__ double dadd<double>(double a, double b) { return __dadd_rn(a, b); }
template <> __device__ __forceinline__ float dadd<float>(float a, float b) { return __fadd_rn(a, b); }
template <typename T> __device__ __forceinline__ T dmul(T a, T b);
template <> __device__ __forceinline__ double dmul<double>(double a, double b) { return __dmul_rn(a, b); }
template <> __device__ __forceinline__ float dmul<float>(float a, float b) { return __fmul_rn(a, b); }

// Stencil weights of cell (x, y) of a block at 1-based coords (cr, cz).
template <typename T>
struct W5 { T zm, rm, rp, zp; };

template <typename T>
__device__ __forceinline__ W5<T> weights(const WTab<T> &wt, int geom, int cr, int cz, int x, int y) {
  W5<T> w{T(1), T(1), T(1), T(1)};
  if (geom == 1) {
    const int i = x - 1 + kM * (cr - 1);
    w.rm = wt.wm[i];
    w.rp = wt.wp[i];
  } else if (geom == 2) {
    const int j = y - 1 + kM * (cz - 1);
    w.zm = wt.wm[j];
    w.zp = wt.wp[j];
  }
  return w;
}

// applystencil, order 2 (src/laplacian.jl:25-49,78-118; src/helmholtz.jl:17-57):
// v = 0; v += c * u[I+S] over S = (0,-1), (-1,0), (0,0), (1,0), (0,1), each product and
// sum rounded on its own: the uncontracted reading of the reference's @fastmath
// stencil, and a rounding that does not depend on the context the body is inlined
// into (the compiler's choice of FMAs would).
template <typename T>
__device__ __forceinline__ T apply5(const T *ub, int x, int y, const W5<T> &w, T centre) {
  const int o = x + kS * y;
  T v = dadd<T>(T(0), dmul<T>(w.zm, ub[o - kS]));
  v = dadd<T>(v, dmul<T>(w.rm, ub[o - 1]));
  v = dadd<T>(v, dmul<T>(centre, ub[o]));
  v = dadd<T>(v, dmul<T>(w.rp, ub[o + 1]));
  v = dadd<T>(v, dmul<T>(w.zp, ub[o + kS]));
  return v;
}

// ---- compact order-4 Laplacian, LaplacianDiscretization{2,4} -------------------------
// applystencil (src/laplacian.jl:133-202): a 3x3 literal, rows along dimension 1 and
// columns along dimension 2, accumulated column-major (k = (d1 + 1) + 3 (d2 + 1),
// v = 0; v += c_k u) and divided by 6.  The cylindrical coefficients are integer
// polynomials of the radial 1-based global index i divided as doubles; every operation
// is rounded on its own (no contraction), so results are bit-exact against the oracle.
__device__ __forceinline__ void coeffs9(int geom, int64_t ir, int64_t iz, double c[9]) {
  if (geom == 0) {
    c[0] = 1; c[1] = 4; c[2] = 1; c[3] = 4; c[4] = -20; c[5] = 4; c[6] = 1; c[7] = 4; c[8] = 1;
    return;
  }
  const int64_t i = geom == 1 ? ir : iz;
  const int64_t q = 2 * i - 1;
  const double am = __ddiv_rn((double)(2 * (i - 1)), (double)q);
  const double ap = __ddiv_rn((double)(2 * i), (double)q);
  const double q3 = (double)(q * q * q);
  const double em = __ddiv_rn((double)(4 * (-2 + 9 * i - 16 * i * i + 8 * i * i * i)), q3);
  const double cc = __ddiv_rn((double)(-16 * (1 - 5 * i + 5 * i * i)), (double)((1 - 2 * i) * (1 - 2 * i)));
  const double ep = __ddiv_rn((double)(4 * (1 + i - 8 * i * i + 8 * i * i * i)), q3);
  if (geom == 1) {  // r = dimension 1 (src/laplacian.jl:156-164)
    c[0] = am; c[1] = 4; c[2] = ap; c[3] = em; c[4] = cc; c[5] = ep; c[6] = am; c[7] = 4; c[8] = ap;
  } else {          // r = dimension 2 (src/laplacian.jl:176-184)
    c[0] = am; c[1] = em; c[2] = am; c[3] = 4; c[4] = cc; c[5] = 4; c[6] = ap; c[7] = ep; c[8] = ap;
  }
}

template <typename T>
__device__ __forceinline__ T apply9(const T *ub, int x, int y, int geom, int64_t ir, int64_t iz) {
  double c[9];
  coeffs9(geom, ir, iz, c);
  T v = T(0);
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const int d1 = k % 3 - 1, d2 = k / 3 - 1;
    v = dadd<T>(v, dmul<T>(T(c[k]), ub[(x + d1) + kS * (y + d2)]));
  }
  return v / T(6);
}

// diagelm, order 4 (src/laplacian.jl:150-151, 205-209).
__device__ __forceinline__ double diagelm4(int geom, int64_t ir, int64_t iz) {
  if (geom == 0) return -20.0 / 6.0;
  const int64_t i = geom == 1 ? ir : iz;
  return __ddiv_rn(__ddiv_rn((double)(-16 * (1 - 5 * i + 5 * i * i)), (double)((1 - 2 * i) * (1 - 2 * i))), 6.0);
}

// 1-based global indices of local cell (x, y) of a block at 1-based coords (cr, cz)
// (global_first, src/mesh.jl:76-78).
__device__ __forceinline__ int64_t gidx(int c, int x) { return (int64_t)kM * (c - 1) + x - 1; }

// The left-hand side of any supported discretisation at cell (x, y).
template <typename T>
__device__ __forceinline__ T lhs_apply(const T *ub, int x, int y, const OpParams<T> &p, const WTab<T> &wt,
                                       int cr, int cz) {
  if (p.op == 2) return apply9<T>(ub, x, y, p.geom, gidx(cr, x), gidx(cz, y));
  const W5<T> w = weights<T>(wt, p.geom, cr, cz, x, y);
  return apply5<T>(ub, x, y, w, p.centre);
}

// ---- ghost fill (src/connectivity.jl:155-258) --------------------------------------
template <typename T>
__device__ __forceinline__ void fill_corner_cell(T *__restrict__ u, const LevelView &lv, const Signs &sg, int phase,
                                                 int64_t t);

// One warp per (block, face): lane -> (layer g = lane/16, position k = lane%16).  On a
// BoxStencil tree (lv.cfaces set) the launch covers one pass (mask 1, 2 or 4) or the
// copy and boundary passes together (mask 3), and also fills the corner cells of those
// passes (fill_corner_cell).
template <typename T>
__device__ __forceinline__ void d_fill_ghost(T *__restrict__ u, LevelView lv, Signs sg, int mask) {
  const int lane = threadIdx.x & 31;
  const int warps_per_cta = blockDim.x >> 5;
  const int g = lane >> 4, k = lane & 15;
  const int total = lv.nblk * 4;
  for (int w = blockIdx.x * warps_per_cta + (threadIdx.x >> 5); w < total;
       w += gridDim.x * warps_per_cta) {
    const int bi = w >> 2, f = w & 3;
    const int4 fi = lv.faces[w];
    if (fi.x == FACE_NONE) continue;
    const int blk = lv.blocks[bi].x;
    T *ub = u + (int64_t)blk * kSS;
    int x, y;
    if (f == 0) { x = g; y = 2 + k; }
    else if (f == 1) { x = 18 + g; y = 2 + k; }
    else if (f == 2) { x = 2 + k; y = g; }
    else { x = 2 + k; y = 18 + g; }
    if (fi.x == FACE_NEIGHBOR) {
      if (!(mask & 1)) continue;
      // _fill_ghost_copy! (src/connectivity.jl:184-198): ghost <- neighbour's valid
      // cell M positions away along the face normal.
      const T *src = u + (int64_t)fi.y * kSS;
      int sx = x, sy = y;
      if (f == 0) sx = x + kM; else if (f == 1) sx = x - kM;
      else if (f == 2) sy = y + kM; else sy = y - kM;
      ub[x + kS * y] = src[sx + kS * sy];
    } else if (fi.x == FACE_BOUNDARY) {
      if (!(mask & 2)) continue;
      // fill_ghost_bnd! (src/connectivity.jl:217-231), mirrorghost (src/blockfield.jl:513-521)
      int mx = x, my = y;
      if (f == 0) mx = 2 * kG - 1 - x; else if (f == 1) mx = 2 * (kG + kM) - 1 - x;
      else if (f == 2) my = 2 * kG - 1 - y; else my = 2 * (kG + kM) - 1 - y;
      const T a = T(sg.v[face_sign_index(f)]);
      ub[x + kS * y] = dmul<T>(a, ub[mx + kS * my]);
    } else {
      if (!(mask & 4)) continue;
      // fill_ghost_interp! (src/connectivity.jl:251-258) + interp! (src/interp.jl:24-63)
      // from the coarse block's subblockbnd(subblock, -face) (src/blockfield.jl:416-434).
      const T *cb = u + (int64_t)fi.y * kSS;
      const int sbr = fi.z, sbz = fi.w;
      int jr, jz, ir, iz;  // coarse source cell and the 0/1 child offsets per dim
      if (f <= 1) {
        jr = (f == 0) ? (1 + 8 * sbr) : (2 + 8 * (sbr - 1));
        ir = g;
        jz = 2 + 8 * (sbz - 1) + (k >> 1);
        iz = k & 1;
      } else {
        jz = (f == 2) ? (1 + 8 * sbz) : (2 + 8 * (sbz - 1));
        iz = g;
        jr = 2 + 8 * (sbr - 1) + (k >> 1);
        ir = k & 1;
      }
      const int o = jr + kS * jz;
      if (mask & 8) {  // InterpCopy (src/interp.jl:66-85): the coarse cell's value itself
        ub[x + kS * y] = cb[o];
        continue;
      }
      T v = dmul<T>(T(0.5), cb[o]);
      v = dadd<T>(v, dmul<T>(T(0.25), cb[o + (2 * ir - 1)]));
      v = dadd<T>(v, dmul<T>(T(0.25), cb[o + kS * (2 * iz - 1)]));
      ub[x + kS * y] = v;
    }
  }
  if (lv.cfaces && (mask == 1 || mask == 2 || mask == 3 || mask == 4)) {
    const int64_t ct = (int64_t)lv.nblk * 16;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ct; t += (int64_t)gridDim.x * blockDim.x)
      fill_corner_cell<T>(u, lv, sg, mask, t);
  }
}

// ---- red-black Gauss-Seidel colour sweep (src/multigrid.jl:153-180, 238-243) ------
// Colour P updates valid cells with (x + y + 1) & 1 == P (0-based local indices).
// Ghost pushes of a colour sweep (2D trees, per-operation path): for every valid cell
// whose value a copy-and-boundary fill (fill_ghost! passes 1 and 2) writes into ghost
// cells, the list of those ghosts, CSR by (level-local block, cell): off[bi*256 + cell]
// .. off[bi*256 + cell + 1] index ent, ent = {ghost's index in the field, boundary-table
// entries of the mirrors on the way (low and high 4 bits, 15 = none)}.  The sweep that
// updates the cell writes them, so no fill launch has to follow it.  Built from the
// fill itself (srmg.cu, ensure_gs_push).  The boundary table reaches the sweep packed,
// two bits an entry (entry + 1: the pushes are used only where every entry is -1, 0 or 1).
struct PushView {
  const int *off;
  const int2 *ent;
};

template <typename T>
__device__ __forceinline__ void push_ghosts(T *__restrict__ u, const PushView &pv, unsigned sg, int bi, int x, int y,
                                            T v) {
  const int c = bi * 256 + (x - kG) + kM * (y - kG);
  const int e1 = pv.off[c + 1];
  for (int e = pv.off[c]; e < e1; ++e) {
    const int2 d = pv.ent[e];
    T w = v;
    // boundary-table entries are -1, 0 or 1: the products are exact in any order
    const int k1 = d.y & 15, k2 = d.y >> 4;
    if (k1 < 9) w = dmul<T>(T((int)((sg >> (2 * k1)) & 3u) - 1), w);
    if (k2 < 9) w = dmul<T>(T((int)((sg >> (2 * k2)) & 3u) - 1), w);
    u[d.x] = w;
  }
}

template <typename T, bool kPush>
__device__ __forceinline__ void d_gs_colour_impl(T *__restrict__ u, const T *__restrict__ b, LevelView lv,
                                                 OpParams<T> p, WTab<T> wt, int parity, PushView pv,
                                                 unsigned sg) {
  const int64_t total = (int64_t)lv.nblk * 128;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t >> 7), c = (int)(t & 127);
    const int y = 2 + (c >> 3);
    const int x = 2 + 2 * (c & 7) + ((parity ^ (y + 1)) & 1);
    const int4 bk = lv.blocks[bi];
    T *ub = u + (int64_t)bk.x * kSS;
    const W5<T> w = weights<T>(wt, p.geom, bk.y, bk.z, x, y);
    const T Lu = apply5<T>(ub, x, y, w, p.centre);
    const int o = x + kS * y;
    const T v = fma(p.s, b[(int64_t)bk.x * kSS + o], Lu);
    const T nv = fma(p.nwc, v, ub[o]);
    ub[o] = nv;
    if (kPush) push_ghosts<T>(u, pv, sg, bi, x, y, nv);
  }
}

template <typename T>
__device__ __forceinline__ void d_gs_colour(T *__restrict__ u, const T *__restrict__ b, LevelView lv,
                                            OpParams<T> p, WTab<T> wt, int parity) {
  d_gs_colour_impl<T, false>(u, b, lv, p, wt, parity, PushView{nullptr, nullptr}, 0u);
}

// ---- residual (src/multigrid.jl:309-323, 349-354): r = -(b + Lu/s) ---------------
template <typename T>
__device__ __forceinline__ void d_residual(T *__restrict__ r, const T *__restrict__ u, const T *__restrict__ b,
                           LevelView lv, OpParams<T> p, WTab<T> wt) {
  const int64_t total = (int64_t)lv.nblk * 256;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t >> 8), c = (int)(t & 255);
    const int x = 2 + (c & 15), y = 2 + (c >> 4);
    const int4 bk = lv.blocks[bi];
    const int64_t base = (int64_t)bk.x * kSS;
    const T Lu = lhs_apply<T>(u + base, x, y, p, wt, bk.y, bk.z);
    const int64_t o = base + x + kS * y;
    r[o] = -(b[o] + Lu / p.s);
  }
}

// ---- FAS coarse RHS (src/multigrid.jl:112-119, 331-344) ----------------------------
// For each Child edge of this level, on the coarse subblock: bf = -(r + L(u)/s_c).
template <typename T>
__device__ __forceinline__ void d_postrestrict(T *__restrict__ bf, const T *__restrict__ u, const T *__restrict__ r,
                               LevelView lv, const int2 *__restrict__ coord_of, OpParams<T> p,
                               WTab<T> wt) {
  const int64_t total = (int64_t)lv.nch * 64;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int e = (int)(t >> 6), c = (int)(t & 63);
    const int4 ch = lv.child[e];
    const int cblk = ch.y;
    const int x = 2 + 8 * (ch.z - 1) + (c & 7), y = 2 + 8 * (ch.w - 1) + (c >> 3);
    const int2 cc = coord_of[cblk];
    const int64_t base = (int64_t)cblk * kSS;
    const T Lu = lhs_apply<T>(u + base, x, y, p, wt, cc.x, cc.y);
    const int64_t o = base + x + kS * y;
    bf[o] = -(r[o] + Lu / p.s);
  }
}

// ---- restriction (src/restrict.jl:5-37) --------------------------------------------
// coarse = ((((0 + f00) + f10) + f01) + f11) / 4 for each Child edge of this level.
template <typename T>
__device__ __forceinline__ void d_restrict(T *__restrict__ u, LevelView lv) {
  const int64_t total = (int64_t)lv.nch * 64;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int e = (int)(t >> 6), c = (int)(t & 63);
    const int4 ch = lv.child[e];
    const int kx = c & 7, ky = c >> 3;
    const T *fb = u + (int64_t)ch.x * kSS + (2 + 2 * kx) + kS * (2 + 2 * ky);
    T f = dadd<T>(T(0), fb[0]);
    f = dadd<T>(f, fb[1]);
    f = dadd<T>(f, fb[kS]);
    f = dadd<T>(f, fb[kS + 1]);
    u[(int64_t)ch.y * kSS + (2 + 8 * (ch.z - 1) + kx) + kS * (2 + 8 * (ch.w - 1) + ky)] =
        dmul<T>(f, T(0.25));
  }
}

// ---- prolongation-add (src/interp.jl:24-63, 107-115): u_f += P(u1_c) -------------
template <typename T>
__device__ __forceinline__ void d_interp_add(T *__restrict__ u, const T *__restrict__ u1, LevelView lv) {
  const int64_t total = (int64_t)lv.nch * 256;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int e = (int)(t >> 8), c = (int)(t & 255);
    const int4 ch = lv.child[e];
    const int dx = c & 15, dy = c >> 4;
    const int ir = dx & 1, iz = dy & 1;
    const int jr = 2 + 8 * (ch.z - 1) + (dx >> 1), jz = 2 + 8 * (ch.w - 1) + (dy >> 1);
    const T *cb = u1 + (int64_t)ch.y * kSS;
    const int o = jr + kS * jz;
    T v = dmul<T>(T(0.5), cb[o]);
    v = dadd<T>(v, dmul<T>(T(0.25), cb[o + (2 * ir - 1)]));
    v = dadd<T>(v, dmul<T>(T(0.25), cb[o + kS * (2 * iz - 1)]));
    T *d = u + (int64_t)ch.x * kSS + (2 + dx) + kS * (2 + dy);
    *d = dadd<T>(v, *d);
  }
}

// ---- whole-block copy / difference over a level (src/blockfield.jl:557-576) ------
template <typename T>
__device__ __forceinline__ void d_copy_level(T *__restrict__ dst, const T *__restrict__ src, LevelView lv) {
  const int64_t total = (int64_t)lv.nblk * kSS;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t / kSS), c = (int)(t % kSS);
    const int64_t o = (int64_t)lv.blocks[bi].x * kSS + c;
    dst[o] = src[o];
  }
}

template <typename T>
__device__ __forceinline__ void d_diff_level(T *__restrict__ dst, const T *__restrict__ a1, const T *a2,
                             LevelView lv) {
  const int64_t total = (int64_t)lv.nblk * kSS;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t / kSS), c = (int)(t % kSS);
    const int64_t o = (int64_t)lv.blocks[bi].x * kSS + c;
    dst[o] = a1[o] - a2[o];
  }
}

// ---- residual norm pieces -----------------------------------------------------------
// Sum over the level's LEAF cells (cells of subblocks without a child) of
// w_l * f(x)^2, with f = residual (mode 0) or the field itself (mode 1).  One partial
// per CTA, written to part[blockIdx.x]: deterministic for a fixed grid.
// This is the value resnorm! (src/multigrid.jl:391-417) obtains by squaring every
// cell and restricting the squares down to level 1: a leaf cell of level l ends up
// weighted by 4^-(l-1).
template <typename T, int NT>
__global__ void __launch_bounds__(NT) k_leafsq(double *__restrict__ part, const T *__restrict__ u,
                                               const T *__restrict__ b, LevelView lv,
                                               OpParams<T> p, WTab<T> wt, double wl, int mode) {
  double acc = 0.0;
  const int64_t total = (int64_t)lv.nblk * 256;
  for (int64_t t = blockIdx.x * (int64_t)NT + threadIdx.x; t < total; t += (int64_t)gridDim.x * NT) {
    const int bi = (int)(t >> 8), c = (int)(t & 255);
    const int x = 2 + (c & 15), y = 2 + (c >> 4);
    const int4 bk = lv.blocks[bi];
    const int sub = ((x - 2) >> 3) + 2 * ((y - 2) >> 3);
    if ((bk.w >> sub) & 1) continue;  // covered by a child: not a leaf cell
    const int64_t base = (int64_t)bk.x * kSS;
    const int64_t o = base + x + kS * y;
    double v;
    if (mode == 0) {
      const T Lu = lhs_apply<T>(u + base, x, y, p, wt, bk.y, bk.z);
      v = (double)(-(b[o] + Lu / p.s));
    } else {
      v = (double)b[o];
    }
    acc = fma(v, v, acc);
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

// Final fixed-order reduction of n partials into out[0] (sqrt applied).
template <int NT>
__global__ void __launch_bounds__(NT) k_reduce_sqrt(double *__restrict__ out,
                                                    const double *__restrict__ part, int n) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += NT) acc += part[i];
  __shared__ double sh[NT / 32];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = (threadIdx.x < NT / 32) ? sh[threadIdx.x] : 0.0;
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if (threadIdx.x == 0) out[0] = sqrt(v);
  }
}

// gauss_seidel!(..., FourColors{P1,P2}) (src/multigrid.jl:206-232): cells
// (2 + 2a + p1, 2 + 2b + p2), u -= omega (Lu + s b) / c, unfused.
template <typename T, bool kPush>
__device__ __forceinline__ void d_gs4_impl(T *__restrict__ u, const T *__restrict__ b, LevelView lv, OpParams<T> p,
                                           int p1, int p2, PushView pv, unsigned sg) {
  const int64_t total = (int64_t)lv.nblk * 64;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t >> 6), c = (int)(t & 63);
    const int x = 2 + 2 * (c & 7) + p1, y = 2 + 2 * (c >> 3) + p2;
    const int4 bk = lv.blocks[bi];
    T *ub = u + (int64_t)bk.x * kSS;
    const int64_t ir = gidx(bk.y, x), iz = gidx(bk.z, y);
    const T Lu = apply9<T>(ub, x, y, p.geom, ir, iz);
    const int o = x + kS * y;
    const T cdiag = T(diagelm4(p.geom, ir, iz));
    const T upd = dmul<T>(p.omega, dadd<T>(Lu, dmul<T>(p.s, b[(int64_t)bk.x * kSS + o]))) / cdiag;
    const T nv = ub[o] - upd;
    ub[o] = nv;
    if (kPush) push_ghosts<T>(u, pv, sg, bi, x, y, nv);
  }
}

template <typename T>
__device__ __forceinline__ void d_gs4(T *__restrict__ u, const T *__restrict__ b, LevelView lv, OpParams<T> p, int p1, int p2) {
  d_gs4_impl<T, false>(u, b, lv, p, p1, p2, PushView{nullptr, nullptr}, 0u);
}

// rhs! over rhs_level! (src/multigrid.jl:363-388): q1 = R q on the valid cells.  Order
// 2: the identity (src/laplacian.jl:86-91,120-125).  Order 4: the literal
// (src/laplacian.jl:141-148,166-173,186-193) walked over its nonzero entries
// (0,-1), (-1,0), (0,0), (1,0), (0,1), then divided by 12.
template <typename T>
__global__ void k_rhs(T *__restrict__ q1, const T *__restrict__ q, LevelView lv, int op, int geom) {
  const int64_t total = (int64_t)lv.nblk * 256;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t >> 8), c = (int)(t & 255);
    const int x = 2 + (c & 15), y = 2 + (c >> 4);
    const int4 bk = lv.blocks[bi];
    const T *qb = q + (int64_t)bk.x * kSS;
    const int o = x + kS * y;
    if (op != 2) {
      q1[(int64_t)bk.x * kSS + o] = qb[o];
      continue;
    }
    T wzm = T(1), wrm = T(1), wrp = T(1), wzp = T(1);
    if (geom != 0) {
      const int64_t i = geom == 1 ? gidx(bk.y, x) : gidx(bk.z, y);
      const T wm = __ddiv_rn((double)(2 * i - 2), (double)(2 * i - 1));
      const T wp = __ddiv_rn((double)(2 * i), (double)(2 * i - 1));
      if (geom == 1) { wrm = wm; wrp = wp; } else { wzm = wm; wzp = wp; }
    }
    T v = T(0);
    v = dadd<T>(v, dmul<T>(wzm, qb[o - kS]));
    v = dadd<T>(v, dmul<T>(wrm, qb[o - 1]));
    v = dadd<T>(v, dmul<T>(T(8), qb[o]));
    v = dadd<T>(v, dmul<T>(wrp, qb[o + 1]));
    v = dadd<T>(v, dmul<T>(wzp, qb[o + kS]));
    q1[(int64_t)bk.x * kSS + o] = v / T(12);
  }
}

// Corner ghosts of a BoxStencil tree (src/connectivity.jl:155-258 with diagonal faces):
// 2 x 2 cells per corner, one thread (index t) per cell.  `mask` selects the passes:
// 1 = copy from the diagonal neighbour, 2 = boundary mirror, 4 = linear interpolation
// from the parent's subblockbnd cell (src/blockfield.jl:416-434, src/interp.jl:24-63).
// A boundary corner whose bnd is zero along one dimension mirrors the adjacent face's
// ghost cells, which fill_ghost! writes in an earlier pass.  fill_ghost! runs copy,
// boundary and interpolation in that order; here copy and boundary may share one launch
// (mask 3): such a corner then evaluates the face ghost it mirrors from that face's own
// source -- the neighbour's valid cell, or the mirrored valid cell -- with the same
// operations as the face pass, instead of reading it.  Interpolation (mask 4) stays a
// launch of its own after them: the boundary pass reads a refinement face's ghosts as
// they were before this fill.
template <typename T>
__device__ __forceinline__ T face_ghost_value(const T *__restrict__ u, const T *ub, const LevelView &lv,
                                              const Signs &sg, int bi, int f, int x, int y) {
  const int4 ff = lv.faces[4 * bi + f];
  if (ff.x == FACE_NEIGHBOR) {  // as the copy pass of d_fill_ghost
    const T *src = u + (int64_t)ff.y * kSS;
    int sx = x, sy = y;
    if (f == 0) sx = x + kM; else if (f == 1) sx = x - kM;
    else if (f == 2) sy = y + kM; else sy = y - kM;
    return src[sx + kS * sy];
  }
  if (ff.x == FACE_BOUNDARY) {  // as the boundary pass of d_fill_ghost
    int mx = x, my = y;
    if (f == 0) mx = 2 * kG - 1 - x; else if (f == 1) mx = 2 * (kG + kM) - 1 - x;
    else if (f == 2) my = 2 * kG - 1 - y; else my = 2 * (kG + kM) - 1 - y;
    return dmul<T>(T(sg.v[face_sign_index(f)]), ub[mx + kS * my]);
  }
  return ub[x + kS * y];  // a refinement face: not written by the copy and boundary passes
}

template <typename T>
__device__ __forceinline__ void fill_corner_cell(T *__restrict__ u, const LevelView &lv, const Signs &sg, int mask,
                                                 int64_t t) {
  {
    const int bi = (int)(t >> 4), q = (int)((t >> 2) & 3), cell = (int)(t & 3);
    const int4 fi = lv.cfaces[4 * bi + q];
    const int type = fi.x;
    if (type == FACE_NONE) return;
    if ((type == FACE_NEIGHBOR && !(mask & 1)) || (type == FACE_BOUNDARY && !(mask & 2)) ||
        (type == FACE_REFBND && !(mask & 4)))
      return;
    const int fr = 2 * (q & 1) - 1, fz = 2 * (q >> 1) - 1;  // ghost direction
    const int ir = cell & 1, iz = cell >> 1;
    const int x = (fr < 0 ? 0 : kM + kG) + ir, y = (fz < 0 ? 0 : kM + kG) + iz;
    T *ub = u + (int64_t)lv.blocks[bi].x * kSS;
    if (type == FACE_NEIGHBOR) {
      const T *src = u + (int64_t)fi.y * kSS;
      ub[x + kS * y] = src[(x - kM * fr) + kS * (y - kM * fz)];
    } else if (type == FACE_BOUNDARY) {
      const int b0 = fi.z, b1 = fi.w;
      const int mx = b0 < 0 ? 2 * kG - 1 - x : b0 > 0 ? 2 * (kG + kM) - 1 - x : x;
      const int my = b1 < 0 ? 2 * kG - 1 - y : b1 > 0 ? 2 * (kG + kM) - 1 - y : y;
      const T a = T(sg.v[(1 + b0) + 3 * (1 + b1)]);
      T src;
      if ((mask & 1) && (b0 == 0) != (b1 == 0)) {
        // the mirror lands in the ghost cells of the face along the zero component,
        // which the copy part of this launch writes: evaluate that cell directly
        const int f = b0 == 0 ? (fr < 0 ? 0 : 1) : (fz < 0 ? 2 : 3);
        src = face_ghost_value<T>(u, ub, lv, sg, bi, f, mx, my);
      } else {
        src = ub[mx + kS * my];
      }
      ub[x + kS * y] = dmul<T>(a, src);
    } else {
      const T *cb = u + (int64_t)fi.y * kSS;
      const int sbr = fi.z, sbz = fi.w;
      // subblockbnd(subblock, -face): the last cell of the subblock along a dimension
      // where the ghost lies below, the first where it lies above
      const int jr = fr < 0 ? 1 + 8 * sbr : 2 + 8 * (sbr - 1);
      const int jz = fz < 0 ? 1 + 8 * sbz : 2 + 8 * (sbz - 1);
      const int o = jr + kS * jz;
      T v = dmul<T>(T(0.5), cb[o]);
      v = dadd<T>(v, dmul<T>(T(0.25), cb[o + (2 * ir - 1)]));
      v = dadd<T>(v, dmul<T>(T(0.25), cb[o + kS * (2 * iz - 1)]));
      ub[x + kS * y] = v;
    }
  }
}


// The kernels of the per-operation path: each a grid-stride loop over its work, so the
// same bodies also run as the operations of one cooperative launch (srmg_seq.cu).
template <typename T>
__global__ void k_fill_ghost(T *__restrict__ u, LevelView lv, Signs sg, int mask) {
  d_fill_ghost<T>(u, lv, sg, mask);
}

template <typename T>
__global__ void k_gs_colour(T *__restrict__ u, const T *__restrict__ b, LevelView lv,
                            OpParams<T> p, WTab<T> wt, int parity) {
  d_gs_colour<T>(u, b, lv, p, wt, parity);
}

template <typename T>
__global__ void k_residual(T *__restrict__ r, const T *__restrict__ u, const T *__restrict__ b,
                           LevelView lv, OpParams<T> p, WTab<T> wt) {
  d_residual<T>(r, u, b, lv, p, wt);
}

template <typename T>
__global__ void k_postrestrict(T *__restrict__ bf, const T *__restrict__ u, const T *__restrict__ r,
                               LevelView lv, const int2 *__restrict__ coord_of, OpParams<T> p,
                               WTab<T> wt) {
  d_postrestrict<T>(bf, u, r, lv, coord_of, p, wt);
}

template <typename T>
__global__ void k_restrict(T *__restrict__ u, LevelView lv) {
  d_restrict<T>(u, lv);
}

template <typename T>
__global__ void k_interp_add(T *__restrict__ u, const T *__restrict__ u1, LevelView lv) {
  d_interp_add<T>(u, u1, lv);
}

template <typename T>
__global__ void k_copy_level(T *__restrict__ dst, const T *__restrict__ src, LevelView lv) {
  d_copy_level<T>(dst, src, lv);
}

template <typename T>
__global__ void k_diff_level(T *__restrict__ dst, const T *__restrict__ a1, const T *a2,
                             LevelView lv) {
  d_diff_level<T>(dst, a1, a2, lv);
}

template <typename T>
__global__ void k_gs4(T *__restrict__ u, const T *__restrict__ b, LevelView lv, OpParams<T> p, int p1, int p2) {
  d_gs4<T>(u, b, lv, p, p1, p2);
}

// The colour sweeps with their ghost pushes (PushView).
template <typename T>
__global__ void k_gs_colour_push(T *__restrict__ u, const T *__restrict__ b, LevelView lv, OpParams<T> p,
                                 WTab<T> wt, int parity, PushView pv, unsigned sg) {
  d_gs_colour_impl<T, true>(u, b, lv, p, wt, parity, pv, sg);
}

template <typename T>
__global__ void k_gs4_push(T *__restrict__ u, const T *__restrict__ b, LevelView lv, OpParams<T> p, int p1, int p2,
                           PushView pv, unsigned sg) {
  d_gs4_impl<T, true>(u, b, lv, p, p1, p2, pv, sg);
}

}  // namespace srmg
