// srmg_engine.cuh -- the persistent V-cycle engine: one cooperative launch runs a whole
// FAS V-cycle (src/multigrid.jl:60-106) with grid barriers between dependent phases.
//
// Phases (per level l, fine to coarse and back):
//   GS iteration     : one full red-black Gauss-Seidel iteration (red sweep, copy and
//                      mirror ghost fills, black sweep, fills; src/multigrid.jl:250-265)
//                      in ONE phase.  The iteration reads the level's current buffer and
//                      writes the other one (ping-pong per level).  Each CTA stages its
//                      block with ghosts in shared memory, updates the red cells, then
//                      recomputes the red update of every neighbour edge cell its black
//                      cells will read (their stencils touch only black cells and stored
//                      ghosts of the old buffer, so the values are bit-identical to the
//                      neighbour's own), updates the black cells, and writes the block
//                      plus the ghost values it feeds: the facing ghosts of its
//                      neighbours (fill_ghost_copy!), its mirror ghosts (fill_ghost_bnd!)
//                      and its frozen refinement ghosts.  No two CTAs write one address.
//   restrict         : per fine block: residual (src/multigrid.jl:309-323) and the
//                      restriction of r and u to the parent's subblock
//                      (src/restrict.jl:5-25, same summation order), with pushes of the
//                      restricted u into the coarse ghosts.  The FAS right-hand side
//                      (src/multigrid.jl:331-344) is formed at the start of the coarse
//                      level's first GS iteration, whose old buffer is exactly the
//                      post-restriction state; a neighbour's covered edge cells get the
//                      same FAS value recomputed from the same tile values.
//   prolongate       : per fine block: u += P(e) (src/interp.jl:24-63), pushes of the
//                      new edge values, and the block's refinement-boundary ghosts
//                      interpolated from the (final) coarser level.
// The coarse correction e = u - u1 of a level (diffto!, src/blockfield.jl:569-576) and
// its ghosts are produced in that level's last GS iteration.  Levels 1..local_top are
// processed by CTA 0 alone with CTA barriers.  Block tiles reach shared memory through
// bulk asynchronous copies (cp.async.bulk, no multicast) into a triple-buffered
// per-slot pipeline; every wait on an mbarrier or a barrier is bounded in time.
//
// One launch can carry several independent problems ("items"): the trees of a forest,
// each with its own operator (Poisson or Helmholtz k^2, scale s, boundary table).  The
// item of a block sits in bits 8.. of its child-mask word; operator parameters come from
// per-item tables.  Norms are per item and formed in a fixed order (per-block warp
// partials, then one CTA per item), so they do not depend on the grid size; an item
// whose norm reaches its tolerance is frozen (no phase touches its blocks again) while
// the others iterate, so every item ends exactly as if it had been solved alone.
#pragma once
#include "srmg_kernels.cuh"

namespace srmg {

constexpr int kMaxLev = 30;
constexpr int kTraceMax = 1024;

struct EngTree {
  const int4 *lvl_rec[kMaxLev];     // per level: 5 int4 per block ({blk, cr, cz, child_mask}, faces)
  const int4 *lvl_blocks[kMaxLev];  // per level: {blk, coord_r, coord_z, child_mask}
  const int4 *lvl_child[kMaxLev];   // per level: {fine, coarse, sb_r, sb_z}
  int nblk[kMaxLev];
  int nch[kMaxLev];
  const int4 *info;    // by block id: {coord_r, coord_z, child_mask, level}
  const int4 *faces;   // by block id * 4 + face: {type, src, sb_r | sb_z << 8 (refinement) or
                       //  the neighbour's child mask (neighbour), push_to}
  const int4 *kids;    // by block id: child block id per subblock, -1 if none
};

// FP64 side of one defect-correction step of the mixed-precision solve.  The launch
// first applies the previous correction (u64 += u), makes u64 a composite-grid function
// of its leaves (restriction chain, ghost refresh), forms the FP64 defect as the FP32
// right-hand side with its leaf norm, and runs the FP32 V-cycle only if the norm is
// still above its tolerance.
struct MixedArgs {
  double *u64;
  const double *b64;
  WTab<double> wt64;
  const double *it_par64;  // per item: kParStride FP64 operator values
  unsigned refbnd_levels;  // bit l: level l has refinement-boundary faces
  int apply_update;        // apply the correction left by a previous launch first
};

template <typename T>
struct EngArgs {
  T *u, *ualt, *b, *u1, *e;   // ualt: the second buffer of the per-level ping-pong
  EngTree tr;
  WTab<T> wt;
  int geom;
  int lmax;          // finest non-empty level taking part
  int ndown, ntop, nup;
  int local_top;     // levels 1..local_top run inside CTA 0
  int smooth_level;  // > 0: run smooth_n GS iterations on this level only (gauss_seidel_iter!)
  int smooth_n;
  int nitems;
  int nlev_tab;                // row length of it_lrange
  const T *it_par;             // per item: kParStride operator values (s_l, centre_l, nwc_l)
  const int *it_sgbits;        // per item: the 3x3 boundary table, entry k as (bc_k + 1) << 2k
  const double *const *it_P;   // per item: P = -s A_1^{-1} of its level 1 (row-major), or null
  const int2 *it_lrange;       // [item * nlev_tab + l - 1]: {first, count} in level l's block list
  int *frozen;                 // per item: nonzero once it has stopped iterating (zero at launch)
  unsigned *bar;     // barrier counter, zero at launch
  int *err;          // error word (0 = ok)
  long long timeout_ns;
  long long *trace;  // optional: CTA 0 stamps %globaltimer after every phase
  MixedArgs mx;            // mixed-precision outer step (mx.u64 != nullptr)
  // Device-side solve loop: with max_cycles > 0 the launch repeats V-cycles until every
  // item's leaf norm of the residual (FP64 mode) or of the FP64 defect (mixed mode) is
  // <= tol * (its leaf norm of b, or 1 if that is 0), or max_cycles V-cycles have run.
  int max_cycles;
  double tol;
  const int4 *chunks;      // norm chunks {level, first position, count, item}, by item
  int nchunk;
  const int2 *it_chunks;   // per item: {first chunk, chunks}
  double *bpart;           // one partial sum per chunk: r^2
  double *bpart_b;         // the same for b^2
  double *inorm;           // per item: {norm, |b|, initial norm, V-cycles run}
  double *out;             // out[0] V-cycles run by the launch
};

__device__ __forceinline__ int item_of(int4 bk) { return bk.w >> 8; }

template <typename T>
__device__ __forceinline__ bool is_frozen(const EngArgs<T> &A, int item) {
  return A.nitems > 1 && A.frozen[item] != 0;
}

// ------------------------------------------------------------------ barriers

__device__ __forceinline__ long long gtimer() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid-wide barrier on a monotonic counter.  A wait longer than timeout_ns sets the
// error word and returns false; every CTA then leaves the kernel at its next check.
__device__ __forceinline__ bool grid_barrier(unsigned *bar, int *err, unsigned &epoch,
                                             long long timeout_ns) {
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    epoch++;
    const unsigned target = epoch * gridDim.x;
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
    int ok = 1;
    const long long t0 = gtimer();
    while (true) {
      unsigned v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
      if (v >= target) break;
      if (*(volatile int *)err) { ok = 0; break; }
      if (gtimer() - t0 > timeout_ns) {
        atomicCAS(err, 0, 1);
        ok = 0;
        break;
      }
      __nanosleep(20);
    }
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

__device__ __forceinline__ void slot_sync(int slot) {
  asm volatile("bar.sync %0, 256;" ::"r"(slot + 1) : "memory");
}

// ------------------------------------------------------------------ helpers

template <typename T>
__device__ __forceinline__ T restrict4(const T *f, int fx, int fy) {
  const int o = fx + kS * fy;
  T v = dadd<T>(T(0), f[o]);
  v = dadd<T>(v, f[o + 1]);
  v = dadd<T>(v, f[o + kS]);
  v = dadd<T>(v, f[o + kS + 1]);
  return dmul<T>(v, T(0.25));
}

// Bulk (TMA, non-multicast) copies global -> shared with an mbarrier, per slot.
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up (and raises the error word) after timeout_ns.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err, long long timeout_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = gtimer();
  while (!mbar_try_wait(bar, parity)) {
    if (gtimer() - t0 > timeout_ns) {
      atomicCAS(err, 0, 2);
      return false;
    }
  }
  return true;
}

// Per-slot staging: triple-buffered block tiles and the records of up to 32 blocks.
constexpr int kBuf = 3;
template <typename T>
struct SlotSmem {
  T tile[kBuf][kSS];
  T tile2[kBuf][kSS];  // prolongation phase: the parent block's e tile
  T red[256];   // restriction phase: the residual of the block being restricted
  int4 recs[32][5];
  uint64_t bar[kBuf];
  int sel[32];  // list positions of the chunk's blocks that take part
  int cnt;
};

// Boundary sign k (-1, 0 or 1) of a packed boundary table.
template <typename F>
__device__ __forceinline__ F sign_at(unsigned sgb, int k) {
  return F((int)((sgb >> (2 * k)) & 3u) - 1);
}

// Write the value v of valid cell (x, y) of block X into the ghosts that copy or mirror
// it, in `field`: the facing ghost of each neighbour (fill_ghost_copy!) and the block's
// own mirror ghost (fill_ghost_bnd!, src/connectivity.jl:191-213).  fc: the block's four
// face records; sgb: the item's packed boundary table.
template <typename F>
__device__ __forceinline__ void push_f(unsigned sgb, F *field, int X, const int4 *fc, int x, int y, F v) {
  F *xb = field + (int64_t)X * kSS;
  if (x <= 3) {
    const int4 fi = fc[0];
    if (fi.w >= 0) field[(int64_t)fi.w * kSS + (x + kM) + kS * y] = v;
    else if (fi.x == FACE_BOUNDARY) xb[(2 * kG - 1 - x) + kS * y] = dmul<F>(sign_at<F>(sgb, 3), v);
  }
  if (x >= 16) {
    const int4 fi = fc[1];
    if (fi.w >= 0) field[(int64_t)fi.w * kSS + (x - kM) + kS * y] = v;
    else if (fi.x == FACE_BOUNDARY) xb[(2 * (kG + kM) - 1 - x) + kS * y] = dmul<F>(sign_at<F>(sgb, 5), v);
  }
  if (y <= 3) {
    const int4 fi = fc[2];
    if (fi.w >= 0) field[(int64_t)fi.w * kSS + x + kS * (y + kM)] = v;
    else if (fi.x == FACE_BOUNDARY) xb[x + kS * (2 * kG - 1 - y)] = dmul<F>(sign_at<F>(sgb, 1), v);
  }
  if (y >= 16) {
    const int4 fi = fc[3];
    if (fi.w >= 0) field[(int64_t)fi.w * kSS + x + kS * (y - kM)] = v;
    else if (fi.x == FACE_BOUNDARY) xb[x + kS * (2 * (kG + kM) - 1 - y)] = dmul<F>(sign_at<F>(sgb, 7), v);
  }
}

template <typename T>
__device__ __forceinline__ void push(const EngArgs<T> &A, int item, T *field, int X, const int4 *fc, int x, int y,
                                     T v) {
  push_f<T>((unsigned)A.it_sgbits[item], field, X, fc, x, y, v);
}

// Ghost cell `lane` (0..31) of face f: layer lane/16, position lane%16.
__device__ __forceinline__ void ghost_xy(int f, int lane, int &x, int &y) {
  const int g = lane >> 4, k = lane & 15;
  if (f == 0) { x = g; y = 2 + k; }
  else if (f == 1) { x = 18 + g; y = 2 + k; }
  else if (f == 2) { x = 2 + k; y = g; }
  else { x = 2 + k; y = 18 + g; }
}

// Refinement-boundary ghost q (0..127) of block X in `dst`, interpolated from `src` on
// the coarser level (fill_ghost_interp!, src/connectivity.jl:251-258).
template <typename T>
__device__ __forceinline__ void refbnd_ghost(T *dst, const T *src, int X, const int4 *fc, int q) {
  const int f = q >> 5, lane = q & 31;
  const int4 fi = fc[f];
  if (fi.x != FACE_REFBND) return;
  const int g = lane >> 4, k = lane & 15;
  int x, y;
  ghost_xy(f, lane, x, y);
  const T *cb = src + (int64_t)fi.y * kSS;
  const int sbr = fi.z & 0xff, sbz = fi.z >> 8;
  int jr, jz, ir, iz;
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
  T v = dmul<T>(T(0.5), cb[o]);
  v = dadd<T>(v, dmul<T>(T(0.25), cb[o + (2 * ir - 1)]));
  v = dadd<T>(v, dmul<T>(T(0.25), cb[o + kS * (2 * iz - 1)]));
  dst[(int64_t)X * kSS + x + kS * y] = v;
}

// ------------------------------------------------------------------ phases

// Issue the bulk copy of one block tile into buffer `buf` of a slot.
template <typename T>
__device__ __forceinline__ void issue_tile(SlotSmem<T> &S, int buf, const T *src, int X) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mbar_expect_tx(&S.bar[buf], (uint32_t)(kSS * sizeof(T)));
  bulk_g2s(S.tile[buf], src + (int64_t)X * kSS, (uint32_t)(kSS * sizeof(T)), &S.bar[buf]);
}

// Two tiles on one mbarrier: block X of src into tile[buf], block Y of src2 into tile2[buf].
template <typename T>
__device__ __forceinline__ void issue_pair(SlotSmem<T> &S, int buf, const T *src, int X, const T *src2, int Y) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mbar_expect_tx(&S.bar[buf], (uint32_t)(2 * kSS * sizeof(T)));
  bulk_g2s(S.tile[buf], src + (int64_t)X * kSS, (uint32_t)(kSS * sizeof(T)), &S.bar[buf]);
  bulk_g2s(S.tile2[buf], src2 + (int64_t)Y * kSS, (uint32_t)(kSS * sizeof(T)), &S.bar[buf]);
}

// Halo cell of thread t < 64: face t/16, position t%16 along the face, in the
// block's frame; (nx, ny) is the same cell in the neighbour's frame.
struct HaloCell {
  int f, jj, hx, hy, nx, ny, nsub;
  bool red;
  int cx, cy;   // the one stencil neighbour that is a ghost corner of this block, or cx < 0
  int cnx, cny; // that corner in the neighbour's frame
};

__device__ __forceinline__ HaloCell halo_cell(int t) {
  HaloCell h;
  h.f = t >> 4;
  h.jj = t & 15;
  if (h.f == 0) { h.hx = 1; h.hy = 2 + h.jj; }
  else if (h.f == 1) { h.hx = 18; h.hy = 2 + h.jj; }
  else if (h.f == 2) { h.hx = 2 + h.jj; h.hy = 1; }
  else { h.hx = 2 + h.jj; h.hy = 18; }
  const int dx = h.f == 0 ? kM : h.f == 1 ? -kM : 0, dy = h.f == 2 ? kM : h.f == 3 ? -kM : 0;
  h.nx = h.hx + dx;
  h.ny = h.hy + dy;
  h.nsub = ((h.nx - 2) >> 3) + 2 * ((h.ny - 2) >> 3);
  h.red = ((h.hx + h.hy) & 1) == 1;
  h.cx = -1;
  h.cy = -1;
  if (h.jj == 0 || h.jj == 15) {
    const int d = h.jj == 0 ? -1 : 1;
    if (h.f <= 1) { h.cx = h.hx; h.cy = h.hy + d; }
    else { h.cx = h.hx + d; h.cy = h.hy; }
  }
  h.cnx = h.cx + dx;
  h.cny = h.cy + dy;
  return h;
}

// One fused red-black GS iteration over level l: src -> dst.  256 threads per block,
// thread t owns valid cell (2 + t%16, 2 + t/16).  Blocks stream through a
// double-buffered shared-memory pipeline fed by bulk copies, and each block's scattered
// inputs (its b, the neighbours' edge b and ghost corners) are loaded into registers
// while the previous block computes.  With `fas`, the FAS right-hand side of the
// covered cells (src/multigrid.jl:112-119) is formed first from the post-restriction
// tile and the restricted residual held in e.
template <typename T>
__device__ bool ph_gsi(const EngArgs<T> &A, int l, const T *src, T *dst, const T *esrc, bool copy_u1,
                       bool make_e, bool fas, int first, int step, int t, int slot, SlotSmem<T> &S,
                       unsigned &pk) {
  const int n = A.tr.nblk[l - 1];
  const int4 *recs = A.tr.lvl_rec[l - 1];
  const int nmine = (first < n) ? (n - 1 - first) / step + 1 : 0;
  if (nmine == 0) return true;
  const int x = 2 + (t & 15), y = 2 + (t >> 4);
  const int o = x + kS * y;
  const bool red = ((x + y) & 1) == 1;  // colour 0 of RedBlack{0}: updated first
  const int mysub = ((x - 2) >> 3) + 2 * ((y - 2) >> 3);
  const HaloCell h = halo_cell(t < 64 ? t : 0);
  // registers prefetched one block ahead
  T b_nx = T(0), e_nx = T(0), hv_nx = T(0), hc_nx = T(0);
  auto prefetch = [&](int j) {
    const int4 bk = S.recs[j][0];
    const int X = bk.x;
    b_nx = A.b[(int64_t)X * kSS + o];
    if (fas && ((bk.w >> mysub) & 1)) e_nx = A.e[(int64_t)X * kSS + o];
    if (t < 64 && h.red) {
      const int4 fi = S.recs[j][1 + h.f];
      if (fi.x == FACE_NEIGHBOR) {
        const int64_t nb = (int64_t)fi.y * kSS;
        hv_nx = (fas && ((fi.z >> h.nsub) & 1)) ? A.e[nb + h.nx + kS * h.ny] : A.b[nb + h.nx + kS * h.ny];
        if (h.cx >= 0) hc_nx = src[nb + h.cnx + kS * h.cny];
      }
    }
  };
  // one item: the operator values stay in registers for the whole level
  T s = A.it_par[l], centre = A.it_par[32 + l], nwc = A.it_par[64 + l];
  for (int c0 = 0; c0 < nmine; c0 += 32) {
    int cn;
    if (A.nitems == 1) {
      cn = min(32, nmine - c0);
      if (t < 5 * cn) {
        const int q = t / 5, k = t - 5 * q;
        S.recs[q][k] = recs[5 * (first + (c0 + q) * step) + k];
      }
      slot_sync(slot);
    } else {
    // the chunk's next 32 list positions, without the blocks of frozen items
    if (t < 32) {
      const int idx = c0 + t;
      int gi = 0;
      bool take = false;
      if (idx < nmine) {
        gi = first + idx * step;
        take = A.nitems == 1 || !A.frozen[item_of(recs[5 * gi])];
      }
      const unsigned m = __ballot_sync(0xffffffffu, take);
      if (take) S.sel[__popc(m & ((1u << t) - 1u))] = gi;
      if (t == 0) S.cnt = __popc(m);
    }
    slot_sync(slot);
    cn = S.cnt;
    if (t < 5 * cn) {
      const int q = t / 5, k = t - 5 * q;
      S.recs[q][k] = recs[5 * S.sel[q] + k];
    }
    slot_sync(slot);
    if (cn == 0) continue;
    }
    if (t == 0) {
      issue_tile<T>(S, pk % kBuf, src, S.recs[0][0].x);
      if (cn > 1) issue_tile<T>(S, (pk + 1) % kBuf, src, S.recs[1][0].x);
    }
    prefetch(0);
    for (int j = 0; j < cn; ++j) {
      const unsigned kb = pk + j;
      const int buf = kb % kBuf;
      const int4 bk = S.recs[j][0];
      const int4 *fc = &S.recs[j][1];
      const int X = bk.x;
      // two blocks ahead: the buffer of block j - 1, free since the end of its item
      if (t == 0 && j + 2 < cn) issue_tile<T>(S, (kb + 2) % kBuf, src, S.recs[j + 2][0].x);
      T bx = b_nx;
      const T ex = e_nx, hv = hv_nx, hc = hc_nx;
      if (j + 1 < cn) prefetch(j + 1);
      if (!mbar_wait(&S.bar[buf], (kb / kBuf) & 1, A.err, A.timeout_ns)) {
        // leave no copy in flight: wait (bounded) for those issued for the next items
        for (int q = 1; q <= 2 && j + q < cn; ++q)
          mbar_wait(&S.bar[(kb + q) % kBuf], ((kb + q) / kBuf) & 1, A.err, A.timeout_ns);
        return false;
      }
      T *tile = S.tile[buf];
      const int item = item_of(bk);
      if (A.nitems > 1) {
        const T *par = A.it_par + item * kParStride;
        s = par[l];
        centre = par[32 + l];
        nwc = par[64 + l];
      }
      const W5<T> w = weights<T>(A.wt, A.geom, bk.y, bk.z, x, y);
      if (copy_u1) A.u1[(int64_t)X * kSS + o] = tile[o];
      if (fas) {
        if ((bk.w >> mysub) & 1) {
          const T Lu = apply5<T>(tile, x, y, w, centre);
          bx = -(ex + Lu / s);
          A.b[(int64_t)X * kSS + o] = bx;
        }
        slot_sync(slot);
      }
      if (red) {
        const T Lu = apply5<T>(tile, x, y, w, centre);
        tile[o] = fma(nwc, fma(s, bx, Lu), tile[o]);
      }
      if (t < 64 && h.red && fc[h.f].x == FACE_NEIGHBOR) {
        // red update of the neighbour's edge cell that sits in this block's ghost layer
        const int4 fi = fc[h.f];
        auto at = [&](int a, int c) -> T { return (a == h.cx && c == h.cy) ? hc : tile[a + kS * c]; };
        const W5<T> wh = weights<T>(A.wt, A.geom, bk.y, bk.z, h.hx, h.hy);
        T v = wh.zm * at(h.hx, h.hy - 1);
        v = v + wh.rm * at(h.hx - 1, h.hy);
        v = v + centre * tile[h.hx + kS * h.hy];
        v = v + wh.rp * at(h.hx + 1, h.hy);
        v = v + wh.zp * at(h.hx, h.hy + 1);
        const T bn = (fas && ((fi.z >> h.nsub) & 1)) ? -(hv + v / s) : hv;
        tile[h.hx + kS * h.hy] = fma(nwc, fma(s, bn, v), tile[h.hx + kS * h.hy]);
      }
      slot_sync(slot);
      if (!red) {
        const T Lu = apply5<T>(tile, x, y, w, centre);
        tile[o] = fma(nwc, fma(s, bx, Lu), tile[o]);
      }
      slot_sync(slot);
      const T nu = tile[o];
      dst[(int64_t)X * kSS + o] = nu;
      push<T>(A, item, dst, X, fc, x, y, nu);
      if (t < 128) {
        const int f = t >> 5, lane = t & 31;
        if (fc[f].x == FACE_REFBND) {
          int gx, gy;
          ghost_xy(f, lane, gx, gy);
          dst[(int64_t)X * kSS + gx + kS * gy] = tile[gx + kS * gy];  // frozen during smoothing
        }
      }
      if (make_e) {
        const T ev = nu - A.u1[(int64_t)X * kSS + o];
        A.e[(int64_t)X * kSS + o] = ev;
        push<T>(A, item, A.e, X, fc, x, y, ev);
        if (t < 128) refbnd_ghost<T>(A.e, esrc, X, fc, t);
      }
      slot_sync(slot);  // the buffer is refilled three items later
    }
    pk += cn;
  }
  return true;
}

// Residual and restriction of r and u, one fine block (Child edge of level l) per
// 256-thread slot: the restricted u goes to the coarse block (and into the coarse
// ghosts that copy it), the restricted r to e, where the coarse level's first GS
// iteration reads it to form the FAS right-hand side.  uf: level l, uc: level l-1.
// The fine blocks' tiles stream through the slot's triple-buffered bulk-copy pipeline
// (as in the GS phase) and each block's b is loaded one block ahead, so the residual
// reads shared memory.  Children of frozen items are skipped.
template <typename T>
__device__ bool ph_restrict(const EngArgs<T> &A, int l, const T *uf, T *uc, int first, int step, int t, int slot,
                            SlotSmem<T> &S, unsigned &pk) {
  const int n = A.tr.nch[l - 1];
  const int4 *ch = A.tr.lvl_child[l - 1];
  const int nmine = (first < n) ? (n - 1 - first) / step + 1 : 0;
  if (nmine == 0) return true;
  const int x = 2 + (t & 15), y = 2 + (t >> 4);
  const int o = x + kS * y;
  T *sr = S.red;
  T b_nx = T(0);
  auto prefetch = [&](int j) { b_nx = A.b[(int64_t)S.recs[j][0].x * kSS + o]; };
  for (int c0 = 0; c0 < nmine; c0 += 32) {
    // the chunk's next 32 child edges, without those of frozen items:
    // recs[q][0] = {fine, coarse, sb_r, sb_z}, recs[q][1] = info of the fine block
    if (t < 32) {
      const int idx = c0 + t;
      int gi = 0;
      bool take = false;
      if (idx < nmine) {
        gi = first + idx * step;
        take = A.nitems == 1 || !A.frozen[A.tr.info[ch[gi].x].z >> 8];
      }
      const unsigned m = __ballot_sync(0xffffffffu, take);
      if (take) S.sel[__popc(m & ((1u << t) - 1u))] = gi;
      if (t == 0) S.cnt = __popc(m);
    }
    slot_sync(slot);
    const int cn = S.cnt;
    if (t < 2 * cn) {
      const int q = t >> 1;
      const int4 e = ch[S.sel[q]];
      S.recs[q][t & 1] = (t & 1) ? A.tr.info[e.x] : e;
    }
    slot_sync(slot);
    if (cn == 0) continue;
    if (t == 0) {
      issue_tile<T>(S, pk % kBuf, uf, S.recs[0][0].x);
      if (cn > 1) issue_tile<T>(S, (pk + 1) % kBuf, uf, S.recs[1][0].x);
    }
    prefetch(0);
    for (int j = 0; j < cn; ++j) {
      const unsigned kb = pk + j;
      const int buf = kb % kBuf;
      const int4 e = S.recs[j][0], fi = S.recs[j][1];
      const int C = e.y;
      if (t == 0 && j + 2 < cn) issue_tile<T>(S, (kb + 2) % kBuf, uf, S.recs[j + 2][0].x);
      const T bx = b_nx;
      if (j + 1 < cn) prefetch(j + 1);
      if (!mbar_wait(&S.bar[buf], (kb / kBuf) & 1, A.err, A.timeout_ns)) {
        for (int q = 1; q <= 2 && j + q < cn; ++q)
          mbar_wait(&S.bar[(kb + q) % kBuf], ((kb + q) / kBuf) & 1, A.err, A.timeout_ns);
        return false;
      }
      const T *tile = S.tile[buf];
      const int item = fi.z >> 8;
      const T *par = A.it_par + item * kParStride;
      const T s = par[l], centre = par[32 + l];
      const W5<T> w = weights<T>(A.wt, A.geom, fi.x, fi.y, x, y);
      const T Lu = apply5<T>(tile, x, y, w, centre);
      sr[t] = -(bx + Lu / s);
      slot_sync(slot);
      if (t < 64) {
        const int kx = t & 7, ky = t >> 3;
        const int cx = 2 + 8 * (e.z - 1) + kx, cy = 2 + 8 * (e.w - 1) + ky;
        // 2x2 sums in the reference's order: (i, j), (i+1, j), (i, j+1), (i+1, j+1)
        const T cu = restrict4<T>(tile, 2 + 2 * kx, 2 + 2 * ky);
        const int i00 = 2 * kx + 16 * 2 * ky;
        T cr = dadd<T>(T(0), sr[i00]);
        cr = dadd<T>(cr, sr[i00 + 1]);
        cr = dadd<T>(cr, sr[i00 + 16]);
        cr = dadd<T>(cr, sr[i00 + 17]);
        cr = dmul<T>(cr, T(0.25));
        uc[(int64_t)C * kSS + cx + kS * cy] = cu;
        push<T>(A, item, uc, C, A.tr.faces + 4 * C, cx, cy, cu);
        A.e[(int64_t)C * kSS + cx + kS * cy] = cr;
      }
      slot_sync(slot);  // sr and the tile buffer are reused
    }
    pk += cn;
  }
  return true;
}

// u_fine += P(e_coarse) on every valid cell (in place in uf), pushes of the new edge
// values, and the fine block's refinement-boundary ghosts from uc (final coarse level).
// Per child edge the fine block's u tile and its parent's e tile arrive together by
// two bulk copies on one mbarrier of the slot's triple-buffered pipeline, and the
// child's face records are staged in shared memory.  Children of frozen items are
// skipped.
template <typename T>
__device__ bool ph_prolong(const EngArgs<T> &A, int l, T *uf, const T *uc, int first, int step, int t, int slot,
                           SlotSmem<T> &S, unsigned &pk) {
  const int n = A.tr.nch[l - 1];
  const int4 *ch = A.tr.lvl_child[l - 1];
  const int nmine = (first < n) ? (n - 1 - first) / step + 1 : 0;
  if (nmine == 0) return true;
  const int dx = t & 15, dy = t >> 4;
  const int x = 2 + dx, y = 2 + dy;
  const int ir = dx & 1, iz = dy & 1;
  for (int c0 = 0; c0 < nmine; c0 += 32) {
    // the chunk's next 32 child edges, without those of frozen items:
    // recs[q][0] = {fine, coarse, sb_r, sb_z}, recs[q][1..4] = the fine block's faces
    if (t < 32) {
      const int idx = c0 + t;
      int gi = 0;
      bool take = false;
      if (idx < nmine) {
        gi = first + idx * step;
        take = A.nitems == 1 || !A.frozen[A.tr.info[ch[gi].x].z >> 8];
      }
      const unsigned m = __ballot_sync(0xffffffffu, take);
      if (take) S.sel[__popc(m & ((1u << t) - 1u))] = gi;
      if (t == 0) S.cnt = __popc(m);
    }
    slot_sync(slot);
    const int cn = S.cnt;
    if (t < 5 * cn) {
      const int q = t / 5, k = t - 5 * q;
      const int4 e = ch[S.sel[q]];
      S.recs[q][k] = k == 0 ? e : A.tr.faces[4 * e.x + k - 1];
    }
    slot_sync(slot);
    if (cn == 0) continue;
    if (t == 0) {
      issue_pair<T>(S, pk % kBuf, uf, S.recs[0][0].x, A.e, S.recs[0][0].y);
      if (cn > 1) issue_pair<T>(S, (pk + 1) % kBuf, uf, S.recs[1][0].x, A.e, S.recs[1][0].y);
    }
    for (int j = 0; j < cn; ++j) {
      const unsigned kb = pk + j;
      const int buf = kb % kBuf;
      const int4 e = S.recs[j][0];
      const int4 *fc = &S.recs[j][1];
      const int F = e.x;
      if (t == 0 && j + 2 < cn)
        issue_pair<T>(S, (kb + 2) % kBuf, uf, S.recs[j + 2][0].x, A.e, S.recs[j + 2][0].y);
      if (!mbar_wait(&S.bar[buf], (kb / kBuf) & 1, A.err, A.timeout_ns)) {
        for (int q = 1; q <= 2 && j + q < cn; ++q)
          mbar_wait(&S.bar[(kb + q) % kBuf], ((kb + q) / kBuf) & 1, A.err, A.timeout_ns);
        return false;
      }
      const T *ut = S.tile[buf], *cb = S.tile2[buf];
      const int jr = 2 + 8 * (e.z - 1) + (dx >> 1), jz = 2 + 8 * (e.w - 1) + (dy >> 1);
      const int oc = jr + kS * jz;
      T v = dmul<T>(T(0.5), cb[oc]);
      v = dadd<T>(v, dmul<T>(T(0.25), cb[oc + (2 * ir - 1)]));
      v = dadd<T>(v, dmul<T>(T(0.25), cb[oc + kS * (2 * iz - 1)]));
      const T nu = dadd<T>(v, ut[x + kS * y]);
      uf[(int64_t)F * kSS + x + kS * y] = nu;
      const int item = A.tr.info[F].z >> 8;
      push<T>(A, item, uf, F, fc, x, y, nu);
      if (t < 128) refbnd_ghost<T>(uf, uc, F, fc, t);
      slot_sync(slot);  // the buffers are refilled three items later
    }
    pk += cn;
  }
  return true;
}

// ---- mixed-precision outer step (FP64) ---------------------------------------------

// u64 += u (FP32 correction) on every valid cell of every level, with pushes of the new
// values into the copy and mirror ghosts of u64.
template <typename T>
__device__ void ph_update64(const EngArgs<T> &A, int t, int gslot, int gstep) {
  const int x = 2 + (t & 15), y = 2 + (t >> 4), o = x + kS * y;
  int base = 0;
  for (int l = 1; l <= A.lmax; ++l) {
    const int n = A.tr.nblk[l - 1];
    const int4 *blocks = A.tr.lvl_blocks[l - 1];
    // items are numbered across levels so that the work spreads over every slot
    for (int i = (gslot - base % gstep + gstep) % gstep; i < n; i += gstep) {
      const int4 bk = blocks[i];
      if (is_frozen(A, item_of(bk))) continue;
      const int X = bk.x;
      double *d = A.mx.u64 + (int64_t)X * kSS + o;
      const double nv = *d + (double)A.u[(int64_t)X * kSS + o];
      *d = nv;
      push_f<double>((unsigned)A.it_sgbits[item_of(bk)], A.mx.u64, X, A.tr.faces + 4 * X, x, y, nv);
    }
    base += n;
  }
}

// Restriction of u64 from level l onto the covered subblocks of level l - 1, with pushes.
template <typename T>
__device__ void ph_restrict64(const EngArgs<T> &A, int l, int t, int gslot, int gstep) {
  const int n = A.tr.nch[l - 1];
  const int4 *ch = A.tr.lvl_child[l - 1];
  if (t >= 64) return;
  const int kx = t & 7, ky = t >> 3;
  for (int i = gslot; i < n; i += gstep) {
    const int4 e = ch[i];
    const int item = A.tr.info[e.y].z >> 8;
    if (is_frozen(A, item)) continue;
    const double v = restrict4<double>(A.mx.u64 + (int64_t)e.x * kSS, 2 + 2 * kx, 2 + 2 * ky);
    const int cx = 2 + 8 * (e.z - 1) + kx, cy = 2 + 8 * (e.w - 1) + ky;
    A.mx.u64[(int64_t)e.y * kSS + cx + kS * cy] = v;
    push_f<double>((unsigned)A.it_sgbits[item], A.mx.u64, e.y, A.tr.faces + 4 * e.y, cx, cy, v);
  }
}

// Refinement-boundary ghosts of u64 on level l from level l - 1.
template <typename T>
__device__ void ph_refbnd64(const EngArgs<T> &A, int l, int t, int gslot, int gstep) {
  const int n = A.tr.nblk[l - 1];
  const int4 *blocks = A.tr.lvl_blocks[l - 1];
  if (t >= 128) return;
  for (int i = gslot; i < n; i += gstep) {
    const int4 bk = blocks[i];
    if (is_frozen(A, item_of(bk))) continue;
    refbnd_ghost<double>(A.mx.u64, A.mx.u64, bk.x, A.tr.faces + 4 * bk.x, t);
  }
}

// Leaf sums of squares per norm chunk (up to kNormChunk consecutive blocks of one item
// and level) at bpart[c]: per thread over the chunk's blocks in order, the warp sums,
// then the 8 warp sums in order.  A leaf cell of level l is weighted by 4^-(l-1); cells
// under a child are skipped (resnorm!, src/multigrid.jl:391-417).
//   defect = false: r = -(b + L u / s_l) of the current iterate u;
//   defect = true : the FP64 defect r = -(b64 + L u64 / s_l) of the mixed solve, also
//                   written as the FP32 right-hand side -r, with the FP32 correction
//                   zeroed (ghosts included).
// with_b adds the same sums for b (b64 in mixed mode) in bpart_b.
template <typename T>
__device__ void ph_blocknorm(const EngArgs<T> &A, bool defect, bool with_b, int t, int slot, int gslot, int gstep,
                             double *red) {
  const int x = 2 + (t & 15), y = 2 + (t >> 4), o = x + kS * y;
  const int mysub = ((x - 2) >> 3) + 2 * ((y - 2) >> 3);
  const int lane = t & 31, w8 = t >> 5;
  int nb = 0;
  for (int c = gslot; c < A.nchunk; c += gstep) {
    const int4 ck = A.chunks[c];  // {level, first, count, item}
    const int item = ck.w;
    if (is_frozen(A, item)) continue;
    const int l = ck.x;
    const int4 *blocks = A.tr.lvl_blocks[l - 1] + ck.y;
    const double wl = 1.0 / (double)((int64_t)1 << (2 * (l - 1)));
    double v = 0.0, vb = 0.0;
    for (int j = 0; j < ck.z; ++j) {
      const int4 bk = blocks[j];
      const int X = bk.x;
      const bool leaf = !((bk.w >> mysub) & 1);
      double r, bv;
      if (!defect) {
        const T *par = A.it_par + item * kParStride;
        const W5<T> w = weights<T>(A.wt, A.geom, bk.y, bk.z, x, y);
        const T Lu = apply5<T>(A.u + (int64_t)X * kSS, x, y, w, par[32 + l]);
        const T bb = A.b[(int64_t)X * kSS + o];
        r = (double)(-(bb + Lu / par[l]));
        bv = (double)bb;
      } else {
        const double *par = A.mx.it_par64 + item * kParStride;
        const W5<double> w = weights<double>(A.mx.wt64, A.geom, bk.y, bk.z, x, y);
        const double Lu = apply5<double>(A.mx.u64 + (int64_t)X * kSS, x, y, w, par[32 + l]);
        bv = A.mx.b64[(int64_t)X * kSS + o];
        r = -(bv + Lu / par[l]);
        A.b[(int64_t)X * kSS + o] = (T)(-r);
        T *eb = A.u + (int64_t)X * kSS;
        eb[t] = T(0);
        if (t < kSS - 256) eb[t + 256] = T(0);
      }
      if (leaf) {
        v = fma(r, r, v);
        vb = fma(bv, bv, vb);
      }
    }
    for (int off = 16; off > 0; off >>= 1) {
      v += __shfl_xor_sync(0xffffffffu, v, off);
      vb += __shfl_xor_sync(0xffffffffu, vb, off);
    }
    // double-buffered per chunk: a buffer is rewritten two chunks later, after the next
    // slot barrier, which thread 0 reaches only once it has read this one
    double *rb = red + 16 * (nb & 1);
    if (lane == 0) {
      rb[w8] = v;
      rb[8 + w8] = vb;
    }
    slot_sync(slot);
    if (t == 0) {
      double sv = 0.0, sb = 0.0;
      for (int q = 0; q < 8; ++q) {
        sv += rb[q];
        sb += rb[8 + q];
      }
      A.bpart[c] = sv * wl;
      if (with_b) A.bpart_b[c] = sb * wl;
    }
    ++nb;
  }
}

// Per-item norms from the chunk partials, one CTA (1024 threads) per item, in a fixed
// order: thread-strided sums over the item's chunk partials, the warp sums, then the
// 32 warp sums in order.  Writes inorm[4 k + 0] (and with `first` the |b| and
// initial-norm entries), the item's V-cycle count, and freezes the item once its norm
// is <= tol * |b| (|b| = 0 counts as 1) or not finite.  Items frozen before are skipped.
template <typename T>
__device__ void ph_itemnorm(const EngArgs<T> &A, bool first, int cycles, double *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = blockIdx.x; k < A.nitems; k += gridDim.x) {
    if (A.frozen[k]) continue;
    double v = 0.0, vb = 0.0;
    const int2 rg = A.it_chunks[k];
    for (int j = threadIdx.x; j < rg.y; j += blockDim.x) {
      v += A.bpart[rg.x + j];
      if (first) vb += A.bpart_b[rg.x + j];
    }
    for (int off = 16; off > 0; off >>= 1) {
      v += __shfl_xor_sync(0xffffffffu, v, off);
      vb += __shfl_xor_sync(0xffffffffu, vb, off);
    }
    if (lane == 0) {
      red[warp] = v;
      red[32 + warp] = vb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double sv = 0.0, sb = 0.0;
      for (int q = 0; q < 32; ++q) {
        sv += red[q];
        sb += red[32 + q];
      }
      const double nrm = sqrt(sv);
      double *io = A.inorm + 4 * k;
      if (first) {
        io[1] = sqrt(sb);
        io[2] = nrm;
      }
      io[0] = nrm;
      io[3] = (double)cycles;
      const double bn = io[1] > 0.0 ? io[1] : 1.0;
      if (!(nrm > A.tol * bn) || !isfinite(nrm)) A.frozen[k] = 1;
    }
    __syncthreads();
  }
}

// Coarsest level solved directly (mixed-precision solve), one item per CTA: FAS
// right-hand side of the covered cells, then u_1 = P b_1 with the item's
// P = -s A_1^{-1} applied in FP64 (one warp per row), ghosts pushed, and the
// correction e = u_1 - u1 of the level.  An item's level 1 has <= 4 blocks.
template <typename T>
__device__ void ph_direct_top(const EngArgs<T> &A, T *u, bool make_e, int first, int step, int t, int slot,
                              double *sol) {
  const int x = 2 + (t & 15), y = 2 + (t >> 4);
  const int o = x + kS * y;
  const int mysub = ((x - 2) >> 3) + 2 * ((y - 2) >> 3);
  for (int k = first; k < A.nitems; k += step) {
    if (is_frozen(A, k)) continue;
    const int2 rg = A.it_lrange[k * A.nlev_tab];
    const int n1 = rg.y;
    const int4 *blocks = A.tr.lvl_blocks[0] + rg.x;
    const T *par = A.it_par + k * kParStride;
    const T s = par[1], centre = par[32 + 1];
    if (slot < n1) {
      const int4 bk = blocks[slot];
      const int X = bk.x;
      const T uo = u[(int64_t)X * kSS + o];
      A.u1[(int64_t)X * kSS + o] = uo;
      if ((bk.w >> mysub) & 1) {
        const W5<T> w = weights<T>(A.wt, A.geom, bk.y, bk.z, x, y);
        const T Lu = apply5<T>(u + (int64_t)X * kSS, x, y, w, centre);
        A.b[(int64_t)X * kSS + o] = -(A.e[(int64_t)X * kSS + o] + Lu / s);
      }
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int n = 256 * n1;
    const double *P = A.it_P[k];
    for (int q = warp; q < n; q += nw) {
      const double *pr = P + (int64_t)q * n;
      double acc = 0.0;
      for (int j = lane; j < n; j += 32) {
        const int c = j & 255;
        const int X = blocks[j >> 8].x;
        acc = fma(pr[j], (double)A.b[(int64_t)X * kSS + (2 + (c & 15)) + kS * (2 + (c >> 4))], acc);
      }
      for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
      if (lane == 0) sol[q] = acc;
    }
    __syncthreads();
    if (slot < n1) {
      const int4 bk = blocks[slot];
      const int X = bk.x;
      const int4 *fc = A.tr.faces + 4 * X;
      const T nu = (T)sol[slot * 256 + (t & 255)];
      u[(int64_t)X * kSS + o] = nu;
      push<T>(A, k, u, X, fc, x, y, nu);
      if (make_e) {
        const T ev = nu - A.u1[(int64_t)X * kSS + o];
        A.e[(int64_t)X * kSS + o] = ev;
        push<T>(A, k, A.e, X, fc, x, y, ev);
      }
    }
    __syncthreads();
  }
}

// Copy level l's blocks (valid cells and face ghosts) from src to dst.
template <typename T>
__device__ void ph_copy_back(const EngArgs<T> &A, int l, const T *src, T *dst, int first, int step, int t) {
  const int n = A.tr.nblk[l - 1];
  const int4 *blocks = A.tr.lvl_blocks[l - 1];
  for (int i = first; i < n; i += step) {
    const int4 bk = blocks[i];
    if (is_frozen(A, item_of(bk))) continue;
    const int X = bk.x;
    for (int k = t; k < kSS; k += 256) {
      const int x = k % kS, y = k / kS;
      const bool corner = (x < 2 || x > 17) && (y < 2 || y > 17);
      if (!corner) dst[(int64_t)X * kSS + k] = src[(int64_t)X * kSS + k];
    }
  }
}

// ------------------------------------------------------------------ the kernel

template <typename T>
constexpr size_t engine_smem_bytes() {
  return 4 * sizeof(SlotSmem<T>);
}

template <typename T>
__global__ void __launch_bounds__(1024, 1) k_engine_vcycle(const __grid_constant__ EngArgs<T> A) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SlotSmem<T> *smem = reinterpret_cast<SlotSmem<T> *>(smem_raw);
  const int nslots = blockDim.x >> 8;
  const int slot = threadIdx.x >> 8, t = threadIdx.x & 255;
  const bool cta0 = blockIdx.x == 0;
  SlotSmem<T> &S = smem[slot];
  if (t == 0) {
    for (int q = 0; q < kBuf; ++q) mbar_init(&S.bar[q]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  unsigned pk = 0;  // items streamed through this slot's buffers so far
  unsigned epoch = 0;
  int ntrace = 0;
  const int L = A.lmax, K = A.local_top;
  unsigned cur = 0;  // bit l: level l currently lives in ualt
  auto fld = [&](int l) -> T * { return ((cur >> l) & 1) ? A.ualt : A.u; };
  auto oth = [&](int l) -> T * { return ((cur >> l) & 1) ? A.u : A.ualt; };
  __shared__ double s_direct[1024];  // coarsest-level direct solution (CTA 0)

  auto first_of = [&](bool loc) { return loc ? slot : blockIdx.x * nslots + slot; };
  auto step_of = [&](bool loc) { return loc ? nslots : gridDim.x * nslots; };
  auto stamp = [&]() {
    if (A.trace && cta0 && threadIdx.x == 0 && ntrace < kTraceMax) A.trace[ntrace++] = gtimer();
  };
  // Barrier after a phase: CTA-local when this and the next phase are both local.
  auto sync = [&](bool ok_in, bool cur_loc, bool next_loc) -> bool {
    bool ok = ok_in;
    if (cur_loc && next_loc) {
      if (cta0) __syncthreads();
      if (!ok_in) atomicCAS(A.err, 0, 3);
    } else {
      if (!ok_in) atomicCAS(A.err, 0, 3);
      ok = grid_barrier(A.bar, A.err, epoch, A.timeout_ns) && ok_in;
    }
    stamp();
    if (cta0 && cur_loc && next_loc) ok = ok && *(volatile int *)A.err == 0;
    return ok;
  };
  auto runs = [&](bool loc) { return !loc || cta0; };
  stamp();

  if (A.smooth_level > 0) {
    // gauss_seidel_iter! (src/multigrid.jl:250-265) on one level
    const int l = A.smooth_level;
    for (int it = 0; it < A.smooth_n; ++it) {
      const bool ok = ph_gsi<T>(A, l, fld(l), oth(l), nullptr, false, false, false, first_of(false),
                                step_of(false), t, slot, S, pk);
      cur ^= 1u << l;
      if (!sync(ok, false, false)) return;
    }
    if ((cur >> l) & 1) {
      ph_copy_back<T>(A, l, A.ualt, A.u, first_of(false), step_of(false), t);
      grid_barrier(A.bar, A.err, epoch, A.timeout_ns);
    }
    if (A.trace && cta0 && threadIdx.x == 0 && ntrace < kTraceMax) A.trace[ntrace] = 0;
    return;
  }

  const int gslot = blockIdx.x * nslots + slot, gstep = gridDim.x * nslots;
  // Norm step: per-block partials, barrier, per-item sums and freezing, barrier.
  auto norm_step = [&](bool defect, bool first, int ncyc) -> bool {
    ph_blocknorm<T>(A, defect, first, t, slot, gslot, gstep, reinterpret_cast<double *>(&S.tile[0][0]));
    if (!sync(true, false, false)) return false;
    ph_itemnorm<T>(A, first, ncyc, s_direct);
    return sync(true, false, false);
  };
  __shared__ int s_live;
  auto any_live = [&]() -> bool {
    if (threadIdx.x == 0) {
      int live = 0;
      for (int k = 0; k < A.nitems && !live; ++k) live = *((volatile int *)A.frozen + k) == 0;
      s_live = live;
    }
    __syncthreads();
    return s_live != 0;
  };

  // One FAS V-cycle (src/multigrid.jl:60-106) on the current fields.
  auto vcycle_body = [&]() -> bool {
    cur = 0;
    // descending leg
    for (int l = L; l >= 2; --l) {
      const bool loc = l <= K;
      for (int it = 0; it < A.ndown; ++it) {
        bool ok = true;
        if (runs(loc))
          ok = ph_gsi<T>(A, l, fld(l), oth(l), nullptr, it == 0 && l < L, false, it == 0 && l < L, first_of(loc),
                         step_of(loc), t, slot, S, pk);
        cur ^= 1u << l;
        if (!sync(ok, loc, loc)) return false;
      }
      bool okr = true;
      if (runs(loc)) okr = ph_restrict<T>(A, l, fld(l), fld(l - 1), first_of(loc), step_of(loc), t, slot, S, pk);
      if (!sync(okr, loc, (l - 1) <= K)) return false;
    }
    // coarsest level
    if (A.it_P) {
      const bool loc = 1 <= K;
      if (runs(loc)) ph_direct_top<T>(A, fld(1), L > 1, loc ? 0 : blockIdx.x, loc ? 1 : gridDim.x, t, slot, s_direct);
      if (!sync(true, loc, 2 <= K || L < 2)) return false;
    } else {
      const bool loc = 1 <= K;
      for (int it = 0; it < A.ntop; ++it) {
        const bool last = it == A.ntop - 1;
        bool ok = true;
        if (runs(loc))
          ok = ph_gsi<T>(A, 1, fld(1), oth(1), nullptr, it == 0 && L > 1, last && L > 1, it == 0 && L > 1,
                         first_of(loc), step_of(loc), t, slot, S, pk);
        cur ^= 1u << 1;
        if (!sync(ok, loc, last ? (2 <= K || L < 2) : loc)) return false;
      }
    }
    // ascending leg
    for (int l = 2; l <= L; ++l) {
      const bool loc = l <= K;
      bool okp = true;
      if (runs(loc)) okp = ph_prolong<T>(A, l, fld(l), fld(l - 1), first_of(loc), step_of(loc), t, slot, S, pk);
      if (!sync(okp, loc, loc)) return false;
      for (int it = 0; it < A.nup; ++it) {
        const bool last = it == A.nup - 1;
        bool ok = true;
        if (runs(loc))
          ok = ph_gsi<T>(A, l, fld(l), oth(l), A.e, false, last && l < L, false, first_of(loc), step_of(loc), t,
                         slot, S, pk);
        cur ^= 1u << l;
        const bool next_loc = last ? ((l + 1) <= K) : loc;
        if (!sync(ok, loc, l == L && last ? false : next_loc)) return false;
      }
    }

    // levels left in the second buffer go back to u
    bool any = false;
    for (int l = 1; l <= L; ++l)
      if ((cur >> l) & 1) {
        ph_copy_back<T>(A, l, A.ualt, A.u, blockIdx.x * nslots + slot, gridDim.x * nslots, t);
        any = true;
      }
    if (any && !grid_barrier(A.bar, A.err, epoch, A.timeout_ns)) return false;
    return true;

  };

  const bool mixed = A.mx.u64 != nullptr;
  const bool loop = A.max_cycles > 0;  // without it: one V-cycle (vcycle!), no norms
  int cycles = 0;
  if (loop && !mixed && !norm_step(false, true, 0)) return;
  for (int iter = 0;; ++iter) {
    if (loop && mixed) {
      // FP64 side of a defect-correction step
      if (A.mx.apply_update || iter > 0) {
        ph_update64<T>(A, t, gslot, gstep);
        if (!sync(true, false, false)) return;
      }
      for (int l = L; l >= 2; --l) {
        ph_restrict64<T>(A, l, t, gslot, gstep);
        if (!sync(true, false, false)) return;
      }
      for (int l = 2; l <= L; ++l)
        if ((A.mx.refbnd_levels >> l) & 1) {
          ph_refbnd64<T>(A, l, t, gslot, gstep);
          if (!sync(true, false, false)) return;
        }
      if (!norm_step(true, iter == 0, cycles)) return;
    }
    if (loop && (!any_live() || cycles >= A.max_cycles)) break;
    if (!vcycle_body()) return;
    cycles++;
    if (!loop) break;
    if (!mixed && !norm_step(false, false, cycles)) return;
  }
  if (loop && A.out && cta0 && threadIdx.x == 0) A.out[0] = (double)cycles;
  if (A.trace && cta0 && threadIdx.x == 0 && ntrace < kTraceMax) A.trace[ntrace] = 0;
}

}  // namespace srmg
