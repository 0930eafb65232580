// srmg_engine.cuh -- the persistent V-cycle engine: one cooperative launch runs a whole
// FAS V-cycle (src/multigrid.jl:60-106) with grid barriers between dependent phases.
//
// Phases (per level l, fine to coarse and back):
//   GS iteration     : one full red-black Gauss-Seidel iteration (red sweep, copy and
//                      mirror ghost fills, black sweep, fills; src/multigrid.jl:250-265)
//                      in ONE phase.  The iteration reads the level's current buffer and
//                      writes the other one (ping-pong per level).  A half slot stages its
//                      block with ghosts in shared memory, updates the red cells, then
//                      recomputes the red update of every neighbour edge cell its black
//                      cells will read (their stencils touch only black cells and stored
//                      ghosts of the old buffer, and every product and sum is rounded as
//                      in the neighbour's own update, so the values are bit-identical),
//                      updates the black cells, and writes the block plus the ghost
//                      values it feeds: the facing ghosts of its neighbours
//                      (fill_ghost_copy!), its mirror ghosts (fill_ghost_bnd!) and its
//                      frozen refinement ghosts.  No two slots write one address.
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
// bulk asynchronous copies (cp.async.bulk, no multicast) into a four-buffer per-slot
// pipeline; every wait on an mbarrier or a barrier is bounded in time.  The arithmetic
// of every phase is the per-operation kernels' (the same products and sums, rounded the
// same way, in the same order), so an FP64 V-cycle equals the oracle's bit for bit.
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
  const T *wrow;     // weight rows per block coordinate (2 x kS values each), or null (geometry 0)
  int geom;
  int bghost;        // b's neighbour-copy ghosts are kept filled (the launch may write them)
  int lmax;          // finest non-empty level taking part
  int ndown, ntop, nup;
  int local_top;     // levels 1..local_top run inside CTA 0
  int top;           // the coarsest level a V-cycle visits: 1, or 2 (a lone item's direct solve there)
  int smooth_level;  // > 0: run smooth_n GS iterations on this level only (gauss_seidel_iter!)
  int smooth_n;
  int nitems;
  int nlev_tab;                // row length of it_lrange
  const T *it_par;             // per item: kParStride operator values (s_l, centre_l, nwc_l)
  const int *it_sgbits;        // per item: the 3x3 boundary table, entry k as (bc_k + 1) << 2k
  const double *const *it_P;   // per item: P = -s_t A_t^{-1} of its level t = top (row-major), or null
  const int2 *it_lrange;       // [item * nlev_tab + l - 1]: {first, count} in level l's block list
  int *frozen;                 // per item: nonzero once it has stopped iterating (zero at launch)
  unsigned *bar;     // barrier counter, zero at launch
  int *err;          // error word (0 = ok)
  long long timeout_ns;
  long long *trace;  // optional: CTA 0 stamps %globaltimer after every phase
  MixedArgs mx;            // mixed-precision outer step (mx.u64 != nullptr)
  int inner;               // mixed: FP32 V-cycles per defect-correction step (>= 1)
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

// Grid-wide barrier on a monotonic counter, also usable in two halves: grid_arrive
// counts this CTA in (its earlier memory operations, loads included, ordered before the
// count by the release) without waiting; grid_wait waits for every CTA of the same
// epoch.  A wait longer than timeout_ns sets the error word and returns false; every CTA
// then leaves the kernel at its next check.
__device__ __forceinline__ void grid_arrive(unsigned *bar, unsigned &epoch) {
  // this phase's generic-proxy stores are ordered before the next phase's bulk copies
  asm volatile("fence.proxy.async.global;" ::: "memory");
  __syncthreads();
  if (threadIdx.x == 0) {
    epoch++;
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
  }
}
__device__ __forceinline__ bool grid_wait(unsigned *bar, int *err, unsigned epoch, long long timeout_ns) {
  __shared__ int ok_s;
  if (threadIdx.x == 0) {
    const unsigned target = epoch * gridDim.x;
    int ok = 1;
    const long long t0 = gtimer();
    // the error word and the clock are read every 32 polls only: each read is another
    // memory round trip between two polls (measured: 1.42 -> 1.29 us per barrier)
    for (unsigned it = 1;; ++it) {
      unsigned v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
      if (v >= target) break;
      if ((it & 31u) == 0) {
        if (*(volatile int *)err) { ok = 0; break; }
        if (gtimer() - t0 > timeout_ns) {
          atomicCAS(err, 0, 1);
          ok = 0;
          break;
        }
      }
      __nanosleep(20);
    }
    ok_s = ok;
  }
  __syncthreads();
  asm volatile("fence.proxy.async.global;" ::: "memory");
  return ok_s != 0;
}
__device__ __forceinline__ bool grid_barrier(unsigned *bar, int *err, unsigned &epoch,
                                             long long timeout_ns) {
  grid_arrive(bar, epoch);
  return grid_wait(bar, err, epoch, timeout_ns);
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

// Per-slot staging: kBuf buffers of block tiles and the records of a chunk of up to
// kChunk blocks.  The GS, restriction and prolongation phases take two blocks per
// iteration (one per half slot), so four buffers hold the current pair and the next.
// Shared memory is kept small on purpose: what the CTA does not claim stays L1 cache for
// the scattered loads (face records, coarse values of refinement ghosts, spills), and a
// larger staging area measured slower.
constexpr int kBuf = 4;
constexpr int kChunk = 32;
// The thread of a slot that issues the GS, restriction and prolongation tile copies: its
// last (warp 3 of the second half), which has neither the GS halo update (warp 1 of
// each half) nor a share of the restriction's 2 x 2 sums (threads 0-63 of each half), so
// that no warp carries two of those extra paths between slot barriers (config 2's mixed
// solve: issuing from thread 0 with the halo on warp 0 cost 4-5%).
constexpr int kIssuer = 255;
constexpr int kWRow = 2 * kS;  // a weight row: wm, then wp, at the tile positions 0..19
// Launch-long record cache: a single-item launch loads, once at its start and level by
// level from the coarsest, a slot's whole share of a level's GS, restriction and
// prolongation records into kRecRows rows of the slot's shared memory while it fits (at
// most one chunk per level and kind), so that those phases issue their tile copies at
// once instead of after one or two dependent record loads.  FP64 keeps the footprint of
// two blocks per level on twelve levels (the 1024-thread FP64 shape is sensitive to the
// L1 it leaves); FP32 takes a third more.
template <typename T>
constexpr int kRecRows = sizeof(T) == 4 ? 96 : 72;
template <typename T>
struct SlotSmem {
  T tile[kBuf][kSS];
  T tile2[kBuf][kSS];  // the second tile of a pair: b (GS, restriction) or the parent's e (prolongation)
  T wst[kBuf][kWRow];  // the block's weight row (GS, restriction)
  int4 recs[kChunk][6];
  // cached rows: GS {blk, cr, cz, mask} + 4 faces; restriction {child edge}, fine info,
  // 4 coarse faces; prolongation {child edge} + 4 fine faces
  int4 rc[kRecRows<T>][6];
  uint64_t bar[kBuf];
  int sel[kChunk];  // list positions of the chunk's blocks that take part
  int cnt;
  int cstep[kMaxLev];                  // the list step the level's cached rows were taken with
  signed char off_gs[kMaxLev];         // first cached row of level l's GS records, or -1
  signed char off_res[kMaxLev];        // ... of its restriction records (child edges at level l)
  signed char off_pro[kMaxLev];        // ... of its prolongation records
  signed char pad_[(16 - (3 * kMaxLev + 4) % 16) % 16];
};
static_assert(kRecRows<float> <= 127 && kRecRows<double> <= 127, "row offsets are signed chars");
// Bulk copies land on 16-byte boundaries: every tile buffer of every slot.
static_assert(sizeof(SlotSmem<double>) % 16 == 0 && sizeof(SlotSmem<float>) % 16 == 0, "slot size");
static_assert((kSS * sizeof(float)) % 16 == 0 && (kBuf * kSS * sizeof(float)) % 16 == 0, "tile offsets");
static_assert((kWRow * sizeof(float)) % 16 == 0, "weight rows");

// Warp 0 of a slot: the list positions first + idx * step, c0 <= idx < min(c0 + kChunk,
// nmine), whose item is live (take(gi) true), compacted in order into S.sel; S.cnt
// their number.  The caller synchronises the slot before reading them.
template <typename T, typename Take>
__device__ __forceinline__ void select_chunk(SlotSmem<T> &S, int t, int c0, int nmine, int first, int step,
                                             Take take_of) {
  if (t < 32) {
    int base = 0;
    for (int h = 0; h < kChunk / 32; ++h) {
      const int idx = c0 + 32 * h + t;
      int gi = 0;
      bool take = false;
      if (idx < nmine) {
        gi = first + idx * step;
        take = take_of(gi);
      }
      const unsigned m = __ballot_sync(0xffffffffu, take);
      if (take) S.sel[base + __popc(m & ((1u << t) - 1u))] = gi;
      base += __popc(m);
    }
    if (t == 0) S.cnt = base;
  }
}

// After a failed wait on block j's buffer: wait (bounded) for the copies issued for
// blocks j + 1 .. j + kBuf - 1 of the chunk, so that none is left in flight.
template <typename T>
__device__ __forceinline__ void drain_slot(const EngArgs<T> &A, SlotSmem<T> &S, unsigned kb, int j, int cn) {
  for (int q = 1; q < kBuf && j + q < cn; ++q)
    mbar_wait(&S.bar[(kb + q) % kBuf], ((kb + q) / kBuf) & 1, A.err, A.timeout_ns);
}

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

// The neighbour copies of push_f only (no mirror ghosts).
template <typename F>
__device__ __forceinline__ void copy_ghost(F *field, int X, const int4 *fc, int x, int y, F v) {
  (void)X;
  if (x <= 3) {
    const int4 fi = fc[0];
    if (fi.w >= 0) field[(int64_t)fi.w * kSS + (x + kM) + kS * y] = v;
  }
  if (x >= 16) {
    const int4 fi = fc[1];
    if (fi.w >= 0) field[(int64_t)fi.w * kSS + (x - kM) + kS * y] = v;
  }
  if (y <= 3) {
    const int4 fi = fc[2];
    if (fi.w >= 0) field[(int64_t)fi.w * kSS + x + kS * (y + kM)] = v;
  }
  if (y >= 16) {
    const int4 fi = fc[3];
    if (fi.w >= 0) field[(int64_t)fi.w * kSS + x + kS * (y - kM)] = v;
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

// Refinement-boundary ghost q (0..127) of a block whose face record for face q / 32 is
// fi: the ghost's position (gx, gy) and its value interpolated from `src` on the
// coarser level (fill_ghost_interp!, src/connectivity.jl:251-258).  fi must be a
// FACE_REFBND record.
template <typename T>
__device__ __forceinline__ T refbnd_val(const T *src, int4 fi, int q, int &gx, int &gy) {
  const int f = q >> 5, lane = q & 31;
  const int g = lane >> 4, k = lane & 15;
  ghost_xy(f, lane, gx, gy);
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
  return v;
}

// Refinement-boundary ghost q (0..127) of block X in `dst`, from `src` on the coarser level.
template <typename T>
__device__ __forceinline__ void refbnd_ghost(T *dst, const T *src, int X, const int4 *fc, int q) {
  const int4 fi = fc[q >> 5];
  if (fi.x != FACE_REFBND) return;
  int x, y;
  const T v = refbnd_val<T>(src, fi, q, x, y);
  dst[(int64_t)X * kSS + x + kS * y] = v;
}

// {type, push target} of face f of a block (a face record's x and w), for pushes from
// records preloaded in registers.
__device__ __forceinline__ int2 face_tw(const int4 *fc, int f) {
  const int4 r = fc[f];
  return make_int2(r.x, r.w);
}

// push_f with the records of the x-face (face 0 if x <= 3, 1 if x >= 16) and the y-face
// (face 2 if y <= 3, 3 if y >= 16) of cell (x, y) given as {type, push target}.
template <typename F>
__device__ __forceinline__ void push_tw(unsigned sgb, F *field, int X, int2 fx, int2 fy, int x, int y, F v) {
  F *xb = field + (int64_t)X * kSS;
  if (x <= 3) {
    if (fx.y >= 0) field[(int64_t)fx.y * kSS + (x + kM) + kS * y] = v;
    else if (fx.x == FACE_BOUNDARY) xb[(2 * kG - 1 - x) + kS * y] = dmul<F>(sign_at<F>(sgb, 3), v);
  }
  if (x >= 16) {
    if (fx.y >= 0) field[(int64_t)fx.y * kSS + (x - kM) + kS * y] = v;
    else if (fx.x == FACE_BOUNDARY) xb[(2 * (kG + kM) - 1 - x) + kS * y] = dmul<F>(sign_at<F>(sgb, 5), v);
  }
  if (y <= 3) {
    if (fy.y >= 0) field[(int64_t)fy.y * kSS + x + kS * (y + kM)] = v;
    else if (fy.x == FACE_BOUNDARY) xb[x + kS * (2 * kG - 1 - y)] = dmul<F>(sign_at<F>(sgb, 1), v);
  }
  if (y >= 16) {
    if (fy.y >= 0) field[(int64_t)fy.y * kSS + x + kS * (y - kM)] = v;
    else if (fy.x == FACE_BOUNDARY) xb[x + kS * (2 * (kG + kM) - 1 - y)] = dmul<F>(sign_at<F>(sgb, 7), v);
  }
}

// ------------------------------------------------------------------ phases

// Two tiles on one mbarrier: block X of src into tile[buf], block Y of src2 into tile2[buf].
template <typename T>
__device__ __forceinline__ void issue_pair(SlotSmem<T> &S, int buf, const T *src, int X, const T *src2, int Y) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mbar_expect_tx(&S.bar[buf], (uint32_t)(2 * kSS * sizeof(T)));
  bulk_g2s(S.tile[buf], src + (int64_t)X * kSS, (uint32_t)(kSS * sizeof(T)), &S.bar[buf]);
  bulk_g2s(S.tile2[buf], src2 + (int64_t)Y * kSS, (uint32_t)(kSS * sizeof(T)), &S.bar[buf]);
}

// The u and b tiles of block X and, with a weight table, the weight row of the block's
// coordinate (cr for geometry 1, cz for geometry 2), on one mbarrier.
template <typename T>
__device__ __forceinline__ void issue_block(const EngArgs<T> &A, SlotSmem<T> &S, int buf, const T *src, int X,
                                            int cr, int cz) {
  const uint32_t wb = A.wrow ? (uint32_t)(kWRow * sizeof(T)) : 0u;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mbar_expect_tx(&S.bar[buf], (uint32_t)(2 * kSS * sizeof(T)) + wb);
  bulk_g2s(S.tile[buf], src + (int64_t)X * kSS, (uint32_t)(kSS * sizeof(T)), &S.bar[buf]);
  bulk_g2s(S.tile2[buf], A.b + (int64_t)X * kSS, (uint32_t)(kSS * sizeof(T)), &S.bar[buf]);
  if (wb) bulk_g2s(S.wst[buf], A.wrow + (int64_t)(A.geom == 1 ? cr : cz) * kWRow, wb, &S.bar[buf]);
}

// weights() from a staged weight row.
template <typename T>
__device__ __forceinline__ W5<T> wrow_w(int geom, const T *row, int x, int y) {
  W5<T> w{T(1), T(1), T(1), T(1)};
  if (geom == 1) {
    w.rm = row[x];
    w.rp = row[kS + x];
  } else if (geom == 2) {
    w.zm = row[y];
    w.zp = row[kS + y];
  }
  return w;
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

// Red halo cell m (0..31) of a block, handled by lane m of warp 1 of a half slot (the
// cell 2 (m % 8) + (m / 8 % 2) of ghost face m / 8), packed into two ints once per CTA:
// {hx | hy << 5 | nx << 10 | ny << 15 | f << 20 | nsub << 22, (cx + 1) | (cy + 1) << 6 |
// (cnx + 1) << 12 | (cny + 1) << 18}, the corner fields all -1 where there is none.
__device__ __forceinline__ int2 halo_pack(int m) {
  const HaloCell h = halo_cell(16 * (m >> 3) + 2 * (m & 7) + ((m >> 3) & 1));
  const int w0 = h.hx | (h.hy << 5) | (h.nx << 10) | (h.ny << 15) | (h.f << 20) | (h.nsub << 22);
  const int w1 = h.cx < 0 ? 0 : (h.cx + 1) | ((h.cy + 1) << 6) | ((h.cnx + 1) << 12) | ((h.cny + 1) << 18);
  return make_int2(w0, w1);
}
__device__ __forceinline__ HaloCell halo_unpack(int2 w) {
  HaloCell h;
  h.hx = w.x & 31;
  h.hy = (w.x >> 5) & 31;
  h.nx = (w.x >> 10) & 31;
  h.ny = (w.x >> 15) & 31;
  h.f = (w.x >> 20) & 3;
  h.nsub = (w.x >> 22) & 3;
  h.jj = 0;
  h.red = true;
  h.cx = (w.y & 63) - 1;
  h.cy = ((w.y >> 6) & 63) - 1;
  h.cnx = ((w.y >> 12) & 63) - 1;
  h.cny = ((w.y >> 18) & 63) - 1;
  return h;
}

// Vector access to the two cells (x, x+1), x even, of a tile row: 16 bytes (FP64) or 8
// bytes (FP32), aligned because tiles and fields are 16-byte aligned and kS is even.
template <typename T> struct Pair2;
template <> struct Pair2<double> { using V = double2; };
template <> struct Pair2<float> { using V = float2; };
template <typename T>
__device__ __forceinline__ void ld_pair(const T *p, T &a, T &b) {
  const typename Pair2<T>::V v = *reinterpret_cast<const typename Pair2<T>::V *>(p);
  a = v.x;
  b = v.y;
}
template <typename T>
__device__ __forceinline__ void st_pair(T *p, T a, T b) {
  typename Pair2<T>::V v;
  v.x = a;
  v.y = b;
  *reinterpret_cast<typename Pair2<T>::V *>(p) = v;
}

// The order-2 stencil of applystencil (src/laplacian.jl:25-49,78-118) on values already
// loaded: apply5's products and sums, in its order, each rounded on its own (no FMA
// contraction), so that the engine's updates equal the per-operation kernels' and the
// halo recompute of a neighbour's red edge cell equals the neighbour's own update bit
// for bit.
template <typename T>
__device__ __forceinline__ T sten5(const W5<T> &w, T centre, T zm, T rm, T c, T rp, T zp) {
  T v = dadd<T>(T(0), dmul<T>(w.zm, zm));
  v = dadd<T>(v, dmul<T>(w.rm, rm));
  v = dadd<T>(v, dmul<T>(centre, c));
  v = dadd<T>(v, dmul<T>(w.rp, rp));
  v = dadd<T>(v, dmul<T>(w.zp, zp));
  return v;
}

// push_f for the two cells (x0, y), (x0 + 1, y) of one thread, x0 even: the copies into
// the neighbours' facing ghosts and (kMirror) the block's own mirror ghosts, as pair
// stores.
template <typename F, bool kMirror = true>
__device__ __forceinline__ void push_pair(unsigned sgb, F *field, int X, const int4 *fc, int x0, int y, F v0,
                                          F v1) {
  F *xb = field + (int64_t)X * kSS;
  if (x0 == 2) {
    const int4 fi = fc[0];
    if (fi.w >= 0) st_pair<F>(field + (int64_t)fi.w * kSS + (x0 + kM) + kS * y, v0, v1);
    else if (kMirror && fi.x == FACE_BOUNDARY) {
      const F sg = sign_at<F>(sgb, 3);
      st_pair<F>(xb + kS * y, dmul<F>(sg, v1), dmul<F>(sg, v0));  // x = 3 -> 0, x = 2 -> 1
    }
  }
  if (x0 == 16) {
    const int4 fi = fc[1];
    if (fi.w >= 0) st_pair<F>(field + (int64_t)fi.w * kSS + (x0 - kM) + kS * y, v0, v1);
    else if (kMirror && fi.x == FACE_BOUNDARY) {
      const F sg = sign_at<F>(sgb, 5);
      st_pair<F>(xb + 18 + kS * y, dmul<F>(sg, v1), dmul<F>(sg, v0));  // x = 17 -> 18, x = 16 -> 19
    }
  }
  if (y <= 3) {
    const int4 fi = fc[2];
    if (fi.w >= 0) st_pair<F>(field + (int64_t)fi.w * kSS + x0 + kS * (y + kM), v0, v1);
    else if (kMirror && fi.x == FACE_BOUNDARY) {
      const F sg = sign_at<F>(sgb, 1);
      st_pair<F>(xb + x0 + kS * (2 * kG - 1 - y), dmul<F>(sg, v0), dmul<F>(sg, v1));
    }
  }
  if (y >= 16) {
    const int4 fi = fc[3];
    if (fi.w >= 0) st_pair<F>(field + (int64_t)fi.w * kSS + x0 + kS * (y - kM), v0, v1);
    else if (kMirror && fi.x == FACE_BOUNDARY) {
      const F sg = sign_at<F>(sgb, 7);
      st_pair<F>(xb + x0 + kS * (2 * (kG + kM) - 1 - y), dmul<F>(sg, v0), dmul<F>(sg, v1));
    }
  }
}

// Named barrier of a slot that also ANDs a predicate over its 256 threads.
__device__ __forceinline__ bool slot_and(int slot, bool ok) {
  uint32_t r;
  asm volatile(
      "{ .reg .pred p, q; setp.ne.u32 q, %1, 0; bar.red.and.pred p, %2, 256, q; selp.u32 %0, 1, 0, p; }"
      : "=r"(r)
      : "r"((uint32_t)ok), "r"(slot + 1)
      : "memory");
  return r != 0;
}

// One fused red-black GS iteration over level l: src -> dst (gauss_seidel_iter!,
// src/multigrid.jl:250-265).  A slot's 256 threads smooth two blocks at a time, one per
// half; thread h of a half owns the cell pair (x0, y), (x0 + 1, y), x0 = 2 + 2 (h % 8),
// y = 2 + h / 8, which holds one red and one black cell.  Each block's u tile (with
// ghosts) and b tile stream through the slot's kBuf-deep shared-memory pipeline as two
// bulk copies on one mbarrier; the few scattered inputs (the FAS restricted residual,
// u1 for e, the neighbours' edge b and ghost corners) are loaded into registers one
// iteration ahead.  Per iteration: the red cells of the pair and the neighbours' red
// edge cells held in this block's ghost layer are updated in shared memory; one slot
// barrier; the black cells are updated in registers and the pair is written out with
// its ghost copies.  With `fas`, the FAS right-hand side of the covered cells
// (src/multigrid.jl:112-119) is formed first from the post-restriction tile and the
// restricted residual held in e, and a second barrier separates those reads from the
// red writes.
template <typename T>
__device__ bool ph_gsi(const EngArgs<T> &A, int l, const T *src, T *dst, const T *esrc, bool copy_u1,
                       bool make_e, bool fas, int first, int step, int t, int slot, SlotSmem<T> &S,
                       unsigned &pk, const int2 *halo_tab) {
  const int n = A.tr.nblk[l - 1];
  const int4 *recs = A.tr.lvl_rec[l - 1];
  const int nmine = (first < n) ? (n - 1 - first) / step + 1 : 0;
  if (nmine == 0) return true;
  const int half = t >> 7, h = t & 127;
  // warp wv of a half holds rows of one parity (wv / 2: even, odd), so that the red and
  // black roles of a thread's two cells are uniform across the warp
  const int wv = h >> 5, lane = h & 31;
  const int x0 = 2 + 2 * (lane & 7), y = 2 + (wv >> 1) + 2 * (4 * (wv & 1) + (lane >> 3));
  const int o0 = x0 + kS * y;
  const bool yodd = (y & 1) != 0;  // red (colour 0 of RedBlack{0}, updated first) is x0 if y is odd
  const int xr = yodd ? x0 : x0 + 1, xbk = yodd ? x0 + 1 : x0;  // the pair's red and black cells
  const int mysub = ((x0 - 2) >> 3) + 2 * ((y - 2) >> 3);
  // warp 1 of a half: the 32 red halo cells, lane m taking entry m of the halo table (one
  // warp issues the halo code instead of a quarter of every warp's lanes; not warp 0,
  // whose first half holds thread 0)
  const bool hthr = wv == 1;
  const int hm = lane;  // this lane's entry of the halo table
  // neighbour values of the halo cell, loaded one iteration ahead
  // (b comes from b's ghost layer when A.bghost, except the FAS right-hand side of a
  // covered neighbour cell, formed here from the neighbour's restricted residual in e)
  T hvn = T(0), hcn = T(0);
  // the records: the launch-long cache of a small level, or the chunk staged in recs
  const int co = A.nitems == 1 && step == S.cstep[l - 1] ? S.off_gs[l - 1] : -1;
  const bool cached = co >= 0;
  int4(*R)[6] = cached ? &S.rc[co] : S.recs;
  auto prefetch = [&](int j) {
    if (hthr) {
      const HaloCell hc_ = halo_unpack(halo_tab[hm]);
      const int4 fi = R[j][1 + hc_.f];
      if (fi.x == FACE_NEIGHBOR) {
        const int64_t nb = (int64_t)fi.y * kSS;
        const bool covn = fas && ((fi.z >> hc_.nsub) & 1);
        if (covn) hvn = A.e[nb + hc_.nx + kS * hc_.ny];
        else if (!A.bghost) hvn = A.b[nb + hc_.nx + kS * hc_.ny];
        if (hc_.cx >= 0) hcn = src[nb + hc_.cnx + kS * hc_.cny];
      }
    }
  };
  auto issue = [&](int j) {
    const int4 bk = R[j][0];
    issue_block<T>(A, S, (pk + j) % kBuf, src, bk.x, bk.y, bk.z);
  };
  // one item: the operator values and the boundary table stay in registers for the
  // whole level
  T s = A.it_par[l], centre = A.it_par[32 + l], nwc = A.it_par[64 + l];
  const unsigned sgb1 = (unsigned)A.it_sgbits[0];
  for (int c0 = 0; c0 < nmine; c0 += kChunk) {
    int cn;
    if (cached) {
      cn = nmine;  // <= kChunk, one chunk
    } else if (A.nitems == 1) {
      cn = min(kChunk, nmine - c0);
      for (int i = t; i < 5 * cn; i += 256) {
        const int q = i / 5, k = i - 5 * q;
        S.recs[q][k] = recs[5 * (first + (c0 + q) * step) + k];
      }
      slot_sync(slot);
    } else {
      // the chunk's next list positions, without the blocks of frozen items
      select_chunk<T>(S, t, c0, nmine, first, step, [&](int gi) { return !A.frozen[item_of(recs[5 * gi])]; });
      slot_sync(slot);
      cn = S.cnt;
      for (int i = t; i < 5 * cn; i += 256) {
        const int q = i / 5, k = i - 5 * q;
        S.recs[q][k] = recs[5 * S.sel[q] + k];
      }
      slot_sync(slot);
      if (cn == 0) continue;
    }
    if (t == kIssuer)
      for (int q = 0; q < kBuf && q < cn; ++q) issue(q);
    if (half < cn) prefetch(half);
    for (int i = 0; 2 * i < cn; ++i) {
      const int j = 2 * i + half;
      const bool act = j < cn;
      const unsigned kb = pk + j;
      const int buf = kb % kBuf;
      const T hv = hvn, hc = hcn;
      if (j + 2 < cn) prefetch(j + 2);
      const int4 bk = R[act ? j : 0][0];
      const int4 *fc = &R[act ? j : 0][1];
      const int64_t xo = (int64_t)bk.x * kSS + o0;
      const bool cov = fas && ((bk.w >> mysub) & 1);
      // the covered cells' restricted residual (FAS), loaded while the tiles arrive, and
      // in FP32 the pair's u1 (for e) as well (the register-capped FP64 shape would spill)
      T ex0 = T(0), ex1 = T(0), uo0 = T(0), uo1 = T(0);
      if (act && cov) ld_pair<T>(A.e + xo, ex0, ex1);
      if (sizeof(T) == 4 && act && make_e) ld_pair<T>(A.u1 + xo, uo0, uo1);
      bool ok = true;
      if (act) ok = mbar_wait(&S.bar[buf], (kb / kBuf) & 1, A.err, A.timeout_ns);
      T *tile = S.tile[buf];
      T cb = T(0), red_new = T(0), bb = T(0);  // the black cell's old value and b; the new red value
      if (act && ok) {
        if (A.nitems > 1) {
          const T *par = A.it_par + item_of(bk) * kParStride;
          s = par[l];
          centre = par[32 + l];
          nwc = par[64 + l];
        }
        T c0v, c1v, b0, b1, dn0, dn1, up0, up1;
        ld_pair<T>(tile + o0, c0v, c1v);
        ld_pair<T>(S.tile2[buf] + o0, b0, b1);
        ld_pair<T>(tile + o0 - kS, dn0, dn1);
        ld_pair<T>(tile + o0 + kS, up0, up1);
        if (copy_u1) st_pair<T>(A.u1 + xo, c0v, c1v);
        T Lr;  // the red cell's stencil
        if (cov) {
          const W5<T> w0 = wrow_w<T>(A.geom, S.wst[buf], x0, y);
          const W5<T> w1 = wrow_w<T>(A.geom, S.wst[buf], x0 + 1, y);
          const T Lu0 = sten5<T>(w0, centre, dn0, tile[o0 - 1], c0v, c1v, up0);
          const T Lu1 = sten5<T>(w1, centre, dn1, c0v, c1v, tile[o0 + 2], up1);
          b0 = -(ex0 + Lu0 / s);
          b1 = -(ex1 + Lu1 / s);
          st_pair<T>(A.b + xo, b0, b1);
          if (A.bghost) push_pair<T, false>(0u, A.b, bk.x, fc, x0, y, b0, b1);
          Lr = yodd ? Lu0 : Lu1;
        } else {
          const W5<T> wr = wrow_w<T>(A.geom, S.wst[buf], xr, y);
          Lr = yodd ? sten5<T>(wr, centre, dn0, tile[o0 - 1], c0v, c1v, up0)
                    : sten5<T>(wr, centre, dn1, c0v, c1v, tile[o0 + 2], up1);
        }
        red_new = yodd ? fma(nwc, fma(s, b0, Lr), c0v) : fma(nwc, fma(s, b1, Lr), c1v);
        cb = yodd ? c1v : c0v;
        bb = yodd ? b1 : b0;
      }
      // red update of the neighbour's edge cell that sits in this block's ghost layer
      T halo_new = T(0);
      int halo_o = -1;
      if (act && ok && hthr) {
        const HaloCell hc_ = halo_unpack(halo_tab[hm]);
        const int4 fi = fc[hc_.f];
        if (fi.x == FACE_NEIGHBOR) {
          auto at = [&](int a, int c) -> T { return (a == hc_.cx && c == hc_.cy) ? hc : tile[a + kS * c]; };
          const W5<T> wh = wrow_w<T>(A.geom, S.wst[buf], hc_.hx, hc_.hy);
          const T v = sten5<T>(wh, centre, at(hc_.hx, hc_.hy - 1), at(hc_.hx - 1, hc_.hy),
                               tile[hc_.hx + kS * hc_.hy], at(hc_.hx + 1, hc_.hy), at(hc_.hx, hc_.hy + 1));
          const T bn = (fas && ((fi.z >> hc_.nsub) & 1)) ? -(hv + v / s)
                       : A.bghost                          ? S.tile2[buf][hc_.hx + kS * hc_.hy]
                                                           : hv;
          halo_o = hc_.hx + kS * hc_.hy;
          halo_new = fma(nwc, fma(s, bn, v), tile[halo_o]);
        }
      }
      if (fas) ok = slot_and(slot, ok);  // every old value is read before the red writes
      if (act && ok) {
        tile[xr + kS * y] = red_new;
        if (halo_o >= 0) tile[halo_o] = halo_new;
      }
      if (!slot_and(slot, ok)) {
        // leave no copy in flight: wait (bounded) for every one issued and not consumed
        const int issued = min(cn, kBuf + 2 * max(0, i - 1));
        for (int q = 2 * i; q < issued; ++q)
          mbar_wait(&S.bar[(pk + q) % kBuf], ((pk + q) / kBuf) & 1, A.err, A.timeout_ns);
        return false;
      }
      // the buffers of the previous iteration are free: refill them kBuf blocks later
      if (t == kIssuer && i >= 1)
        for (int q = 2 * i - 2 + kBuf; q < 2 * i + kBuf && q < cn; ++q) issue(q);
      if (act) {
        T dn0, dn1, up0, up1;
        ld_pair<T>(tile + o0 - kS, dn0, dn1);
        ld_pair<T>(tile + o0 + kS, up0, up1);
        const W5<T> wb = wrow_w<T>(A.geom, S.wst[buf], xbk, y);
        const T Lb = yodd ? sten5<T>(wb, centre, dn1, red_new, cb, tile[o0 + 2], up1)
                          : sten5<T>(wb, centre, dn0, tile[o0 - 1], cb, red_new, up0);
        const T black_new = fma(nwc, fma(s, bb, Lb), cb);
        const T nu0 = yodd ? red_new : black_new, nu1 = yodd ? black_new : red_new;
        const int X = bk.x;
        const unsigned sgb = A.nitems == 1 ? sgb1 : (unsigned)A.it_sgbits[item_of(bk)];
        st_pair<T>(dst + xo, nu0, nu1);
        push_pair<T>(sgb, dst, X, fc, x0, y, nu0, nu1);
        if (fc[wv].x == FACE_REFBND) {  // warp wv: the 32 ghost cells of face wv
          int gx, gy;
          ghost_xy(wv, lane, gx, gy);
          dst[(int64_t)X * kSS + gx + kS * gy] = tile[gx + kS * gy];  // frozen during smoothing
        }
        if (make_e) {
          if (sizeof(T) == 8) ld_pair<T>(A.u1 + xo, uo0, uo1);
          const T ev0 = nu0 - uo0, ev1 = nu1 - uo1;
          st_pair<T>(A.e + xo, ev0, ev1);
          push_pair<T>(sgb, A.e, X, fc, x0, y, ev0, ev1);
          refbnd_ghost<T>(A.e, esrc, X, fc, h);
        }
      }
    }
    pk += cn;
    slot_sync(slot);  // the chunk's records and buffers are no longer read
  }
  return true;
}

// Residual and restriction of r and u (src/multigrid.jl:60-106 with restrict!,
// src/restrict.jl:5-25): the restricted u goes to the coarse block (and into the coarse
// ghosts that copy it), the restricted r to e, where the coarse level's first GS
// iteration reads it to form the FAS right-hand side.  uf: level l, uc: level l-1.
// A slot's halves take one child edge each per iteration; each fine block's u and b
// tiles stream through the slot's kBuf-deep bulk-copy pipeline, thread h of a half
// forms the residual of its cell pair from shared memory, and after one slot barrier
// 64 threads of the half restrict (the coarse block's face records are staged with the
// chunk).  The residual is double-buffered by iteration, so that one barrier per
// iteration suffices.  Children of frozen items are skipped.
template <typename T>
__device__ bool ph_restrict(const EngArgs<T> &A, int l, const T *uf, T *uc, int first, int step, int t, int slot,
                            SlotSmem<T> &S, unsigned &pk) {
  const int n = A.tr.nch[l - 1];
  const int4 *ch = A.tr.lvl_child[l - 1];
  const int nmine = (first < n) ? (n - 1 - first) / step + 1 : 0;
  if (nmine == 0) return true;
  const int half = t >> 7, h = t & 127;
  const int x0 = 2 + 2 * (h & 7), y = 2 + (h >> 3);
  const int o0 = x0 + kS * y;
  const int co = A.nitems == 1 && step == S.cstep[l - 1] ? S.off_res[l - 1] : -1;
  const bool cached = co >= 0;
  int4(*R)[6] = cached ? &S.rc[co] : S.recs;
  // one item: its operator values and boundary table, loaded before the first tile wait
  const T s1 = A.it_par[l], centre1 = A.it_par[32 + l];
  const unsigned sgb1 = (unsigned)A.it_sgbits[0];
  auto issue = [&](int j) {
    const int4 fi = R[j][1];
    issue_block<T>(A, S, (pk + j) % kBuf, uf, R[j][0].x, fi.x, fi.y);
  };
  for (int c0 = 0; c0 < nmine; c0 += kChunk) {
    // the chunk's next child edges, without those of frozen items: recs[q][0] = {fine,
    // coarse, sb_r, sb_z}, recs[q][1] = info of the fine block, recs[q][2..5] = the
    // coarse block's faces (or the launch-long cache of a small level)
    int cn;
    if (cached) {
      cn = nmine;  // <= kChunk, one chunk
    } else {
      select_chunk<T>(S, t, c0, nmine, first, step,
                      [&](int gi) { return A.nitems == 1 || !A.frozen[A.tr.info[ch[gi].x].z >> 8]; });
      slot_sync(slot);
      cn = S.cnt;
      for (int i = t; i < 6 * cn; i += 256) {
        const int q = i / 6, k = i - 6 * q;
        const int4 e = ch[S.sel[q]];
        S.recs[q][k] = k == 0 ? e : k == 1 ? A.tr.info[e.x] : A.tr.faces[4 * e.y + k - 2];
      }
      slot_sync(slot);
      if (cn == 0) continue;
    }
    if (t == kIssuer)
      for (int q = 0; q < kBuf && q < cn; ++q) issue(q);
    for (int i = 0; 2 * i < cn; ++i) {
      const int j = 2 * i + half;
      const bool act = j < cn;
      const unsigned kb = pk + j;
      const int buf = kb % kBuf;
      bool ok = true;
      if (act) ok = mbar_wait(&S.bar[buf], (kb / kBuf) & 1, A.err, A.timeout_ns);
      const T *tile = S.tile[buf];
      const int jj = act ? j : 0;
      const int4 e = R[jj][0], fi = R[jj][1];
      const int item = fi.z >> 8;
      if (act && ok) {
        const T *par = A.it_par + item * kParStride;
        const T s = A.nitems == 1 ? s1 : par[l], centre = A.nitems == 1 ? centre1 : par[32 + l];
        const W5<T> w0 = wrow_w<T>(A.geom, S.wst[buf], x0, y);
        const W5<T> w1 = wrow_w<T>(A.geom, S.wst[buf], x0 + 1, y);
        T c0v, c1v, b0, b1, dn0, dn1, up0, up1;
        ld_pair<T>(tile + o0, c0v, c1v);
        ld_pair<T>(S.tile2[buf] + o0, b0, b1);
        ld_pair<T>(tile + o0 - kS, dn0, dn1);
        ld_pair<T>(tile + o0 + kS, up0, up1);
        const T Lu0 = sten5<T>(w0, centre, dn0, tile[o0 - 1], c0v, c1v, up0);
        const T Lu1 = sten5<T>(w1, centre, dn1, c0v, c1v, tile[o0 + 2], up1);
        // the residual replaces the pair's own b values in the b tile (read by no one else)
        st_pair<T>(S.tile2[buf] + o0, -(b0 + Lu0 / s), -(b1 + Lu1 / s));
      }
      if (!slot_and(slot, ok)) {
        // leave no copy in flight: wait (bounded) for every one issued and not consumed
        const int issued = min(cn, kBuf + 2 * max(0, i - 1));
        for (int q = 2 * i; q < issued; ++q)
          mbar_wait(&S.bar[(pk + q) % kBuf], ((pk + q) / kBuf) & 1, A.err, A.timeout_ns);
        return false;
      }
      // the buffers of the previous iteration are free: refill them kBuf blocks later
      if (t == kIssuer && i >= 1)
        for (int q = 2 * i - 2 + kBuf; q < 2 * i + kBuf && q < cn; ++q) issue(q);
      if (act && h < 64) {
        const int kx = h & 7, ky = h >> 3;
        const int C = e.y;
        const int cx = 2 + 8 * (e.z - 1) + kx, cy = 2 + 8 * (e.w - 1) + ky;
        // 2x2 sums in the reference's order: (i, j), (i+1, j), (i, j+1), (i+1, j+1)
        const T cu = restrict4<T>(tile, 2 + 2 * kx, 2 + 2 * ky);
        const T cr = restrict4<T>(S.tile2[buf], 2 + 2 * kx, 2 + 2 * ky);
        uc[(int64_t)C * kSS + cx + kS * cy] = cu;
        push_f<T>(A.nitems == 1 ? sgb1 : (unsigned)A.it_sgbits[item], uc, C, &R[j][2], cx, cy, cu);
        A.e[(int64_t)C * kSS + cx + kS * cy] = cr;
      }
    }
    pk += cn;
    slot_sync(slot);  // the chunk's records and buffers are no longer read
  }
  return true;
}

// u_fine += P(e_coarse) on every valid cell (in place in uf), pushes of the new edge
// values, and the fine block's refinement-boundary ghosts from uc (final coarse level).
// A slot's halves take one child edge each per iteration; per child edge the fine
// block's u tile and its parent's e tile arrive together by two bulk copies on one
// mbarrier of the slot's kBuf-deep pipeline, and thread h of a half updates the cell
// pair (x0, y), (x0 + 1, y), x0 = 2 + 2 (h % 8), y = 2 + h / 8, and computes refinement
// ghost h, whose coarse values it loads while the tiles arrive.  The child's face records
// are staged in shared memory.  Children of frozen items are skipped.
template <typename T>
__device__ bool ph_prolong(const EngArgs<T> &A, int l, T *uf, const T *uc, int first, int step, int t, int slot,
                           SlotSmem<T> &S, unsigned &pk) {
  const int n = A.tr.nch[l - 1];
  const int4 *ch = A.tr.lvl_child[l - 1];
  const int nmine = (first < n) ? (n - 1 - first) / step + 1 : 0;
  if (nmine == 0) return true;
  const int half = t >> 7, h = t & 127;
  const int x0 = 2 + 2 * (h & 7), y = 2 + (h >> 3);
  const int o0 = x0 + kS * y;
  const int iz = (y - 2) & 1;  // the pair's coarse cell: column h % 8, row (y - 2) / 2 of the subblock
  const int co = A.nitems == 1 && step == S.cstep[l - 1] ? S.off_pro[l - 1] : -1;
  const bool cached = co >= 0;
  int4(*R)[6] = cached ? &S.rc[co] : S.recs;
  const unsigned sgb1 = (unsigned)A.it_sgbits[0];
  auto issue = [&](int j) { issue_pair<T>(S, (pk + j) % kBuf, uf, R[j][0].x, A.e, R[j][0].y); };
  for (int c0 = 0; c0 < nmine; c0 += kChunk) {
    // the chunk's next child edges, without those of frozen items:
    // recs[q][0] = {fine, coarse, sb_r, sb_z}, recs[q][1..4] = the fine block's faces
    // (or the launch-long cache of a small level)
    int cn;
    if (cached) {
      cn = nmine;  // <= kChunk, one chunk
    } else {
      select_chunk<T>(S, t, c0, nmine, first, step,
                      [&](int gi) { return A.nitems == 1 || !A.frozen[A.tr.info[ch[gi].x].z >> 8]; });
      slot_sync(slot);
      cn = S.cnt;
      for (int i = t; i < 5 * cn; i += 256) {
        const int q = i / 5, k = i - 5 * q;
        const int4 e = ch[S.sel[q]];
        S.recs[q][k] = k == 0 ? e : A.tr.faces[4 * e.x + k - 1];
      }
      slot_sync(slot);
      if (cn == 0) continue;
    }
    if (t == kIssuer)
      for (int q = 0; q < kBuf && q < cn; ++q) issue(q);
    for (int i = 0; 2 * i < cn; ++i) {
      const int j = 2 * i + half;
      const bool act = j < cn;
      const unsigned kb = pk + j;
      const int buf = kb % kBuf;
      const int4 e = R[act ? j : 0][0];
      const int4 *fc = &R[act ? j : 0][1];
      const int F = e.x;
      // loaded while the tiles arrive: refinement ghost h from the coarse level, the
      // item's boundary table
      const int4 gf = fc[h >> 5];
      const bool rb = act && gf.x == FACE_REFBND;
      T gv = T(0);
      int gx = 0, gy = 0;
      if (rb) gv = refbnd_val<T>(uc, gf, h, gx, gy);
      const unsigned sgb = (A.nitems == 1 || !act) ? sgb1 : (unsigned)A.it_sgbits[A.tr.info[F].z >> 8];
      bool ok = true;
      if (act) ok = mbar_wait(&S.bar[buf], (kb / kBuf) & 1, A.err, A.timeout_ns);
      if (act && ok) {
        const T *ut = S.tile[buf], *cb = S.tile2[buf];
        const int jr = 2 + 8 * (e.z - 1) + (h & 7), jz = 2 + 8 * (e.w - 1) + ((y - 2) >> 1);
        const int oc = jr + kS * jz;
        // interp (src/interp.jl:24-63): 1/2 of the parent cell, 1/4 of its r and z
        // neighbours on the child cell's side, in that order
        const T cc = dmul<T>(T(0.5), cb[oc]);
        const T cz = dmul<T>(T(0.25), cb[oc + kS * (2 * iz - 1)]);
        const T v0 = dadd<T>(dadd<T>(cc, dmul<T>(T(0.25), cb[oc - 1])), cz);
        const T v1 = dadd<T>(dadd<T>(cc, dmul<T>(T(0.25), cb[oc + 1])), cz);
        T u0, u1;
        ld_pair<T>(ut + o0, u0, u1);
        const T nu0 = dadd<T>(v0, u0), nu1 = dadd<T>(v1, u1);
        st_pair<T>(uf + (int64_t)F * kSS + o0, nu0, nu1);
        push_pair<T>(sgb, uf, F, fc, x0, y, nu0, nu1);
        if (rb) uf[(int64_t)F * kSS + gx + kS * gy] = gv;
      }
      if (!slot_and(slot, ok)) {
        // leave no copy in flight: wait (bounded) for every one issued and not consumed
        const int issued = min(cn, kBuf + 2 * i);
        for (int q = 2 * i; q < issued; ++q)
          mbar_wait(&S.bar[(pk + q) % kBuf], ((pk + q) / kBuf) & 1, A.err, A.timeout_ns);
        return false;
      }
      // this iteration's buffers (and records) are free: refill them kBuf blocks later
      if (t == kIssuer)
        for (int q = 2 * i + kBuf; q < 2 * i + 2 + kBuf && q < cn; ++q) issue(q);
    }
    pk += cn;
  }
  return true;
}

// b's neighbour-copy ghosts: the valid cells next to each face of every block of levels
// 1..lmax are copied into the facing ghost layer of its same-level neighbour
// (fill_ghost_copy!, src/connectivity.jl:191-213, applied to b; the outer ghost layer
// is not needed).  The reference never reads b's ghosts; the engine keeps them so that
// the GS halo update finds a neighbour's b in the b tile.  One warp per block, lane q
// moving cell q / 2 of faces 2 (q & 1) and 2 (q & 1) + 1; the warps of a CTA keep
// their blocks' loads in flight together.
template <typename T>
__device__ void ph_bghost(const EngArgs<T> &A, int gwarp, int nwarps) {
  const int lane = threadIdx.x & 31;
  const int k = 2 + (lane >> 1);  // position along the face
  for (int l = 1; l <= A.lmax; ++l) {
    const int n = A.tr.nblk[l - 1];
    const int4 *blocks = A.tr.lvl_blocks[l - 1];
    for (int i = gwarp; i < n; i += nwarps) {
      const int X = blocks[i].x;
      const int4 *fc = A.tr.faces + 4 * X;
      const T *xb = A.b + (int64_t)X * kSS;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int f = 2 * (lane & 1) + h;
        const int4 fi = fc[f];
        if (fi.w < 0) continue;
        // the valid cell next to face f and its place in the neighbour's ghost layer
        const int x = f == 0 ? 2 : f == 1 ? 17 : k, y = f <= 1 ? k : f == 2 ? 2 : 17;
        const int gx = f == 0 ? 18 : f == 1 ? 1 : k, gy = f <= 1 ? k : f == 2 ? 18 : 1;
        A.b[(int64_t)fi.w * kSS + gx + kS * gy] = xb[x + kS * y];
      }
    }
  }
}

// ---- mixed-precision outer step (FP64) ---------------------------------------------

// u64 += u (the correction) on every element of every block's tile, ghosts included.
// After a V-cycle the correction's copy and mirror ghosts hold exactly the neighbour
// values and the mirrored values (times 1, -1 or 0) that pushes of the new values would
// write into u64's ghosts, and u64's ghosts hold the same copies of its own values, so
// the sums there equal the pushed ones bit for bit; refinement-boundary ghosts are
// recomputed from the coarse level after the restriction.  A slot takes kUpd blocks per
// pass (levels numbered across so that the work spreads over every slot), thread t < 200
// the element pair 2t, 2t + 1 of each, every load issued before the stores.
constexpr int kUpd = 4;
template <typename T>
__device__ void ph_update64(const EngArgs<T> &A, int t, int gslot, int gstep) {
  if (t >= kSS / 2) return;
  const int e2 = 2 * t;
  int base = 0;
  for (int l = 1; l <= A.lmax; ++l) {
    const int n = A.tr.nblk[l - 1];
    const int4 *blocks = A.tr.lvl_blocks[l - 1];
    for (int i = (gslot - base % gstep + gstep) % gstep; i < n; i += kUpd * gstep) {
      int64_t off[kUpd];
      bool on[kUpd];
#pragma unroll
      for (int k = 0; k < kUpd; ++k) {
        const int ik = i + k * gstep;
        on[k] = false;
        off[k] = 0;
        if (ik < n) {
          const int4 bk = blocks[ik];
          on[k] = !is_frozen(A, item_of(bk));
          off[k] = (int64_t)bk.x * kSS + e2;
        }
      }
      double a0[kUpd], a1[kUpd];
      T c0[kUpd], c1[kUpd];
#pragma unroll
      for (int k = 0; k < kUpd; ++k) {
        a0[k] = a1[k] = 0.0;
        c0[k] = c1[k] = T(0);
        if (on[k]) {
          ld_pair<double>(A.mx.u64 + off[k], a0[k], a1[k]);
          ld_pair<T>(A.u + off[k], c0[k], c1[k]);
        }
      }
#pragma unroll
      for (int k = 0; k < kUpd; ++k)
        if (on[k]) st_pair<double>(A.mx.u64 + off[k], a0[k] + (double)c0[k], a1[k] + (double)c1[k]);
    }
    base += n;
  }
}

// Restriction of u64 from level l onto the covered subblocks of level l - 1, with pushes.
// The four 64-thread quarters of a slot take one child edge each, two rounds per pass
// with every load issued before the stores.
template <typename T>
__device__ void ph_restrict64(const EngArgs<T> &A, int l, int t, int gslot, int gstep, bool all = false) {
  constexpr int R = 2;
  const int n = A.tr.nch[l - 1];
  const int4 *ch = A.tr.lvl_child[l - 1];
  const int quarter = t >> 6, c = t & 63, kx = c & 7, ky = c >> 3;
  for (int i = 4 * gslot + quarter; i < n; i += R * 4 * gstep) {
    int4 e[R];
    bool on[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int ik = i + k * 4 * gstep;
      on[k] = ik < n;
      e[k] = on[k] ? ch[ik] : make_int4(0, 0, 1, 1);
    }
    double v[R];
    int item[R];
    int2 fx[R], fy[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      v[k] = 0.0;
      item[k] = 0;
      fx[k] = fy[k] = make_int2(FACE_NONE, -1);
      if (on[k]) {
        item[k] = A.tr.info[e[k].y].z >> 8;
        v[k] = restrict4<double>(A.mx.u64 + (int64_t)e[k].x * kSS, 2 + 2 * kx, 2 + 2 * ky);
        const int cx = 2 + 8 * (e[k].z - 1) + kx, cy = 2 + 8 * (e[k].w - 1) + ky;
        if (cx <= 3 || cx >= 16) fx[k] = face_tw(A.tr.faces + 4 * e[k].y, cx <= 3 ? 0 : 1);
        if (cy <= 3 || cy >= 16) fy[k] = face_tw(A.tr.faces + 4 * e[k].y, cy <= 3 ? 2 : 3);
      }
    }
#pragma unroll
    for (int k = 0; k < R; ++k) {
      if (!on[k] || (!all && is_frozen(A, item[k]))) continue;
      const int cx = 2 + 8 * (e[k].z - 1) + kx, cy = 2 + 8 * (e[k].w - 1) + ky;
      A.mx.u64[(int64_t)e[k].y * kSS + cx + kS * cy] = v[k];
      push_tw<double>((unsigned)A.it_sgbits[item[k]], A.mx.u64, e[k].y, fx[k], fy[k], cx, cy, v[k]);
    }
  }
}

// The restriction of u64 onto every covered cell whose four children are leaf cells,
// for all levels in one phase: a 64-thread quarter of a slot takes one child edge (of
// any level), each thread one 2 x 2 group of the fine block, skipped when the fine
// block has a child over that group.  It reads only leaf cells, which no thread of the
// phase writes, so the levels need no order.  These are the only covered cells a leaf
// cell's stencil reads (directly, through a neighbour's copy ghost, or through the
// refinement ghosts of a finer block): under the tree's 2:1 nesting a covered cell next
// to a leaf region, or next to a refinement boundary, has leaf children.  So the
// defect of the mixed solve needs only this phase between two defects; the deeper
// covered cells keep stale values until the full chain (ph_restrict64, level by level)
// at the end of the solve makes u64 a composite-grid function again.  The values are
// the chain's own (same order of the four additions), so the iterates do not change.
template <typename T>
__device__ void ph_restrict64_leaf(const EngArgs<T> &A, int t, int gslot, int gstep) {
  const int quarter = t >> 6, c = t & 63, kx = c & 7, ky = c >> 3;
  int total = 0;
  for (int l = 2; l <= A.lmax; ++l) total += A.tr.nch[l - 1];
  for (int i = 4 * gslot + quarter; i < total; i += 4 * gstep) {
    int l = 2, off = i;
    while (off >= A.tr.nch[l - 1]) {
      off -= A.tr.nch[l - 1];
      ++l;
    }
    const int4 e = A.tr.lvl_child[l - 1][off];  // {fine, coarse, sb_r, sb_z}
    const int fsub = (kx >> 2) + 2 * (ky >> 2);
    if ((A.tr.info[e.x].z >> fsub) & 1) continue;  // the fine block has a child over this group
    const int item = A.tr.info[e.y].z >> 8;
    if (is_frozen(A, item)) continue;
    const double v = restrict4<double>(A.mx.u64 + (int64_t)e.x * kSS, 2 + 2 * kx, 2 + 2 * ky);
    const int cx = 2 + 8 * (e.z - 1) + kx, cy = 2 + 8 * (e.w - 1) + ky;
    int2 fx = make_int2(FACE_NONE, -1), fy = make_int2(FACE_NONE, -1);
    if (cx <= 3 || cx >= 16) fx = face_tw(A.tr.faces + 4 * e.y, cx <= 3 ? 0 : 1);
    if (cy <= 3 || cy >= 16) fy = face_tw(A.tr.faces + 4 * e.y, cy <= 3 ? 2 : 3);
    A.mx.u64[(int64_t)e.y * kSS + cx + kS * cy] = v;
    push_tw<double>((unsigned)A.it_sgbits[item], A.mx.u64, e.y, fx, fy, cx, cy, v);
  }
}

// Refinement-boundary ghosts of u64 on level l from level l - 1: the two halves of a slot
// take one block each, two rounds per pass, loads before stores.
template <typename T>
__device__ void ph_refbnd64(const EngArgs<T> &A, int l, int t, int gslot, int gstep, bool all = false) {
  constexpr int R = 2;
  const int n = A.tr.nblk[l - 1];
  const int4 *blocks = A.tr.lvl_blocks[l - 1];
  const int half = t >> 7, q = t & 127;
  for (int i = 2 * gslot + half; i < n; i += R * 2 * gstep) {
    int X[R];
    int4 fi[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int ik = i + k * 2 * gstep;
      X[k] = -1;
      fi[k] = make_int4(FACE_NONE, 0, 0, -1);
      if (ik < n) {
        const int4 bk = blocks[ik];
        if (all || !is_frozen(A, item_of(bk))) {
          X[k] = bk.x;
          fi[k] = A.tr.faces[4 * bk.x + (q >> 5)];
        }
      }
    }
    double v[R];
    int gx[R], gy[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      v[k] = 0.0;
      gx[k] = gy[k] = 0;
      if (X[k] >= 0 && fi[k].x == FACE_REFBND) v[k] = refbnd_val<double>(A.mx.u64, fi[k], q, gx[k], gy[k]);
    }
#pragma unroll
    for (int k = 0; k < R; ++k)
      if (X[k] >= 0 && fi[k].x == FACE_REFBND) A.mx.u64[(int64_t)X[k] * kSS + gx[k] + kS * gy[k]] = v[k];
  }
}

// Leaf sums of squares per norm chunk (up to kNormChunk consecutive blocks of one item
// and level) at bpart[c]: the two halves of the slot take the chunk's blocks j = half,
// half + 2, thread h of a half the cell pair (x0, y), (x0 + 1, y), x0 = 2 + 2 (h % 8),
// y = 2 + h / 8; per thread over its blocks in order, then the warp sums, then the 8 warp
// sums in order.  A leaf cell of level l is weighted by 4^-(l-1); cells under a child
// are skipped (resnorm!, src/multigrid.jl:391-417).
//   defect = false: r = -(b + L u / s_l) of the current iterate u;
//   defect = true : the FP64 defect r = -(b64 + L u64 / s_l) of the mixed solve, also
//                   written as the FP32 right-hand side -r (with its neighbour-copy
//                   ghosts when b's ghosts are kept), with the FP32 correction zeroed
//                   (ghosts included).
// with_b adds the same sums for b (b64 in mixed mode) in bpart_b.  kPer of a half's
// blocks have their loads in flight together (1 in the register-capped 1024-thread
// shape, whose spills would cost more than the overlap).
template <typename T, int kPer>
__device__ void ph_blocknorm(const EngArgs<T> &A, bool defect, bool with_b, int t, int slot, int gslot, int gstep,
                             double *red) {
  const int half = t >> 7, h = t & 127;
  const int x0 = 2 + 2 * (h & 7), y = 2 + (h >> 3), o0 = x0 + kS * y;
  const int mysub = ((x0 - 2) >> 3) + 2 * ((y - 2) >> 3);
  const bool edge = x0 == 2 || x0 == 16 || y <= 3 || y >= 16;
  const int lane = t & 31, w8 = t >> 5;
  int nb = 0;
  for (int c = gslot; c < A.nchunk; c += gstep) {
    const int4 ck = A.chunks[c];  // {level, first, count, item}
    const int item = ck.w;
    if (is_frozen(A, item)) continue;
    const int l = ck.x;
    const int4 *blocks = A.tr.lvl_blocks[l - 1] + ck.y;
    const double wl = 1.0 / (double)((int64_t)1 << (2 * (l - 1)));
    constexpr int kMine = (kNormChunk + 1) / 2;
    static_assert(kMine % kPer == 0, "passes of kPer blocks");
    double v = 0.0, vb = 0.0;
#pragma unroll 1
    for (int p0 = 0; p0 < kMine; p0 += kPer) {
      // kPer of this half's blocks of the chunk: records first, then every block's residual
      // pair (loads of all blocks in flight together: no store in between), then the
      // stores and the sums in order
      int4 bks[kPer];
#pragma unroll
      for (int q = 0; q < kPer; ++q) {
        const int j = 2 * (p0 + q) + half;
        bks[q] = j < ck.z ? blocks[j] : make_int4(0, 0, 0, 0);
      }
      double rr0[kPer], rr1[kPer], bb0[kPer], bb1[kPer];
#pragma unroll
      for (int q = 0; q < kPer; ++q) {
        rr0[q] = rr1[q] = bb0[q] = bb1[q] = 0.0;
        if (2 * (p0 + q) + half >= ck.z) continue;
        const int4 bk = bks[q];
        const int64_t xo = (int64_t)bk.x * kSS + o0;
        if (!defect) {
          const T *par = A.it_par + item * kParStride;
          const T s = par[l], centre = par[32 + l];
          const W5<T> w0 = weights<T>(A.wt, A.geom, bk.y, bk.z, x0, y);
          const W5<T> w1 = weights<T>(A.wt, A.geom, bk.y, bk.z, x0 + 1, y);
          T c0v, c1v, dn0, dn1, up0, up1, b0, b1;
          ld_pair<T>(A.u + xo, c0v, c1v);
          ld_pair<T>(A.u + xo - kS, dn0, dn1);
          ld_pair<T>(A.u + xo + kS, up0, up1);
          ld_pair<T>(A.b + xo, b0, b1);
          const T Lu0 = sten5<T>(w0, centre, dn0, A.u[xo - 1], c0v, c1v, up0);
          const T Lu1 = sten5<T>(w1, centre, dn1, c0v, c1v, A.u[xo + 2], up1);
          rr0[q] = (double)(-(b0 + Lu0 / s));
          rr1[q] = (double)(-(b1 + Lu1 / s));
          bb0[q] = (double)b0;
          bb1[q] = (double)b1;
        } else {
          const double *par = A.mx.it_par64 + item * kParStride;
          const double s = par[l], centre = par[32 + l];
          const W5<double> w0 = weights<double>(A.mx.wt64, A.geom, bk.y, bk.z, x0, y);
          const W5<double> w1 = weights<double>(A.mx.wt64, A.geom, bk.y, bk.z, x0 + 1, y);
          const double *ub = A.mx.u64;
          double c0v, c1v, dn0, dn1, up0, up1;
          ld_pair<double>(ub + xo, c0v, c1v);
          ld_pair<double>(ub + xo - kS, dn0, dn1);
          ld_pair<double>(ub + xo + kS, up0, up1);
          ld_pair<double>(A.mx.b64 + xo, bb0[q], bb1[q]);
          const double Lu0 = sten5<double>(w0, centre, dn0, ub[xo - 1], c0v, c1v, up0);
          const double Lu1 = sten5<double>(w1, centre, dn1, c0v, c1v, ub[xo + 2], up1);
          rr0[q] = -(bb0[q] + Lu0 / s);
          rr1[q] = -(bb1[q] + Lu1 / s);
        }
      }
#pragma unroll
      for (int q = 0; q < kPer; ++q) {
        if (2 * (p0 + q) + half >= ck.z) continue;
        const int4 bk = bks[q];
        const int X = bk.x;
        if (defect) {
          const T v0 = (T)(-rr0[q]), v1 = (T)(-rr1[q]);
          st_pair<T>(A.b + (int64_t)X * kSS + o0, v0, v1);
          if (A.bghost && edge) push_pair<T, false>(0u, A.b, X, A.tr.faces + 4 * X, x0, y, v0, v1);
          float4 *eb = reinterpret_cast<float4 *>(A.u + (int64_t)X * kSS);
          for (int k = h; k < (int)(kSS * sizeof(T) / 16); k += 128) eb[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        if (!((bk.w >> mysub) & 1)) {  // leaf cells
          v = fma(rr0[q], rr0[q], v);
          v = fma(rr1[q], rr1[q], v);
          vb = fma(bb0[q], bb0[q], vb);
          vb = fma(bb1[q], bb1[q], vb);
        }
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

// Per-item norms from the chunk partials, one CTA per item, in a fixed order: sums over
// the item's chunk partials strided by kNormLanes lanes, the warp sums, then the
// kNormLanes / 32 warp sums in order.  Writes the item's record (norm; with `first` |b|
// and the initial norm; V-cycles and steps run) and freezes the item once its norm is
// <= tol * |b| (|b| = 0 counts as 1) or not finite.  Items frozen before are skipped.
constexpr int kNormLanes = 768;  // <= the smaller launch shape
template <typename T>
__device__ void ph_itemnorm(const EngArgs<T> &A, bool first, int cycles, int steps, double *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = blockIdx.x; k < A.nitems; k += gridDim.x) {
    if (A.frozen[k]) continue;
    double v = 0.0, vb = 0.0;
    const int2 rg = A.it_chunks[k];
    // a fixed width of kNormLanes lanes, whatever the CTA size, so that an item's norm
    // has the same rounding in every launch shape (a batch matches its solo solves)
    if (threadIdx.x < kNormLanes)
      for (int j = threadIdx.x; j < rg.y; j += kNormLanes) {
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
      for (int q = 0; q < kNormLanes / 32; ++q) {
        sv += red[q];
        sb += red[32 + q];
      }
      const double nrm = sqrt(sv);
      double *io = A.inorm + kItemRec * k;
      if (first) {
        io[1] = sqrt(sb);
        io[2] = nrm;
      }
      io[0] = nrm;
      // V-cycles run: the launch's count (FP64); in mixed mode the step bookkeeping
      // counts them per item (items may run fewer V-cycles in a step than others)
      if (first || A.mx.u64 == nullptr) io[3] = (double)cycles;
      io[4] = (double)steps;
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
                              double *sol, double *rhs) {
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
    // the level's right-hand side once into shared memory, then every warp four rows of
    // P at a time (four independent accumulators keep more of P's loads in flight);
    // each row sums lane-strided partials, then the warp, in a fixed order
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
      const int c = j & 255;
      rhs[j] = (double)A.b[(int64_t)blocks[j >> 8].x * kSS + (2 + (c & 15)) + kS * (2 + (c >> 4))];
    }
    __syncthreads();
    for (int q0 = 4 * warp; q0 < n; q0 += 4 * nw) {  // n is a multiple of 256: all four rows exist
      const double *pr = P + (int64_t)q0 * n;
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 4
      for (int j = lane; j < n; j += 32) {
        const double bj = rhs[j];
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[r] = fma(pr[(int64_t)r * n + j], bj, acc[r]);
      }
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        double a = acc[r];
        for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
        if (lane == 0) sol[q0 + r] = a;
      }
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

// The direct solve on level 2 of a lone item (<= 4 blocks, n <= 1024 unknowns), spread
// over every CTA in two phases with a grid barrier between them.  First half: every CTA
// forms the level's whole FAS right-hand side in shared memory -- b = -(e + L(u)/s) on
// covered cells (e holds the restricted residual), b itself on leaf cells, as
// ph_direct_top does on level 1 -- and keeps the old u of the rows it will solve.  No
// CTA writes u or e before the barrier, so every one reads the same old values.
template <typename T>
__device__ void ph_direct2_rhs(const EngArgs<T> &A, const T *u, int lt, double *rhs, double *uold) {
  const int2 rg = A.it_lrange[lt - 1];  // item 0
  const int n = 256 * rg.y;
  const int4 *blocks = A.tr.lvl_blocks[lt - 1] + rg.x;
  const T s = A.it_par[lt], centre = A.it_par[32 + lt];
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const int c = j & 255, x = 2 + (c & 15), y = 2 + (c >> 4);
    const int4 bk = blocks[j >> 8];
    const int64_t o = (int64_t)bk.x * kSS + x + kS * y;
    const int mysub = ((x - 2) >> 3) + 2 * ((y - 2) >> 3);
    T bv;
    if ((bk.w >> mysub) & 1) {
      const W5<T> w = weights<T>(A.wt, A.geom, bk.y, bk.z, x, y);
      const T Lu = apply5<T>(u + (int64_t)bk.x * kSS, x, y, w, centre);
      bv = -(A.e[o] + Lu / s);
    } else {
      bv = A.b[o];
    }
    rhs[j] = (double)bv;
  }
  const int rpc = (n + gridDim.x - 1) / gridDim.x, r0 = blockIdx.x * rpc;
  for (int q = threadIdx.x; q < rpc && r0 + q < n; q += blockDim.x) {
    const int j = r0 + q, c = j & 255;
    uold[q] = (double)u[(int64_t)blocks[j >> 8].x * kSS + (2 + (c & 15)) + kS * (2 + (c >> 4))];
  }
}

// Second half: CTA c solves rows [c rpc, (c + 1) rpc) of u = P rhs in FP64, one warp per
// row (lane-strided partial sums, then the warp, in a fixed order), and writes the row's
// new u, the correction e = u - u_old and their ghost pushes in place.
template <typename T>
__device__ void ph_direct2_rows(const EngArgs<T> &A, T *u, int lt, bool make_e, const double *rhs,
                                const double *uold) {
  const int2 rg = A.it_lrange[lt - 1];
  const int n = 256 * rg.y;
  const int4 *blocks = A.tr.lvl_blocks[lt - 1] + rg.x;
  const double *P = A.it_P[0];
  const int rpc = (n + gridDim.x - 1) / gridDim.x, r0 = blockIdx.x * rpc, r1 = min(n, r0 + rpc);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int q = r0 + warp; q < r1; q += nw) {
    const double *pr = P + (int64_t)q * n;
    double acc = 0.0;
    for (int j = lane; j < n; j += 32) acc = fma(pr[j], rhs[j], acc);
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (lane == 0) {
      const int c = q & 255, x = 2 + (c & 15), y = 2 + (c >> 4);
      const int X = blocks[q >> 8].x;
      const int4 *fc = A.tr.faces + 4 * X;
      const T nu = (T)acc;
      u[(int64_t)X * kSS + x + kS * y] = nu;
      push<T>(A, 0, u, X, fc, x, y, nu);
      if (make_e) {
        const T ev = nu - (T)uold[q - r0];
        A.e[(int64_t)X * kSS + x + kS * y] = ev;
        push<T>(A, 0, A.e, X, fc, x, y, ev);
      }
    }
  }
}

// ph_direct2_rows around a split barrier, for grids whose CTAs hold at most one row per
// warp: the CTA counts itself in once its right-hand side reads of level 2 are done,
// forms its rows' products (the same sums in the same order) while the other CTAs
// arrive, and writes them after the wait, so that the products overlap the barrier
// instead of following it.
template <typename T>
__device__ bool ph_direct2_rows_split(const EngArgs<T> &A, T *u, int lt, bool make_e, const double *rhs,
                                      const double *uold, unsigned &epoch) {
  const int2 rg = A.it_lrange[lt - 1];
  const int n = 256 * rg.y;
  const int4 *blocks = A.tr.lvl_blocks[lt - 1] + rg.x;
  const double *P = A.it_P[0];
  const int rpc = (n + gridDim.x - 1) / gridDim.x, r0 = blockIdx.x * rpc, r1 = min(n, r0 + rpc);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = r0 + warp;
  grid_arrive(A.bar, epoch);
  double acc = 0.0;
  if (q < r1) {
    const double *pr = P + (int64_t)q * n;
    for (int j = lane; j < n; j += 32) acc = fma(pr[j], rhs[j], acc);
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  }
  if (!grid_wait(A.bar, A.err, epoch, A.timeout_ns)) return false;
  if (q < r1 && lane == 0) {
    const int c = q & 255, x = 2 + (c & 15), y = 2 + (c >> 4);
    const int X = blocks[q >> 8].x;
    const int4 *fc = A.tr.faces + 4 * X;
    const T nu = (T)acc;
    u[(int64_t)X * kSS + x + kS * y] = nu;
    push<T>(A, 0, u, X, fc, x, y, nu);
    if (make_e) {
      const T ev = nu - (T)uold[q - r0];
      A.e[(int64_t)X * kSS + x + kS * y] = ev;
      push<T>(A, 0, A.e, X, fc, x, y, ev);
    }
  }
  return true;
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

// Threads per CTA of the persistent kernel: 1024 (four 256-thread slots, 64 registers a
// thread) or 768 (three slots, 80 registers).  The wider CTA carries more blocks at a
// time on large levels; the narrower one spills far less, which shortens the latency
// chains that small trees are made of.
constexpr int kEngineWide = 1024, kEngineNarrow = 768;

template <typename T>
constexpr size_t engine_smem_bytes(int threads) {
  return (size_t)(threads / 256) * sizeof(SlotSmem<T>);
}

template <typename T, int NT>
__global__ void __launch_bounds__(NT, 1) k_engine_vcycle(const __grid_constant__ EngArgs<T> A) {
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
  __shared__ int2 s_halo[32];  // the GS halo cells, packed (halo_pack)
  if (threadIdx.x < 32) s_halo[threadIdx.x] = halo_pack(threadIdx.x);
  // the launch-long record cache (single item): level by level from the coarsest, the
  // slot's GS records, then its restriction and prolongation records, while they fit
  if (t == 0)
    for (int l = 0; l < kMaxLev; ++l) {
      S.off_gs[l] = S.off_res[l] = S.off_pro[l] = -1;
      S.cstep[l] = 0;
    }
  slot_sync(slot);
  if (A.nitems == 1) {
    int used = 0;
    for (int l = 1; l <= A.lmax; ++l) {
      const bool loc = l <= A.local_top;
      if (loc && blockIdx.x != 0) continue;
      const int first = loc ? slot : blockIdx.x * nslots + slot, step = loc ? nslots : gridDim.x * nslots;
      if (t == 0) S.cstep[l - 1] = step;
      int n = A.tr.nblk[l - 1];
      int nm = (first < n) ? (n - 1 - first) / step + 1 : 0;
      if (nm > 0 && nm <= kChunk && used + nm <= kRecRows<T>) {
        for (int i = t; i < 5 * nm; i += 256) {
          const int q = i / 5, k = i - 5 * q;
          S.rc[used + q][k] = A.tr.lvl_rec[l - 1][5 * (first + q * step) + k];
        }
        if (t == 0) S.off_gs[l - 1] = (signed char)used;
        used += nm;
      }
      // the child edges of level l (fine at l)
      n = l >= 2 ? A.tr.nch[l - 1] : 0;
      nm = (first < n) ? (n - 1 - first) / step + 1 : 0;
      if (nm > 0 && nm <= kChunk && used + 2 * nm <= kRecRows<T>) {
        for (int i = t; i < 6 * nm; i += 256) {
          const int q = i / 6, k = i - 6 * q;
          const int4 e = A.tr.lvl_child[l - 1][first + q * step];
          S.rc[used + q][k] = k == 0 ? e : k == 1 ? A.tr.info[e.x] : A.tr.faces[4 * e.y + k - 2];
          if (k < 5) S.rc[used + nm + q][k] = k == 0 ? e : A.tr.faces[4 * e.x + k - 1];
        }
        if (t == 0) {
          S.off_res[l - 1] = (signed char)used;
          S.off_pro[l - 1] = (signed char)(used + nm);
        }
        used += 2 * nm;
      }
    }
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
  __shared__ double s_rhs[1024];     // its right-hand side

  auto first_of = [&](bool loc) { return loc ? slot : blockIdx.x * nslots + slot; };
  auto step_of = [&](bool loc) { return loc ? nslots : gridDim.x * nslots; };
  auto stamp = [&]() {
    if (A.trace && cta0 && threadIdx.x == 0 && ntrace < kTraceMax) A.trace[ntrace++] = gtimer();
  };
  // Barrier after a phase: CTA-local when this and the next phase are both local.
  auto sync = [&](bool ok_in, bool cur_loc, bool next_loc) -> bool {
    bool ok = ok_in;
    if (cur_loc && next_loc) {
      if (cta0) {
        asm volatile("fence.proxy.async.global;" ::: "memory");
        __syncthreads();
        asm volatile("fence.proxy.async.global;" ::: "memory");
      }
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
                                step_of(false), t, slot, S, pk, s_halo);
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
  int steps = 0;  // mixed: defect-correction steps run
  auto norm_step = [&](bool defect, bool first, int ncyc) -> bool {
    ph_blocknorm<T, NT == 1024 ? 1 : 2>(A, defect, first, t, slot, gslot, gstep,
                                         reinterpret_cast<double *>(&S.tile[0][0]));
    if (!sync(true, false, false)) return false;
    ph_itemnorm<T>(A, first, ncyc, steps, s_direct);
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
  // Mixed: V-cycles of a defect-correction step, up to A.inner.  An item runs one per
  // decade of its norm / (tol |b|) (a contraction of 0.1 per cycle), so a nearly
  // converged solve runs no extra cycle; the step runs as many as the item furthest from
  // its tolerance needs, and an item that has run its share is paused (frozen = 2) for
  // the rest of the step.  An item's V-cycles are therefore those of its solo solve.
  auto want_cycles = [&](int i) -> int {
    const volatile double *io = A.inorm + kItemRec * i;
    const double bn = io[1] > 0.0 ? io[1] : 1.0;
    const double rho = io[0] / (A.tol * bn);
    int k = 1;
    for (double th = 10.0; k < A.inner && rho > th; th *= 10.0) ++k;
    return k;
  };
  __shared__ int s_inner;
  auto inner_now = [&]() -> int {
    if (threadIdx.x == 0) {
      int kmax = 1;
      for (int i = 0; i < A.nitems; ++i)
        if (*((volatile int *)A.frozen + i) == 0) kmax = max(kmax, want_cycles(i));
      s_inner = min(kmax, max(1, A.inner));
    }
    __syncthreads();
    return s_inner;
  };
  // After V-cycle k (0-based) of a step of nv: count it for every item that ran it, then
  // pause the items whose share is done, or, after the last one, resume them (CTA 0; the
  // caller's grid barrier publishes the flags).
  auto step_books = [&](int k, int nv) {
    if (!(cta0 && threadIdx.x == 0)) return;
    for (int i = 0; i < A.nitems; ++i) {
      volatile int *fz = (volatile int *)A.frozen + i;
      volatile double *io = A.inorm + kItemRec * i;
      if (*fz == 0) io[3] = io[3] + 1.0;
      if (k + 1 < nv) {
        if (*fz == 0 && want_cycles(i) <= k + 1) *fz = 2;
      } else if (*fz == 2) {
        *fz = 0;
      }
    }
  };

  // One FAS V-cycle (src/multigrid.jl:60-106) on the current fields.
  auto vcycle_body = [&]() -> bool {
    cur = 0;
    // descending leg, down to the level above the coarsest one visited
    const int lt = A.top;
    for (int l = L; l >= lt + 1; --l) {
      const bool loc = l <= K;
      for (int it = 0; it < A.ndown; ++it) {
        bool ok = true;
        if (runs(loc))
          ok = ph_gsi<T>(A, l, fld(l), oth(l), nullptr, it == 0 && l < L, false, it == 0 && l < L, first_of(loc),
                         step_of(loc), t, slot, S, pk, s_halo);
        cur ^= 1u << l;
        if (!sync(ok, loc, loc)) return false;
      }
      bool okr = true;
      if (runs(loc)) okr = ph_restrict<T>(A, l, fld(l), fld(l - 1), first_of(loc), step_of(loc), t, slot, S, pk);
      if (!sync(okr, loc, (l - 1) <= K)) return false;
    }
    // coarsest level
    if (A.it_P && lt == 2) {
      // a lone item's direct solve on level 2, grid-wide (never CTA-local: local_top = 0)
      ph_direct2_rhs<T>(A, fld(2), 2, s_rhs, s_direct);
      const int n2 = 256 * A.it_lrange[1].y;
      if ((n2 + (int)gridDim.x - 1) / (int)gridDim.x <= (int)(blockDim.x >> 5)) {
        if (!ph_direct2_rows_split<T>(A, fld(2), 2, L > 2, s_rhs, s_direct, epoch)) return false;
        stamp();
      } else {
        if (!sync(true, false, false)) return false;
        ph_direct2_rows<T>(A, fld(2), 2, L > 2, s_rhs, s_direct);
      }
      if (!sync(true, false, false)) return false;
    } else if (A.it_P) {
      const bool loc = 1 <= K;
      if (runs(loc))
        ph_direct_top<T>(A, fld(1), L > 1, loc ? 0 : blockIdx.x, loc ? 1 : gridDim.x, t, slot, s_direct, s_rhs);
      if (!sync(true, loc, 2 <= K || L < 2)) return false;
    } else {
      const bool loc = 1 <= K;
      for (int it = 0; it < A.ntop; ++it) {
        const bool last = it == A.ntop - 1;
        bool ok = true;
        if (runs(loc))
          ok = ph_gsi<T>(A, 1, fld(1), oth(1), nullptr, it == 0 && L > 1, last && L > 1, it == 0 && L > 1,
                         first_of(loc), step_of(loc), t, slot, S, pk, s_halo);
        cur ^= 1u << 1;
        if (!sync(ok, loc, last ? (2 <= K || L < 2) : loc)) return false;
      }
    }
    // ascending leg
    for (int l = lt + 1; l <= L; ++l) {
      const bool loc = l <= K;
      bool okp = true;
      if (runs(loc)) okp = ph_prolong<T>(A, l, fld(l), fld(l - 1), first_of(loc), step_of(loc), t, slot, S, pk);
      if (!sync(okp, loc, loc)) return false;
      for (int it = 0; it < A.nup; ++it) {
        const bool last = it == A.nup - 1;
        bool ok = true;
        if (runs(loc))
          ok = ph_gsi<T>(A, l, fld(l), oth(l), A.e, false, last && l < L, false, first_of(loc), step_of(loc), t,
                         slot, S, pk, s_halo);
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
  if (A.bghost && !mixed) {
    ph_bghost<T>(A, blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), gridDim.x * (blockDim.x >> 5));
    if (!sync(true, false, false)) return;
  }
  if (loop && !mixed && !norm_step(false, true, 0)) return;
  for (int iter = 0;; ++iter) {
    if (loop && mixed) {
      // FP64 side of a defect-correction step
      if (A.mx.apply_update || iter > 0) {
        ph_update64<T>(A, t, gslot, gstep);
        if (!sync(true, false, false)) return;
      }
      if (L >= 2) {
        ph_restrict64_leaf<T>(A, t, gslot, gstep);
        if (!sync(true, false, false)) return;
      }
      for (int l = 2; l <= L; ++l)
        if ((A.mx.refbnd_levels >> l) & 1) {
          ph_refbnd64<T>(A, l, t, gslot, gstep);
          if (!sync(true, false, false)) return;
        }
      if (!norm_step(true, iter == 0, cycles)) return;
    }
    if (loop && (!any_live() || cycles >= A.max_cycles)) {
      if (mixed) {
        // u64 a composite-grid function of its leaves again, every item: the full
        // restriction chain, level by level, and the refinement ghosts
        for (int l = L; l >= 2; --l) {
          ph_restrict64<T>(A, l, t, gslot, gstep, true);
          if (!sync(true, false, false)) return;
        }
        for (int l = 2; l <= L; ++l)
          if ((A.mx.refbnd_levels >> l) & 1) {
            ph_refbnd64<T>(A, l, t, gslot, gstep, true);
            if (!sync(true, false, false)) return;
          }
      }
      break;
    }
    // mixed: up to A.inner FP32 V-cycles on the same defect, the correction carried over
    const int nv = (mixed && loop) ? inner_now() : 1;
    for (int k = 0; k < nv; ++k) {
      if (!vcycle_body()) return;
      cycles++;
      if (mixed && loop) {
        step_books(k, nv);
        // a lone item is never paused inside its step (nv is its own share), and CTA 0,
        // which wrote the books, is the one that reads them: no barrier needed
        if (A.nitems > 1 && !sync(true, false, false)) return;
      }
    }
    if (mixed) steps++;
    if (!loop) break;
    if (!mixed && !norm_step(false, false, cycles)) return;
  }
  if (loop && A.out && cta0 && threadIdx.x == 0) A.out[0] = (double)cycles;
  if (A.trace && cta0 && threadIdx.x == 0 && ntrace < kTraceMax) A.trace[ntrace] = 0;
}

}  // namespace srmg
