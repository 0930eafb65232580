// srmg_internal.h -- internal helpers shared by the library's translation units.
#pragma once
#include <initializer_list>
#include <vector>

#include "srmg_ctx.h"

namespace srmg {

int fail(srmg_ctx *c, int code, const char *fmt, ...);
int cuda_check(srmg_ctx *c, cudaError_t e, const char *what);
int ensure(srmg_ctx *ctx, DevBuf &b, size_t bytes);
int check_call(srmg_ctx *ctx, int64_t nblk_alloc, int op, int geom, const int8_t *bc);
// check_call for the entry points that also run on three-dimensional trees (3^D-entry
// boundary table, Cartesian geometry there); check_call refuses D = 3 contexts.
int check_call_any(srmg_ctx *ctx, int64_t nblk_alloc, int op, int geom, const int8_t *bc);
// values per block of the context's fields: 20^D
inline int64_t block_elems(const srmg_ctx *ctx) { return ctx->D == 3 ? (int64_t)kS * kS * kS : (int64_t)kSS; }
void free_tree(srmg_ctx *ctx);
// Builds the Gauss-Seidel push tables of the context's tree once (not while the stream
// is capturing or a sequence is recorded): push_state becomes 1 or -1.  On octrees only
// where the sweeps of operator `op` do not push by rule (BoxStencil{3} or order 4).
int ensure_gs_push(srmg_ctx *ctx, int op);
int d3_ensure_push(srmg_ctx *ctx);
void drop_op_graphs(srmg_ctx *ctx);
// One cooperative launch of the sequencer over `nops` recorded operations (srmg_seq.cu).
int seq_launch(srmg_ctx *ctx, const void *d_ops, int nops);
size_t seq_op_bytes();
// The same for three-dimensional trees (srmg3.cu).
int seq_launch3(srmg_ctx *ctx, const void *d_ops, int nops);
size_t seq3_op_bytes();
// `ncycles` per-operation FP64 V-cycles (2D trees off the persistent engine, or 3D),
// replayed from a captured CUDA graph when the option `op_graphs` is on (default).
int vcycle_ops(srmg_ctx *ctx, double *u, double *b, double *r, double *u1, double s, int op, double k2, int geom,
               const int8_t *bc, int lmax, int ndown, int ntop, int nup, double omega, int ncycles);
// the D = 3 bodies of the generic entry points (srmg3.cu)
int d3_fill_ghost(srmg_ctx *ctx, double *u, int level, const int8_t *bc, int mask);
int d3_gs_level(srmg_ctx *ctx, double *u, const double *b, int level, double omega, double sl, int op, double k2,
                int colour);
int d3_gs_iter(srmg_ctx *ctx, double *u, const double *b, int level, double omega, double sl, int n, int op, double k2,
               const int8_t *bc);
int d3_residual_level(srmg_ctx *ctx, double *r, const double *u, const double *b, int level, double sl, int op,
                      double k2);
int d3_restrict_level(srmg_ctx *ctx, double *u, int level);
int d3_interp_add_level(srmg_ctx *ctx, double *u, const double *u1, int level);
int d3_postrestrict_level(srmg_ctx *ctx, double *b, const double *u, const double *r, int level, double s, int op,
                          double k2);
int d3_rhs_level(srmg_ctx *ctx, double *q1, const double *q, int level, int op);
int d3_vcycle(srmg_ctx *ctx, double *u, double *b, double *r, double *u1, double s, int op, double k2,
              const int8_t *bc, int lmax, int ndown, int ntop, int nup, double omega);
int d3_fmg(srmg_ctx *ctx, double *u, double *b, double *r, double *u1, double s, int op, double k2, const int8_t *bc,
           int ndown, int ntop, int nup, double omega);
int d3_leafnorm(srmg_ctx *ctx, const double *u, const double *b, double s, int op, double k2, int mode, int slot);
int d3_solve(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, double s, int op, double k2,
             const int8_t *bc, const srmg_solve_opts *o, srmg_stats *st);
Signs make_signs(const int8_t *bc);
std::vector<int8_t> bc_of(const Signs &sg);
int build_tree(srmg_ctx *ctx, int nlev, const int64_t *npairs, const srmg_pair *const *pairs,
               const int64_t *nnb, const srmg_neighbor *const *nb, const int64_t *nbd,
               const srmg_boundary *const *bd, const int64_t *nrb, const srmg_refbnd *const *rb,
               const int64_t *nch, const srmg_child *const *ch, uint64_t generation,
               const std::vector<int> *item_of, int nitems);
double level_scale(double s, int l);

template <typename T>
OpParams<T> op_params(int op, int geom, double k2, double sl, double omega);

template <typename T> int L_fill_ghost(srmg_ctx *ctx, T *u, int l, const Signs &sg, int mask);
template <typename T> int L_gs_colour(srmg_ctx *ctx, T *u, const T *b, int l, const OpParams<T> &p, int parity);
template <typename T> int L_gs_iter(srmg_ctx *ctx, T *u, const T *b, int l, const OpParams<T> &p, int n, const Signs &sg);
template <typename T> int L_residual(srmg_ctx *ctx, T *r, const T *u, const T *b, int l, const OpParams<T> &p);
template <typename T> int L_postrestrict(srmg_ctx *ctx, T *bf, const T *u, const T *r, int l, const OpParams<T> &pc);
template <typename T> int L_restrict(srmg_ctx *ctx, T *u, int l);
template <typename T> int L_interp_add(srmg_ctx *ctx, T *u, const T *u1, int l);
template <typename T> int L_copy(srmg_ctx *ctx, T *dst, const T *src, int l);
template <typename T> int L_diff(srmg_ctx *ctx, T *dst, const T *a1, const T *a2, int l);

template <typename T>
int vcycle_dev(srmg_ctx *ctx, T *u, T *b, T *r, T *u1, double s, int op, double k2, int geom,
               const Signs &sg, int lmax, int ndown, int ntop, int nup, double omega);
template <typename T>
int leafnorm_dev(srmg_ctx *ctx, const T *u, const T *b, double s, int op, double k2, int geom,
                 int mode, int slot);
int read_small(srmg_ctx *ctx, int n);

int engine_local_top(srmg_ctx *ctx, int lmax);

// Device tables of the items' operators, uploaded by prepare_items.
struct ItemTabs {
  const double *par64 = nullptr;     // per item kParStride FP64 values
  const float *par32 = nullptr;      // per item kParStride FP32 values
  const int *sgbits = nullptr;       // per item: boundary table, entry k as (bc_k + 1) << 2k
  const double *const *P = nullptr;  // per item direct coarsest-level inverse, or null
  const double *P0 = nullptr;        // item 0's inverse (per-operation kernels)
  int n0 = 0;                        // its unknowns
  int top = 1;                       // the level the inverses belong to (1, or 2 for a lone tree)
};
// Upload the per-item tables for operators `specs` (ctx->nitems entries).  With
// smooth_level > 0 the level's entries use the scale smooth_sl instead of s_l.  With
// want_P the direct-solve inverse of every item on level `top` is prepared (cached);
// with top = 2 and no usable level-2 inverse it falls back to level 1; tabs->P stays
// null when some item's level has more than 4 blocks, a face without a ghost source on
// that level, or a singular operator.
int prepare_items(srmg_ctx *ctx, const ItemSpec *specs, int geom, double omega, bool want_P,
                  int smooth_level, double smooth_sl, ItemTabs *tabs, int top = 1);
// The level of the persistent engine's direct solve for this context: 2 for a lone
// two-dimensional tree whose level 2 holds 1..4 blocks (option "direct_level" not 1),
// else 1.
int direct_top(srmg_ctx *ctx);
// The same operator for every item.
std::vector<ItemSpec> uniform_items(srmg_ctx *ctx, double s, int op, double k2, const int8_t *bc);

// Optional parts of a persistent-engine launch.
struct EngineRun {
  bool direct = false;               // FP64 direct solve of the coarsest level (tabs.P)
  double *u64 = nullptr;             // mixed precision: FP64 iterate and right-hand side
  const double *b64 = nullptr;
  int apply_update = 0;
  int inner = 1;                     // mixed: FP32 V-cycles per defect-correction step
  int max_cycles = 0;                // > 0: device-side loop until every item has converged
  double tol = 0.0;                  // relative to each item's leaf norm of b
};
template <typename T>
int engine_vcycle(srmg_ctx *ctx, T *u, T *b, T *u1, T *e, const ItemTabs &tabs, int geom, int lmax,
                  int ndown, int ntop, int nup, const EngineRun *run = nullptr);
int engine_check(srmg_ctx *ctx);
template <typename T>
int engine_smooth(srmg_ctx *ctx, T *u, const T *b, const ItemTabs &tabs, int geom, int level, int n);
// Copy the per-item results of the last device loop ({norm, |b|, initial, cycles} per
// item, kItemRec values each, then the launch's V-cycle count) to ctx->h_items and
// check the error word.
int read_items(srmg_ctx *ctx);
int items_host_reserve(srmg_ctx *ctx);  // the pinned mirror (read_items calls it)
int items_d2h(srmg_ctx *ctx);           // the copy alone, stream-ordered
bool engine_ok(srmg_ctx *ctx, const srmg_solve_opts *o, std::initializer_list<const void *> ptrs);
int solve_reserve(srmg_ctx *ctx, int64_t nblk_alloc, int mode);
int solve_enqueue(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, const ItemTabs &tabs, int geom,
                  const srmg_solve_opts *o);
void items_stats(srmg_ctx *ctx, const srmg_solve_opts *o, srmg_stats *st);
// Tolerance-driven solve of every item of the context (statistics per item in st).
int solve_items(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, const ItemSpec *specs,
                int geom, const srmg_solve_opts *opts, srmg_stats *st);
int stage_in(srmg_ctx *ctx, int slot, const double *h, int64_t nblk_alloc, double **d);
int stage_out(srmg_ctx *ctx, double *h, const double *d, int64_t nblk_alloc);

}  // namespace srmg
