// srmg_internal.h -- internal helpers shared by the library's translation units.
#pragma once
#include "srmg_ctx.h"

namespace srmg {

int fail(srmg_ctx *c, int code, const char *fmt, ...);
int cuda_check(srmg_ctx *c, cudaError_t e, const char *what);
int ensure(srmg_ctx *ctx, DevBuf &b, size_t bytes);
int check_call(srmg_ctx *ctx, int64_t nblk_alloc, int op, int geom, const int8_t *bc);
Signs make_signs(const int8_t *bc);
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
// Optional parts of a persistent-engine launch.
struct EngineRun {
  const double *coarse_P = nullptr;  // FP64 direct solve of the coarsest level
  int coarse_n = 0;
  double *u64 = nullptr;             // mixed precision: FP64 iterate and right-hand side
  const double *b64 = nullptr;
  int apply_update = 0;
  int max_cycles = 0;                // > 0: device-side loop until the norm <= tol_abs
  double tol_abs = 0.0;
};
template <typename T>
int engine_vcycle(srmg_ctx *ctx, T *u, T *b, T *u1, T *e, double s, int op, double k2, int geom,
                  const Signs &sg, int lmax, int ndown, int ntop, int nup, double omega,
                  const EngineRun *run = nullptr);
int engine_check(srmg_ctx *ctx);
template <typename T>
int engine_smooth(srmg_ctx *ctx, T *u, const T *b, int level, double omega, double sl, int n, int op,
                  double k2, int geom, const Signs &sg);
int stage_in(srmg_ctx *ctx, int slot, const double *h, int64_t nblk_alloc, double **d);
int stage_out(srmg_ctx *ctx, double *h, const double *d, int64_t nblk_alloc);

}  // namespace srmg
