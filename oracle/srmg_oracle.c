/*
 * srmg_oracle.c -- CPU FP64 restatement of Steamroller.jl's FAS multigrid field solve.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle).  Loaded by tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / reference legs; never by the product library.
 *
 * Parity: UNPINNED -- the reference ships no tests or golden vectors and its Julia
 * toolchain is absent here; see srmg_oracle.h.
 *
 * Every routine restates one reference routine (file:line given), keeping its
 * operation order.  Julia does not contract a*b+c into an FMA unless asked
 * (@fastmath / muladd), so this file is compiled with -ffp-contract=off and uses
 * fma() exactly where the reference calls muladd.  OpenMP parallel loops stand in
 * for Polyester's @batch; every parallel loop writes disjoint data, as @batch does.
 */
#include "srmg_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Linear offset of 1-based (i, j) in 1-based block blk (src/blockfield.jl:148,223-227). */
static inline int64_t IX(int S, int i, int j, int64_t blk) {
    return (int64_t)(i - 1) + (int64_t)S * (j - 1) + (int64_t)S * S * (blk - 1);
}

void orc_tree_index(orc_tree *t) {
    for (int64_t k = 0; k < 2 * t->nblk_alloc; k++) t->coord_of[k] = -1;
    for (int l = 0; l < t->nlev; l++)
        for (int64_t p = 0; p < t->npairs[l]; p++) {
            const orc_pair *pr = &t->pairs[l][p];
            t->coord_of[2 * (pr->blk - 1)] = pr->coord[0];
            t->coord_of[2 * (pr->blk - 1) + 1] = pr->coord[1];
        }
}

/* ---- ghost fills -------------------------------------------------------------- */

/* _fill_ghost_copy! (src/connectivity.jl:184-198). */
static void copy_edge(double *u, int M, int G, const orc_neighbor *e) {
    const int S = M + 2 * G;
    const int64_t f[2] = {e->face[0], e->face[1]};
    int n[2];
    for (int d = 0; d < 2; d++) n[d] = (f[d] == 0) ? M : G;
    for (int i2 = 1; i2 <= n[1]; i2++)
        for (int i1 = 1; i1 <= n[0]; i1++) {
            int i[2] = {i1, i2}, from[2], to[2];
            for (int d = 0; d < 2; d++) {
                from[d] = f[d] == 0 ? G + i[d] : (f[d] == -1 ? i[d] + G : i[d] + M);
                to[d] = f[d] == 0 ? G + i[d] : (f[d] == 1 ? i[d] : i[d] + M + G);
            }
            u[IX(S, to[0], to[1], e->to)] = u[IX(S, from[0], from[1], e->from)];
        }
}

void orc_fill_ghost_copy(double *u, const orc_tree *t, int l) {
    const orc_neighbor *v = t->nb[l - 1];
    const int64_t n = t->nnb[l - 1];
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) copy_edge(u, t->M, t->G, &v[k]);
}

/* ghostrange (src/blockfield.jl:470-472) and validrange (:475-477), 1-based bounds. */
static void ghost_bounds(int M, int G, int64_t face, int *lo, int *hi) {
    if (face == 0) { *lo = G + 1; *hi = G + M; }
    else if (face == -1) { *lo = 1; *hi = G; }
    else { *lo = M + G + 1; *hi = M + 2 * G; }
}

/* mirrorghost (src/blockfield.jl:513-521). */
static inline int mirror(int M, int G, int i, int64_t dir) {
    if (dir == -1) return 2 * G - i + 1;
    if (dir == 1) return 2 * (G + M) - i + 1;
    return i;
}

/* fill_ghost_bnd! (src/connectivity.jl:217-231) with getbc (src/boundary.jl:45-47):
 * ghost = a[2+bnd1, 2+bnd2] * mirror(valid); the 3x3 Int8 table is column-major. */
void orc_fill_ghost_bnd(double *u, const orc_tree *t, int l, const int8_t bc[9]) {
    const orc_boundary *v = t->bd[l - 1];
    const int64_t n = t->nbd[l - 1];
    const int M = t->M, G = t->G, S = M + 2 * G;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) {
        const orc_boundary *e = &v[k];
        int lo[2], hi[2];
        for (int d = 0; d < 2; d++) ghost_bounds(M, G, e->face[d], &lo[d], &hi[d]);
        const double a = (double)bc[(1 + e->bnd[0]) + 3 * (1 + e->bnd[1])];
        for (int j = lo[1]; j <= hi[1]; j++)
            for (int i = lo[0]; i <= hi[0]; i++) {
                int vi = mirror(M, G, i, e->bnd[0]), vj = mirror(M, G, j, e->bnd[1]);
                u[IX(S, i, j, e->block)] = a * u[IX(S, vi, vj, e->block)];
            }
    }
}

/* interp!(InterpLinear, ...) (src/interp.jl:24-63) with weights __w0 = 1/2, __w1 = 1/4
 * (:7-8).  dest/src are blocks; idest/isrc are 1-based rectangles [lo, hi].  When add
 * is set the result is f + dest, i.e. func = + (interp_add_level!, :107-115). */
static void interp_linear(double *dest, const int dlo[2], const double *src, const int slo[2],
                          const int shi[2], int S, int add) {
    for (int k2 = 0; k2 <= shi[1] - slo[1]; k2++)
        for (int k1 = 0; k1 <= shi[0] - slo[0]; k1++) {
            const int jd0[2] = {dlo[0] + 2 * k1, dlo[1] + 2 * k2};
            const int js[2] = {slo[0] + k1, slo[1] + k2};
            for (int i2 = 0; i2 <= 1; i2++)
                for (int i1 = 0; i1 <= 1; i1++) {
                    const int jd[2] = {jd0[0] + i1, jd0[1] + i2};
                    double f = 0.5 * src[IX(S, js[0], js[1], 1)];
                    f += 0.25 * src[IX(S, js[0] + 2 * i1 - 1, js[1], 1)];
                    f += 0.25 * src[IX(S, js[0], js[1] + 2 * i2 - 1, 1)];
                    double *dp = &dest[IX(S, jd[0], jd[1], 1)];
                    *dp = add ? (f + *dp) : f;
                }
        }
}

/* subblockindices (src/blockfield.jl:407-412). */
static void subblock_bounds(int M, int G, int64_t sb, int *lo, int *hi) {
    const int mh = M / 2;
    *lo = G + 1 + (int)(sb - 1) * mh;
    *hi = G + (int)sb * mh;
}

/* fill_ghost_interp! (src/connectivity.jl:251-258): fine ghosts at face from the
 * coarse parent's subblockbnd(subblock, -face) (src/blockfield.jl:416-434). */
void orc_fill_ghost_interp(double *u, const orc_tree *t, int l) {
    const orc_refbnd *v = t->rb[l - 1];
    const int64_t n = t->nrb[l - 1];
    const int M = t->M, G = t->G, S = M + 2 * G, gh = G / 2;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) {
        const orc_refbnd *e = &v[k];
        int dlo[2], dhi[2], slo[2], shi[2];
        for (int d = 0; d < 2; d++) {
            ghost_bounds(M, G, e->face[d], &dlo[d], &dhi[d]);
            int lo, hi;
            subblock_bounds(M, G, e->subblock[d], &lo, &hi);
            const int64_t mf = -e->face[d];
            if (mf == -1) { slo[d] = lo; shi[d] = lo + gh - 1; }
            else if (mf == 1) { slo[d] = hi - gh + 1; shi[d] = hi; }
            else { slo[d] = lo; shi[d] = hi; }
        }
        (void)dhi;
        interp_linear(u + (int64_t)S * S * (e->fine - 1), dlo,
                      u + (int64_t)S * S * (e->coarse - 1), slo, shi, S, 0);
    }
}

/* fill_ghost! (src/connectivity.jl:155-159): copy, then boundary, then interp. */
void orc_fill_ghost(double *u, const orc_tree *t, int l, const int8_t bc[9]) {
    orc_fill_ghost_copy(u, t, l);
    orc_fill_ghost_bnd(u, t, l, bc);
    orc_fill_ghost_interp(u, t, l);
}

/* ---- transfers -------------------------------------------------------------- */

/* restrict! (src/restrict.jl:5-25) over restrict_level! (:31-37): coarse cell =
 * (((0 + f00) + f10) + f01) + f11) / 4, i_1 innermost (Base.Cartesian @nloops). */
void orc_restrict_level(double *u, const orc_tree *t, int l) {
    const orc_child *v = t->ch[l - 1];
    const int64_t n = t->nch[l - 1];
    const int M = t->M, G = t->G, S = M + 2 * G, mh = M / 2;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) {
        const orc_child *e = &v[k];
        const double *src = u + (int64_t)S * S * (e->fine - 1);
        double *dst = u + (int64_t)S * S * (e->coarse - 1);
        int dlo[2], dhi[2];
        for (int d = 0; d < 2; d++) subblock_bounds(M, G, e->subblock[d], &dlo[d], &dhi[d]);
        for (int k2 = 1; k2 <= mh; k2++)
            for (int k1 = 1; k1 <= mh; k1++) {
                const int js0 = G + 2 * k1 - 1, js1 = G + 2 * k2 - 1;
                double f = 0.0;
                for (int i2 = 0; i2 <= 1; i2++)
                    for (int i1 = 0; i1 <= 1; i1++) f += src[IX(S, js0 + i1, js1 + i2, 1)];
                dst[IX(S, dlo[0] + k1 - 1, dlo[1] + k2 - 1, 1)] = f / 4;
            }
    }
}

/* restrict_full! (src/restrict.jl:43-47). */
void orc_restrict_full(double *u, const orc_tree *t) {
    for (int l = t->nlev; l >= 1; l--) orc_restrict_level(u, t, l);
}

/* interp_add_level! (src/interp.jl:107-115): u[fine, valid] += P(u1[coarse, subblock]). */
void orc_interp_add_level(double *u, const double *u1, const orc_tree *t, int l) {
    const orc_child *v = t->ch[l - 1];
    const int64_t n = t->nch[l - 1];
    const int M = t->M, G = t->G, S = M + 2 * G;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) {
        const orc_child *e = &v[k];
        int slo[2], shi[2];
        for (int d = 0; d < 2; d++) subblock_bounds(M, G, e->subblock[d], &slo[d], &shi[d]);
        const int dlo[2] = {G + 1, G + 1};
        interp_linear(u + (int64_t)S * S * (e->fine - 1), dlo,
                      u1 + (int64_t)S * S * (e->coarse - 1), slo, shi, S, 1);
    }
}

/* copyto! / diffto! over a layer (src/blockfield.jl:557-576): whole blocks, ghosts included. */
void orc_copyto_level(double *dst, const double *src, const orc_tree *t, int l) {
    const int S = t->M + 2 * t->G;
    const orc_pair *p = t->pairs[l - 1];
    const int64_t n = t->npairs[l - 1];
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) {
        const int64_t off = (int64_t)S * S * (p[k].blk - 1);
        memcpy(dst + off, src + off, sizeof(double) * S * S);
    }
}

void orc_diffto_level(double *dst, const double *a1, const double *a2, const orc_tree *t, int l) {
    const int S = t->M + 2 * t->G;
    const orc_pair *p = t->pairs[l - 1];
    const int64_t n = t->npairs[l - 1];
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) {
        const int64_t off = (int64_t)S * S * (p[k].blk - 1);
        for (int q = 0; q < S * S; q++) dst[off + q] = a1[off + q] - a2[off + q];
    }
}

/* ---- stencils --------------------------------------------------------------- */

/* applystencil, order-2, 2D (src/laplacian.jl:78-128, src/helmholtz.jl:17-67).
 * @stencil (src/laplacian.jl:25-49) walks the 3x3 literal column-major, skipping
 * literal zeros, and accumulates v = 0; v += c * u[I + S] in that order:
 * (0,-1), (-1,0), (0,0), (+1,0), (0,+1).  The cylindrical weights are
 * (2i-2)/(2i-1) and 2i/(2i-1) with i the 1-based global cell index along the radial
 * dimension; the centre is -4 (Laplacian) or -4 - s*k2 (Helmholtz). */
typedef struct { double wzm, wrm, cc, wrp, wzp; } stencil5;

static inline void weights(const orc_operator *op, double s, int64_t iglob_r, int64_t iglob_z,
                           stencil5 *w) {
    w->wzm = w->wrm = w->wrp = w->wzp = 1.0;
    w->cc = (op->op == 1) ? (-4.0 - s * op->k2) : -4.0;
    if (op->geom == 1) {
        const int64_t i = iglob_r;
        w->wrm = (double)(2 * i - 2) / (double)(2 * i - 1);
        w->wrp = (double)(2 * i) / (double)(2 * i - 1);
    } else if (op->geom == 2) {
        const int64_t i = iglob_z;
        w->wzm = (double)(2 * i - 2) / (double)(2 * i - 1);
        w->wzp = (double)(2 * i) / (double)(2 * i - 1);
    }
}

static inline double apply5(const double *ub, int S, int i, int j, const stencil5 *w) {
    double v = 0.0;
    v += w->wzm * ub[IX(S, i, j - 1, 1)];
    v += w->wrm * ub[IX(S, i - 1, j, 1)];
    v += w->cc * ub[IX(S, i, j, 1)];
    v += w->wrp * ub[IX(S, i + 1, j, 1)];
    v += w->wzp * ub[IX(S, i, j + 1, 1)];
    return v;
}

/* diagelm (src/laplacian.jl:94-95,127-128; src/helmholtz.jl:34-35,66-67). */
static inline double diagelm(const orc_operator *op, double s) {
    return (op->op == 1) ? (-4 - s * op->k2) : -4.0;
}

/* ---- order-4 compact discretisation, LaplacianDiscretization{2,4} ------------------
 * applystencil (src/laplacian.jl:133-202): @stencil over a 3x3 literal whose rows are
 * offsets along dimension 1 and columns along dimension 2, walked column-major, so the
 * coefficient k = (d1 + 1) + 3 (d2 + 1) is accumulated k = 0..8 (v = 0; v += c_k u),
 * then divided by 6.  Cylindrical coefficients are integer polynomials of the 1-based
 * global index i along the radial dimension, divided as Float64 (Int / Int). */
static void coeffs9(int geom, int64_t ir, int64_t iz, double c[9]) {
    if (geom == 0) {
        static const double cart[9] = {1, 4, 1, 4, -20, 4, 1, 4, 1};
        for (int k = 0; k < 9; k++) c[k] = cart[k];
        return;
    }
    const int64_t i = (geom == 1) ? ir : iz;
    const double am = (double)(2 * (i - 1)) / (double)(2 * i - 1);   /* 2(i-1)/(2i-1) */
    const double ap = (double)(2 * i) / (double)(2 * i - 1);         /* 2i/(2i-1) */
    const int64_t q = 2 * i - 1;
    const int64_t p1 = -2 + 9 * i - 16 * i * i + 8 * i * i * i;
    const int64_t p2 = 1 - 5 * i + 5 * i * i;
    const int64_t p3 = 1 + i - 8 * i * i + 8 * i * i * i;
    const double em = (double)(4 * p1) / (double)(q * q * q);        /* radial -1 neighbour */
    const double cc = (double)(-16 * p2) / (double)((1 - 2 * i) * (1 - 2 * i));
    const double ep = (double)(4 * p3) / (double)(q * q * q);        /* radial +1 neighbour */
    if (geom == 1) {  /* r = dimension 1 (src/laplacian.jl:156-164) */
        const double v[9] = {am, 4, ap, em, cc, ep, am, 4, ap};
        for (int k = 0; k < 9; k++) c[k] = v[k];
    } else {          /* r = dimension 2 (src/laplacian.jl:176-184) */
        const double v[9] = {am, em, am, 4, cc, 4, ap, ep, ap};
        for (int k = 0; k < 9; k++) c[k] = v[k];
    }
}

static inline double apply9(const double *ub, int S, int i, int j, const double c[9]) {
    double v = 0.0;
    for (int d2 = -1; d2 <= 1; d2++)
        for (int d1 = -1; d1 <= 1; d1++) v += c[(d1 + 1) + 3 * (d2 + 1)] * ub[IX(S, i + d1, j + d2, 1)];
    return v / 6;
}

/* diagelm for order 4 (src/laplacian.jl:150-151, 205-209): -20/6, or
 * -16 (1 - 5i + 5i^2) / (1 - 2i)^2 / 6 with i the radial global index. */
static inline double diagelm4(int geom, int64_t ir, int64_t iz) {
    if (geom == 0) return -20.0 / 6.0;
    const int64_t i = (geom == 1) ? ir : iz;
    return (double)(-16 * (1 - 5 * i + 5 * i * i)) / (double)((1 - 2 * i) * (1 - 2 * i)) / 6;
}

/* The :lhs stencil of any supported discretisation at 1-based (i, j) with global
 * indices (J1, J2), scale s. */
static inline double lhs_apply(const orc_operator *op, double s, const double *ub, int S, int i, int j,
                               int64_t J1, int64_t J2) {
    if (op->op == 2) {
        double c[9];
        coeffs9(op->geom, J1, J2, c);
        return apply9(ub, S, i, j, c);
    }
    stencil5 w;
    weights(op, s, J1, J2, &w);
    return apply5(ub, S, i, j, &w);
}

/* gauss_seidel!(..., RedBlack{P}) (src/multigrid.jl:153-180) on every block of level l
 * (gauss_seidel_level!, :238-243).  Colour P updates the cells whose 1-based local
 * indices satisfy (I1 - G - 1) % 2 == P xor (I2 & 1). */
void orc_gs_level(double *u, const double *b, double omega, double s, const orc_tree *t, int l,
                  const orc_operator *op, int parity) {
    const int M = t->M, G = t->G, S = M + 2 * G;
    const orc_pair *p = t->pairs[l - 1];
    const int64_t n = t->npairs[l - 1];
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) {
        const int64_t blk = p[k].blk;
        const int64_t g0r = (int64_t)M * (p[k].coord[0] - 1) + 1;  /* global_first, mesh.jl:76-78 */
        const int64_t g0z = (int64_t)M * (p[k].coord[1] - 1) + 1;
        double *ub = u + (int64_t)S * S * (blk - 1);
        const double *bb = b + (int64_t)S * S * (blk - 1);
        for (int i2 = G + 1; i2 <= G + M; i2++)
            for (int i1 = G + 1; i1 <= G + M; i1 += 2) {
                const int pp = parity ^ (i2 & 1);
                const int I1 = i1 + pp, I2 = i2;
                const int64_t J1 = I1 - G + g0r - 1, J2 = I2 - G + g0z - 1;
                stencil5 w;
                weights(op, s, J1, J2, &w);
                const double c = diagelm(op, s);
                const double Lu = apply5(ub, S, I1, I2, &w);
                const double v = fma(s, bb[IX(S, I1, I2, 1)], Lu);
                ub[IX(S, I1, I2, 1)] = fma(-(omega / c), v, ub[IX(S, I1, I2, 1)]);
            }
    }
}

/* gauss_seidel!(..., FourColors{P1,P2}) (src/multigrid.jl:206-232): the cells
 * (G+1+2a+P1, G+1+2b+P2) of every block of level l, updated as
 * u -= omega (Lu + s b) / c (no fused operations). */
void orc_gs4_level(double *u, const double *b, double omega, double s, const orc_tree *t, int l,
                   const orc_operator *op, int p1, int p2) {
    const int M = t->M, G = t->G, S = M + 2 * G;
    const orc_pair *p = t->pairs[l - 1];
    const int64_t n = t->npairs[l - 1];
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) {
        const int64_t blk = p[k].blk;
        const int64_t g0r = (int64_t)M * (p[k].coord[0] - 1) + 1;
        const int64_t g0z = (int64_t)M * (p[k].coord[1] - 1) + 1;
        double *ub = u + (int64_t)S * S * (blk - 1);
        const double *bb = b + (int64_t)S * S * (blk - 1);
        for (int i2 = G + 1; i2 <= G + M; i2 += 2)
            for (int i1 = G + 1; i1 <= G + M; i1 += 2) {
                const int I1 = i1 + p1, I2 = i2 + p2;
                const int64_t J1 = I1 - G + g0r - 1, J2 = I2 - G + g0z - 1;
                const double c = diagelm4(op->geom, J1, J2);
                double cf[9];
                coeffs9(op->geom, J1, J2, cf);
                const double Lu = apply9(ub, S, I1, I2, cf);
                const double upd = omega * (Lu + s * bb[IX(S, I1, I2, 1)]) / c;
                ub[IX(S, I1, I2, 1)] = ub[IX(S, I1, I2, 1)] - upd;
            }
    }
}

/* gauss_seidel_iter! (src/multigrid.jl:250-295): order 2 runs red, copy+bnd ghosts,
 * black, copy+bnd ghosts; order 4 the four colours {0,0}, {0,1}, {1,0}, {1,1}, each
 * followed by copy+bnd ghosts.  Refinement-boundary ghosts stay frozen. */
void orc_gs_iter(double *u, const double *b, double omega, double s, int n, int l,
                 const orc_tree *t, const orc_operator *op) {
    if (op->op == 2) {
        for (int it = 0; it < n; it++)
            for (int c = 0; c < 4; c++) {
                orc_gs4_level(u, b, omega, s, t, l, op, c >> 1, c & 1);
                orc_fill_ghost_copy(u, t, l);
                orc_fill_ghost_bnd(u, t, l, op->bc);
            }
        return;
    }
    for (int it = 0; it < n; it++) {
        orc_gs_level(u, b, omega, s, t, l, op, 0);
        orc_fill_ghost_copy(u, t, l);
        orc_fill_ghost_bnd(u, t, l, op->bc);
        orc_gs_level(u, b, omega, s, t, l, op, 1);
        orc_fill_ghost_copy(u, t, l);
        orc_fill_ghost_bnd(u, t, l, op->bc);
    }
}

/* residual! over residual_level! (src/multigrid.jl:309-323, 349-354): r = -(b + Lu/s). */
void orc_residual_level(double *r, const double *u, const double *b, double s,
                        const orc_tree *t, int l, const orc_operator *op) {
    const int M = t->M, G = t->G, S = M + 2 * G;
    const orc_pair *p = t->pairs[l - 1];
    const int64_t n = t->npairs[l - 1];
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) {
        const int64_t blk = p[k].blk;
        const int64_t g0r = (int64_t)M * (p[k].coord[0] - 1) + 1;
        const int64_t g0z = (int64_t)M * (p[k].coord[1] - 1) + 1;
        const double *ub = u + (int64_t)S * S * (blk - 1);
        for (int I2 = G + 1; I2 <= G + M; I2++)
            for (int I1 = G + 1; I1 <= G + M; I1++) {
                const double Lu = lhs_apply(op, s, ub, S, I1, I2, I1 - G + g0r - 1, I2 - G + g0z - 1);
                const int64_t o = IX(S, I1, I2, blk);
                r[o] = -(b[o] + Lu / s);
            }
    }
}

/* residual_postrestrict_level! + residual_subblock! (src/multigrid.jl:112-119, 331-344):
 * for each Child edge of level l, on the coarse subblock:
 * bfield = -(r + L(u)/s), s being the coarse-level scale (the caller passes 4*s_l). */
void orc_residual_postrestrict_level(double *bfield, const double *u, const double *r, double s,
                                     const orc_tree *t, int l, const orc_operator *op) {
    const int M = t->M, G = t->G, S = M + 2 * G;
    const orc_child *v = t->ch[l - 1];
    const int64_t n = t->nch[l - 1];
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) {
        const int64_t blk = v[k].coarse;
        const int64_t c0 = t->coord_of[2 * (blk - 1)], c1 = t->coord_of[2 * (blk - 1) + 1];
        const int64_t g0r = (int64_t)M * (c0 - 1) + 1, g0z = (int64_t)M * (c1 - 1) + 1;
        int lo[2], hi[2];
        for (int d = 0; d < 2; d++) subblock_bounds(M, G, v[k].subblock[d], &lo[d], &hi[d]);
        const double *ub = u + (int64_t)S * S * (blk - 1);
        for (int I2 = lo[1]; I2 <= hi[1]; I2++)
            for (int I1 = lo[0]; I1 <= hi[0]; I1++) {
                const double Lu = lhs_apply(op, s, ub, S, I1, I2, I1 - G + g0r - 1, I2 - G + g0z - 1);
                const int64_t o = IX(S, I1, I2, blk);
                bfield[o] = -(r[o] + Lu / s);
            }
    }
}

static inline double level_scale(double s, int l) {
    const int64_t f = (int64_t)1 << (l - 1);
    return s / (double)(f * f);
}

/* vcycle! (src/multigrid.jl:60-106). */
void orc_vcycle(double *u, double *b, double *r, double *u1, double s, const orc_tree *t,
                const orc_operator *op, int lmax, int ndown, int ntop, int nup, double omega) {
    if (lmax == 0) lmax = t->nlev;
    for (int l = lmax; l >= 2; l--) {
        const double sl = level_scale(s, l);
        orc_gs_iter(u, b, omega, sl, ndown, l, t, op);
        orc_restrict_level(u, t, l);
        orc_fill_ghost(u, t, l - 1, op->bc);
        orc_copyto_level(u1, u, t, l - 1);
        orc_residual_level(r, u, b, sl, t, l, op);
        orc_fill_ghost(r, t, l, op->bc);
        orc_restrict_level(r, t, l);
        orc_fill_ghost(r, t, l - 1, op->bc);
        orc_residual_postrestrict_level(b, u, r, 4 * sl, t, l, op);
    }
    orc_gs_iter(u, b, omega, s, ntop, 1, t, op);
    for (int l = 2; l <= lmax; l++) {
        const double sl = level_scale(s, l);
        orc_diffto_level(u1, u, u1, t, l - 1);
        orc_fill_ghost(u1, t, l - 1, op->bc);
        orc_interp_add_level(u, u1, t, l);
        orc_fill_ghost(u, t, l, op->bc);
        orc_gs_iter(u, b, omega, sl, nup, l, t, op);
        orc_fill_ghost(u, t, l, op->bc);
    }
}

static int finest_level(const orc_tree *t) {
    int lmax = 0;
    for (int l = 1; l <= t->nlev; l++)
        if (t->npairs[l - 1] > 0) lmax = l;
    return lmax;
}

/* fmg! (src/multigrid.jl:17-51).  As in the reference, lmax is always the finest
 * non-empty level. */
void orc_fmg(double *u, double *b, double *r, double *u1, double s, const orc_tree *t,
             const orc_operator *op, int ndown, int ntop, int nup, double omega) {
    const int lmax = finest_level(t);
    for (int l = lmax; l >= 2; l--) {
        const double sl = level_scale(s, l);
        orc_restrict_level(u, t, l);
        orc_fill_ghost(u, t, l - 1, op->bc);
        orc_residual_level(r, u, b, sl, t, l, op);
        orc_fill_ghost(r, t, l, op->bc);
        orc_restrict_level(r, t, l);
        orc_fill_ghost(r, t, l - 1, op->bc);
        orc_residual_postrestrict_level(b, u, r, 4 * sl, t, l, op);
    }
    for (int l = 1; l <= lmax; l++) {
        orc_copyto_level(u1, u, t, l);
        if (l > 1) {
            orc_diffto_level(u1, u, u1, t, l - 1);
            orc_fill_ghost(u1, t, l - 1, op->bc);
            orc_interp_add_level(u, u1, t, l);
        }
        orc_fill_ghost(u, t, l, op->bc);
        orc_vcycle(u, b, r, u1, s, t, op, l, ndown, ntop, nup, omega);
    }
}

/* Sum of squares of the level-1 valid cells after restricting squares down the tree:
 * the tail of resnorm! (src/multigrid.jl:400-416).  The reference writes the
 * squaring as `m .= m.^2` over r.u, which only runs for :vector storage; the intended
 * elementwise square is restated here. */
static double restricted_square_sum(double *r, const orc_tree *t) {
    const int M = t->M, G = t->G, S = M + 2 * G;
    const int64_t total = t->nblk_alloc * S * S;
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < total; q++) r[q] = r[q] * r[q];
    for (int l = t->nlev - 1; l >= 1; l--) orc_restrict_level(r, t, l + 1);
    double w = 0.0;
    for (int64_t k = 0; k < t->npairs[0]; k++) {
        const int64_t blk = t->pairs[0][k].blk;
        double part = 0.0;
        int first = 1;
        for (int j = G + 1; j <= G + M; j++)
            for (int i = G + 1; i <= G + M; i++) {
                const double x = r[IX(S, i, j, blk)];
                if (first) { part = x; first = 0; } else part += x;
            }
        w += part;
    }
    return sqrt(w);
}

/* resnorm! (src/multigrid.jl:391-417). */
double orc_resnorm(double *r, const double *b, const double *u, double s, const orc_tree *t,
                   const orc_operator *op) {
    for (int l = t->nlev; l >= 1; l--) orc_residual_level(r, u, b, level_scale(s, l), t, l, op);
    return restricted_square_sum(r, t);
}

/* The same area-weighted leaf norm applied to an arbitrary field (used for |b|). */
double orc_leafnorm(double *scratch, const double *f, const orc_tree *t) {
    const int S = t->M + 2 * t->G;
    memcpy(scratch, f, sizeof(double) * t->nblk_alloc * S * S);
    return restricted_square_sum(scratch, t);
}

int orc_solve(double *u, double *b, double *r, double *u1, double s, const orc_tree *t,
              const orc_operator *op, int ndown, int ntop, int nup, double omega,
              double tol, int max_cycles, double *rel) {
    const double bn = orc_leafnorm(r, b, t);
    const double scale = bn > 0 ? bn : 1.0;
    double x = orc_resnorm(r, b, u, s, t, op) / scale;
    int c = 0;
    while (x > tol && c < max_cycles) {
        orc_vcycle(u, b, r, u1, s, t, op, 0, ndown, ntop, nup, omega);
        c++;
        x = orc_resnorm(r, b, u, s, t, op) / scale;
    }
    if (rel) *rel = x;
    return c;
}

/* ---- stage preparation and post-processing --------------------------------------- */

/* rhs_level! over rhs! (src/multigrid.jl:363-388): q1 = R q on the valid cells of every
 * block of level l.  Order 2: the identity (src/laplacian.jl:86-91,120-125,
 * src/helmholtz.jl:27-32,59-64).  Order 4: the compact right-hand side
 * (src/laplacian.jl:141-148,166-173,186-193), a 3x3 literal walked column-major
 * (v = 0; v += c u) over its nonzero entries, then divided by 12. */
void orc_rhs_level(double *q1, const double *q, const orc_tree *t, int l, const orc_operator *op) {
    const int M = t->M, G = t->G, S = M + 2 * G;
    const orc_pair *p = t->pairs[l - 1];
    const int64_t n = t->npairs[l - 1];
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) {
        const int64_t blk = p[k].blk;
        const int64_t g0r = (int64_t)M * (p[k].coord[0] - 1) + 1;
        const int64_t g0z = (int64_t)M * (p[k].coord[1] - 1) + 1;
        const double *qb = q + (int64_t)S * S * (blk - 1);
        for (int I2 = G + 1; I2 <= G + M; I2++)
            for (int I1 = G + 1; I1 <= G + M; I1++) {
                const int64_t o = IX(S, I1, I2, blk);
                if (op->op != 2) {
                    q1[o] = q[o];
                    continue;
                }
                /* nonzero entries in walk order: (0,-1), (-1,0), (0,0), (1,0), (0,1) */
                double wzm = 1, wrm = 1, wrp = 1, wzp = 1;
                if (op->geom == 1) {
                    const int64_t i = I1 - G + g0r - 1;
                    wrm = (double)(2 * i - 2) / (double)(2 * i - 1);
                    wrp = (double)(2 * i) / (double)(2 * i - 1);
                } else if (op->geom == 2) {
                    const int64_t i = I2 - G + g0z - 1;
                    wzm = (double)(2 * i - 2) / (double)(2 * i - 1);
                    wzp = (double)(2 * i) / (double)(2 * i - 1);
                }
                double v = 0.0;
                v += wzm * qb[IX(S, I1, I2 - 1, 1)];
                v += wrm * qb[IX(S, I1 - 1, I2, 1)];
                v += 8 * qb[IX(S, I1, I2, 1)];
                v += wrp * qb[IX(S, I1 + 1, I2, 1)];
                v += wzp * qb[IX(S, I1, I2 + 1, 1)];
                q1[o] = v / 12;
            }
    }
}

/* netcharge! (src/streamer.jl:369-373): q[I] = dot(n[I], species_charge) over the valid
 * cells of every block; NetIonization charges are (-1, +1) (src/chemistry.jl:80), so
 * q = (n_e * -1) + (n_ion * 1), the products exact. */
void orc_netcharge(double *q, const double *ne, const double *nion, const orc_tree *t) {
    const int M = t->M, G = t->G, S = M + 2 * G;
    for (int l = 1; l <= t->nlev; l++) {
        const orc_pair *p = t->pairs[l - 1];
        const int64_t n = t->npairs[l - 1];
#pragma omp parallel for schedule(static)
        for (int64_t k = 0; k < n; k++)
            for (int j = G + 1; j <= G + M; j++)
                for (int i = G + 1; i <= G + M; i++) {
                    const int64_t o = IX(S, i, j, p[k].blk);
                    q[o] = ne[o] * -1.0 + nion[o] * 1.0;
                }
    }
}

/* electric_field! (src/multigrid.jl:421-449) with a constant field e0 (the SVector
 * method, :451).  e is a VectorBlockField (src/blockfield.jl:84-95): (S+1)^2 x 2 values
 * per block, component d at offset d (S+1)^2.  h_l = h / (1 << (level - 1)).  For
 * d = 1, 2 and I in validindices(e, d) (src/blockfield.jl:403-405: G+1..G+M+1 along d,
 * G+1..G+M across): e[I, d] = (u[I - e_d] - u[I]) / h_l + e0[d].  Then for the valid
 * cells: f2 = 0; f2 += (e[I, d] + e[I + e_d, d])^2 / 4 for d = 1, 2; eabs = sqrt(f2). */
void orc_electric_field(double *e, double *eabs, const double *u, double h, const double e0[2],
                        const orc_tree *t) {
    const int M = t->M, G = t->G, S = M + 2 * G, SV = S + 1;
    for (int l = 1; l <= t->nlev; l++) {
        const orc_pair *p = t->pairs[l - 1];
        const int64_t n = t->npairs[l - 1];
        const double hl = h / (double)((int64_t)1 << (l - 1));
#pragma omp parallel for schedule(static)
        for (int64_t k = 0; k < n; k++) {
            const int64_t blk = p[k].blk;
            double *eb = e + (int64_t)2 * SV * SV * (blk - 1);
            for (int d = 0; d < 2; d++)
                for (int j = G + 1; j <= G + M + (d == 1); j++)
                    for (int i = G + 1; i <= G + M + (d == 0); i++) {
                        const int i1 = d == 0 ? i - 1 : i, j1 = d == 1 ? j - 1 : j;
                        eb[(i - 1) + SV * (j - 1) + SV * SV * d] =
                            (u[IX(S, i1, j1, blk)] - u[IX(S, i, j, blk)]) / hl + e0[d];
                    }
            for (int j = G + 1; j <= G + M; j++)
                for (int i = G + 1; i <= G + M; i++) {
                    double f2 = 0.0;
                    for (int d = 0; d < 2; d++) {
                        const int ip = d == 0 ? i + 1 : i, jp = d == 1 ? j + 1 : j;
                        const double sum = eb[(i - 1) + SV * (j - 1) + SV * SV * d] +
                                           eb[(ip - 1) + SV * (jp - 1) + SV * SV * d];
                        f2 += sum * sum / 4;
                    }
                    eabs[IX(S, i, j, blk)] = sqrt(f2);
                }
        }
    }
}
