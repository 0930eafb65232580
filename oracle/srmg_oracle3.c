/*
 * srmg_oracle3.c -- CPU FP64 restatement of Steamroller.jl's multigrid field solve in
 * three dimensions (D = 3, CartesianGeometry: the only geometry the reference defines
 * 3D stencils for).
 *
 * TEST INFRASTRUCTURE ONLY (the oracle): loaded by tests/; never by the product.
 * Parity: UNPINNED, as for the 2D oracle (no reference tests; no Julia here); pinned
 * by known-answer tests in tests/test_oracle3.py.
 *
 * The reference's solver code is dimension-generic (Base.Cartesian @nloops, with the
 * first index innermost); this file writes out D = 3 with the same operation order:
 *   ghost fills      src/connectivity.jl:155-258 (any face in {-1,0,1}^3)
 *   interpolation    src/interp.jl:24-63 with __w0(Val(3)) = __w1(Val(3)) = 1/4 (:7-11)
 *   restriction      src/restrict.jl:5-47 (sum of 8 fine cells, then / 8)
 *   stencils         src/laplacian.jl:274-340, src/helmholtz.jl:74-100
 *   Gauss-Seidel     src/multigrid.jl:153-232 (RedBlack and FourColors for D = 3)
 *   V-cycle, FMG, resnorm, rhs_level  src/multigrid.jl:17-119, 309-417
 * Compiled with -ffp-contract=off; fma() exactly where the reference calls muladd.
 */
#include "srmg_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

static inline int64_t IX3(int S, int i, int j, int k, int64_t blk) {
    return (int64_t)(i - 1) + (int64_t)S * (j - 1) + (int64_t)S * S * (k - 1) + (int64_t)S * S * S * (blk - 1);
}

void orc3_tree_index(orc3_tree *t) {
    for (int64_t q = 0; q < 3 * t->nblk_alloc; q++) t->coord_of[q] = -1;
    for (int l = 0; l < t->nlev; l++)
        for (int64_t p = 0; p < t->npairs[l]; p++) {
            const orc3_pair *pr = &t->pairs[l][p];
            for (int d = 0; d < 3; d++) t->coord_of[3 * (pr->blk - 1) + d] = pr->coord[d];
        }
}

/* ---- ghost fills -------------------------------------------------------------- */

/* _fill_ghost_copy! (src/connectivity.jl:184-198) for D = 3. */
void orc3_fill_ghost_copy(double *u, const orc3_tree *t, int l) {
    const int M = t->M, G = t->G, S = M + 2 * G;
    const orc3_neighbor *v = t->nb[l - 1];
    const int64_t n = t->nnb[l - 1];
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; q++) {
        const orc3_neighbor *e = &v[q];
        int cnt[3];
        for (int d = 0; d < 3; d++) cnt[d] = e->face[d] == 0 ? M : G;
        for (int i3 = 1; i3 <= cnt[2]; i3++)
            for (int i2 = 1; i2 <= cnt[1]; i2++)
                for (int i1 = 1; i1 <= cnt[0]; i1++) {
                    const int i[3] = {i1, i2, i3};
                    int fr[3], to[3];
                    for (int d = 0; d < 3; d++) {
                        const int64_t f = e->face[d];
                        fr[d] = f == 0 ? G + i[d] : (f == -1 ? i[d] + G : i[d] + M);
                        to[d] = f == 0 ? G + i[d] : (f == 1 ? i[d] : i[d] + M + G);
                    }
                    u[IX3(S, to[0], to[1], to[2], e->to)] = u[IX3(S, fr[0], fr[1], fr[2], e->from)];
                }
    }
}

static void ghost_bounds(int M, int G, int64_t face, int *lo, int *hi) {
    if (face == 0) { *lo = G + 1; *hi = G + M; }
    else if (face == -1) { *lo = 1; *hi = G; }
    else { *lo = M + G + 1; *hi = M + 2 * G; }
}

static inline int mirror(int M, int G, int i, int64_t dir) {
    if (dir == -1) return 2 * G - i + 1;
    if (dir == 1) return 2 * (G + M) - i + 1;
    return i;
}

/* fill_ghost_bnd! (src/connectivity.jl:217-231), getbc (src/boundary.jl:45-47): the
 * 3x3x3 table a[2+b1, 2+b2, 2+b3], column-major. */
void orc3_fill_ghost_bnd(double *u, const orc3_tree *t, int l, const int8_t bc[27]) {
    const int M = t->M, G = t->G, S = M + 2 * G;
    const orc3_boundary *v = t->bd[l - 1];
    const int64_t n = t->nbd[l - 1];
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; q++) {
        const orc3_boundary *e = &v[q];
        int lo[3], hi[3];
        for (int d = 0; d < 3; d++) ghost_bounds(M, G, e->face[d], &lo[d], &hi[d]);
        const double a = (double)bc[(1 + e->bnd[0]) + 3 * (1 + e->bnd[1]) + 9 * (1 + e->bnd[2])];
        for (int k = lo[2]; k <= hi[2]; k++)
            for (int j = lo[1]; j <= hi[1]; j++)
                for (int i = lo[0]; i <= hi[0]; i++) {
                    const int mi = mirror(M, G, i, e->bnd[0]), mj = mirror(M, G, j, e->bnd[1]),
                              mk = mirror(M, G, k, e->bnd[2]);
                    u[IX3(S, i, j, k, e->block)] = a * u[IX3(S, mi, mj, mk, e->block)];
                }
    }
}

/* interp!(InterpLinear, dest, idest, src, isrc, func) (src/interp.jl:24-63), D = 3:
 * per coarse cell, children in @nloops order (first offset innermost),
 * f = 1/4 src[Js] + 1/4 src[Js +- e1] + 1/4 src[Js +- e2] + 1/4 src[Js +- e3]. */
static void interp3(double *dest, const int dlo[3], const double *src, const int slo[3], const int shi[3], int S,
                    int add) {
    for (int k3 = 0; k3 <= shi[2] - slo[2]; k3++)
        for (int k2 = 0; k2 <= shi[1] - slo[1]; k2++)
            for (int k1 = 0; k1 <= shi[0] - slo[0]; k1++) {
                const int js[3] = {slo[0] + k1, slo[1] + k2, slo[2] + k3};
                const int jd0[3] = {dlo[0] + 2 * k1, dlo[1] + 2 * k2, dlo[2] + 2 * k3};
                for (int i3 = 0; i3 <= 1; i3++)
                    for (int i2 = 0; i2 <= 1; i2++)
                        for (int i1 = 0; i1 <= 1; i1++) {
                            const int ii[3] = {i1, i2, i3};
                            double f = 0.25 * src[IX3(S, js[0], js[1], js[2], 1)];
                            for (int j = 0; j < 3; j++) {
                                int o[3] = {js[0], js[1], js[2]};
                                o[j] += 2 * ii[j] - 1;
                                f += 0.25 * src[IX3(S, o[0], o[1], o[2], 1)];
                            }
                            double *dp = &dest[IX3(S, jd0[0] + i1, jd0[1] + i2, jd0[2] + i3, 1)];
                            *dp = add ? (f + *dp) : f;
                        }
            }
}

static void subblock_bounds(int M, int G, int64_t sb, int *lo, int *hi) {
    const int mh = M / 2;
    *lo = G + 1 + (int)(sb - 1) * mh;
    *hi = G + (int)sb * mh;
}

/* fill_ghost_interp! (src/connectivity.jl:251-258) with subblockbnd
 * (src/blockfield.jl:416-434). */
void orc3_fill_ghost_interp(double *u, const orc3_tree *t, int l) {
    const int M = t->M, G = t->G, S = M + 2 * G, gh = G / 2;
    const orc3_refbnd *v = t->rb[l - 1];
    const int64_t n = t->nrb[l - 1];
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; q++) {
        const orc3_refbnd *e = &v[q];
        int dlo[3], dhi[3], slo[3], shi[3];
        for (int d = 0; d < 3; d++) {
            ghost_bounds(M, G, e->face[d], &dlo[d], &dhi[d]);
            int lo, hi;
            subblock_bounds(M, G, e->subblock[d], &lo, &hi);
            const int64_t mf = -e->face[d];
            if (mf == -1) { slo[d] = lo; shi[d] = lo + gh - 1; }
            else if (mf == 1) { slo[d] = hi - gh + 1; shi[d] = hi; }
            else { slo[d] = lo; shi[d] = hi; }
        }
        (void)dhi;
        interp3(u + (int64_t)S * S * S * (e->fine - 1), dlo, u + (int64_t)S * S * S * (e->coarse - 1), slo, shi, S,
                0);
    }
}

void orc3_fill_ghost(double *u, const orc3_tree *t, int l, const int8_t bc[27]) {
    orc3_fill_ghost_copy(u, t, l);
    orc3_fill_ghost_bnd(u, t, l, bc);
    orc3_fill_ghost_interp(u, t, l);
}

/* ---- transfers ------------------------------------------------------------------- */

/* restrict! (src/restrict.jl:5-25), D = 3: f = 0; f += fine over the 8 offsets (first
 * innermost); coarse = f / 8. */
void orc3_restrict_level(double *u, const orc3_tree *t, int l) {
    const int M = t->M, G = t->G, S = M + 2 * G, mh = M / 2;
    const orc3_child *v = t->ch[l - 1];
    const int64_t n = t->nch[l - 1];
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; q++) {
        const orc3_child *e = &v[q];
        const double *src = u + (int64_t)S * S * S * (e->fine - 1);
        double *dst = u + (int64_t)S * S * S * (e->coarse - 1);
        int dlo[3], dhi[3];
        for (int d = 0; d < 3; d++) subblock_bounds(M, G, e->subblock[d], &dlo[d], &dhi[d]);
        for (int c3 = 1; c3 <= mh; c3++)
            for (int c2 = 1; c2 <= mh; c2++)
                for (int c1 = 1; c1 <= mh; c1++) {
                    const int j0 = G + 2 * c1 - 1, j1 = G + 2 * c2 - 1, j2 = G + 2 * c3 - 1;
                    double f = 0.0;
                    for (int i3 = 0; i3 <= 1; i3++)
                        for (int i2 = 0; i2 <= 1; i2++)
                            for (int i1 = 0; i1 <= 1; i1++) f += src[IX3(S, j0 + i1, j1 + i2, j2 + i3, 1)];
                    dst[IX3(S, dlo[0] + c1 - 1, dlo[1] + c2 - 1, dlo[2] + c3 - 1, 1)] = f / 8;
                }
    }
}

void orc3_interp_add_level(double *u, const double *u1, const orc3_tree *t, int l) {
    const int M = t->M, G = t->G, S = M + 2 * G;
    const orc3_child *v = t->ch[l - 1];
    const int64_t n = t->nch[l - 1];
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; q++) {
        const orc3_child *e = &v[q];
        int slo[3], shi[3];
        for (int d = 0; d < 3; d++) subblock_bounds(M, G, e->subblock[d], &slo[d], &shi[d]);
        const int dlo[3] = {G + 1, G + 1, G + 1};
        interp3(u + (int64_t)S * S * S * (e->fine - 1), dlo, u1 + (int64_t)S * S * S * (e->coarse - 1), slo, shi, S,
                1);
    }
}

void orc3_copyto_level(double *dst, const double *src, const orc3_tree *t, int l) {
    const int S = t->M + 2 * t->G;
    const orc3_pair *p = t->pairs[l - 1];
    for (int64_t q = 0; q < t->npairs[l - 1]; q++) {
        const int64_t off = (int64_t)S * S * S * (p[q].blk - 1);
        memcpy(dst + off, src + off, sizeof(double) * S * S * S);
    }
}

void orc3_diffto_level(double *dst, const double *a1, const double *a2, const orc3_tree *t, int l) {
    const int S = t->M + 2 * t->G;
    const orc3_pair *p = t->pairs[l - 1];
    for (int64_t q = 0; q < t->npairs[l - 1]; q++) {
        const int64_t off = (int64_t)S * S * S * (p[q].blk - 1);
        for (int c = 0; c < S * S * S; c++) dst[off + c] = a1[off + c] - a2[off + c];
    }
}

/* ---- stencils --------------------------------------------------------------------
 * @stencil over a 3x3x3 literal (src/laplacian.jl:25-49): walked with the first offset
 * fastest and the slab (third offset) slowest, skipping literal zeros.
 * Order 2 (src/laplacian.jl:274-290, src/helmholtz.jl:74-89): 7 points, centre -6 or
 * -6 - s k2.  Order 4 (:303-340): 19 points (faces 2, edges 1, centre -24) / 6;
 * right-hand side 7 points (centre 6) / 12. */
static double lhs3(const orc_operator *op, double s, const double *ub, int S, int i, int j, int k) {
    if (op->op == 2) {
        double v = 0.0;
        for (int d3 = -1; d3 <= 1; d3++)
            for (int d2 = -1; d2 <= 1; d2++)
                for (int d1 = -1; d1 <= 1; d1++) {
                    const int nz = (d1 != 0) + (d2 != 0) + (d3 != 0);
                    if (nz == 3) continue;  /* the 8 corners are literal zeros */
                    const double c = nz == 0 ? -24.0 : nz == 1 ? 2.0 : 1.0;
                    v += c * ub[IX3(S, i + d1, j + d2, k + d3, 1)];
                }
        return v / 6;
    }
    const double cc = op->op == 1 ? (-6 - s * op->k2) : -6.0;
    double v = 0.0;
    v += ub[IX3(S, i, j, k - 1, 1)];
    v += ub[IX3(S, i, j - 1, k, 1)];
    v += ub[IX3(S, i - 1, j, k, 1)];
    v += cc * ub[IX3(S, i, j, k, 1)];
    v += ub[IX3(S, i + 1, j, k, 1)];
    v += ub[IX3(S, i, j + 1, k, 1)];
    v += ub[IX3(S, i, j, k + 1, 1)];
    return v;
}

static inline double diag3(const orc_operator *op, double s) {
    if (op->op == 2) return -4.0;
    return op->op == 1 ? (-6 - s * op->k2) : -6.0;
}

/* gauss_seidel!(..., RedBlack{P}) for D = 3 (src/multigrid.jl:153-180): i1 steps by 2,
 * p = P xor (i2 & 1) xor (i3 & 1), two muladds. */
void orc3_gs_level(double *u, const double *b, double omega, double s, const orc3_tree *t, int l,
                   const orc_operator *op, int parity) {
    const int M = t->M, G = t->G, S = M + 2 * G;
    const orc3_pair *p = t->pairs[l - 1];
    const int64_t n = t->npairs[l - 1];
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; q++) {
        double *ub = u + (int64_t)S * S * S * (p[q].blk - 1);
        const double *bb = b + (int64_t)S * S * S * (p[q].blk - 1);
        for (int i3 = G + 1; i3 <= G + M; i3++)
            for (int i2 = G + 1; i2 <= G + M; i2++)
                for (int i1 = G + 1; i1 <= G + M; i1 += 2) {
                    const int pp = parity ^ (i2 & 1) ^ (i3 & 1);
                    const int I1 = i1 + pp;
                    const double c = diag3(op, s);
                    const double Lu = lhs3(op, s, ub, S, I1, i2, i3);
                    const double v = fma(s, bb[IX3(S, I1, i2, i3, 1)], Lu);
                    ub[IX3(S, I1, i2, i3, 1)] = fma(-(omega / c), v, ub[IX3(S, I1, i2, i3, 1)]);
                }
    }
}

/* gauss_seidel!(..., FourColors{P1,P2}) for D = 3 (src/multigrid.jl:206-232): cells
 * (i1 + p1, i2 + p2, i3) over validrange2^2 x validrange, p_a = (P_a + i3) mod 2,
 * u -= omega (Lu + s b) / c. */
void orc3_gs4_level(double *u, const double *b, double omega, double s, const orc3_tree *t, int l,
                    const orc_operator *op, int P1, int P2) {
    const int M = t->M, G = t->G, S = M + 2 * G;
    const orc3_pair *p = t->pairs[l - 1];
    const int64_t n = t->npairs[l - 1];
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; q++) {
        double *ub = u + (int64_t)S * S * S * (p[q].blk - 1);
        const double *bb = b + (int64_t)S * S * S * (p[q].blk - 1);
        for (int i3 = G + 1; i3 <= G + M; i3++)
            for (int i2 = G + 1; i2 <= G + M; i2 += 2)
                for (int i1 = G + 1; i1 <= G + M; i1 += 2) {
                    const int p1 = (P1 + i3) % 2, p2 = (P2 + i3) % 2;
                    const int I1 = i1 + p1, I2 = i2 + p2;
                    const double c = diag3(op, s);
                    const double Lu = lhs3(op, s, ub, S, I1, I2, i3);
                    const double upd = omega * (Lu + s * bb[IX3(S, I1, I2, i3, 1)]) / c;
                    ub[IX3(S, I1, I2, i3, 1)] = ub[IX3(S, I1, I2, i3, 1)] - upd;
                }
    }
}

void orc3_gs_iter(double *u, const double *b, double omega, double s, int n, int l, const orc3_tree *t,
                  const orc_operator *op) {
    for (int it = 0; it < n; it++) {
        if (op->op == 2) {
            for (int c = 0; c < 4; c++) {
                orc3_gs4_level(u, b, omega, s, t, l, op, c >> 1, c & 1);
                orc3_fill_ghost_copy(u, t, l);
                orc3_fill_ghost_bnd(u, t, l, op->bc27);
            }
        } else {
            for (int c = 0; c < 2; c++) {
                orc3_gs_level(u, b, omega, s, t, l, op, c);
                orc3_fill_ghost_copy(u, t, l);
                orc3_fill_ghost_bnd(u, t, l, op->bc27);
            }
        }
    }
}

void orc3_residual_level(double *r, const double *u, const double *b, double s, const orc3_tree *t, int l,
                         const orc_operator *op) {
    const int M = t->M, G = t->G, S = M + 2 * G;
    const orc3_pair *p = t->pairs[l - 1];
    const int64_t n = t->npairs[l - 1];
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; q++) {
        const int64_t blk = p[q].blk;
        const double *ub = u + (int64_t)S * S * S * (blk - 1);
        for (int k = G + 1; k <= G + M; k++)
            for (int j = G + 1; j <= G + M; j++)
                for (int i = G + 1; i <= G + M; i++) {
                    const int64_t o = IX3(S, i, j, k, blk);
                    r[o] = -(b[o] + lhs3(op, s, ub, S, i, j, k) / s);
                }
    }
}

void orc3_residual_postrestrict_level(double *bfield, const double *u, const double *r, double s,
                                      const orc3_tree *t, int l, const orc_operator *op) {
    const int M = t->M, G = t->G, S = M + 2 * G;
    const orc3_child *v = t->ch[l - 1];
    const int64_t n = t->nch[l - 1];
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; q++) {
        const int64_t blk = v[q].coarse;
        int lo[3], hi[3];
        for (int d = 0; d < 3; d++) subblock_bounds(M, G, v[q].subblock[d], &lo[d], &hi[d]);
        const double *ub = u + (int64_t)S * S * S * (blk - 1);
        for (int k = lo[2]; k <= hi[2]; k++)
            for (int j = lo[1]; j <= hi[1]; j++)
                for (int i = lo[0]; i <= hi[0]; i++) {
                    const int64_t o = IX3(S, i, j, k, blk);
                    bfield[o] = -(r[o] + lhs3(op, s, ub, S, i, j, k) / s);
                }
    }
}

/* rhs_level! (src/multigrid.jl:363-388): identity at order 2; order 4 the 7-point
 * right-hand side (src/laplacian.jl:322-337) / 12. */
void orc3_rhs_level(double *q1, const double *q, const orc3_tree *t, int l, const orc_operator *op) {
    const int M = t->M, G = t->G, S = M + 2 * G;
    const orc3_pair *p = t->pairs[l - 1];
    for (int64_t c = 0; c < t->npairs[l - 1]; c++) {
        const int64_t blk = p[c].blk;
        const double *qb = q + (int64_t)S * S * S * (blk - 1);
        for (int k = G + 1; k <= G + M; k++)
            for (int j = G + 1; j <= G + M; j++)
                for (int i = G + 1; i <= G + M; i++) {
                    const int64_t o = IX3(S, i, j, k, blk);
                    if (op->op != 2) {
                        q1[o] = q[o];
                        continue;
                    }
                    double v = 0.0;
                    v += qb[IX3(S, i, j, k - 1, 1)];
                    v += qb[IX3(S, i, j - 1, k, 1)];
                    v += qb[IX3(S, i - 1, j, k, 1)];
                    v += 6 * qb[IX3(S, i, j, k, 1)];
                    v += qb[IX3(S, i + 1, j, k, 1)];
                    v += qb[IX3(S, i, j + 1, k, 1)];
                    v += qb[IX3(S, i, j, k + 1, 1)];
                    q1[o] = v / 12;
                }
    }
}

static inline double level_scale(double s, int l) {
    const int64_t f = (int64_t)1 << (l - 1);
    return s / (double)(f * f);
}

/* vcycle! (src/multigrid.jl:60-106). */
void orc3_vcycle(double *u, double *b, double *r, double *u1, double s, const orc3_tree *t, const orc_operator *op,
                 int lmax, int ndown, int ntop, int nup, double omega) {
    if (lmax == 0) lmax = t->nlev;
    for (int l = lmax; l >= 2; l--) {
        const double sl = level_scale(s, l);
        orc3_gs_iter(u, b, omega, sl, ndown, l, t, op);
        orc3_restrict_level(u, t, l);
        orc3_fill_ghost(u, t, l - 1, op->bc27);
        orc3_copyto_level(u1, u, t, l - 1);
        orc3_residual_level(r, u, b, sl, t, l, op);
        orc3_fill_ghost(r, t, l, op->bc27);
        orc3_restrict_level(r, t, l);
        orc3_fill_ghost(r, t, l - 1, op->bc27);
        orc3_residual_postrestrict_level(b, u, r, 4 * sl, t, l, op);
    }
    orc3_gs_iter(u, b, omega, s, ntop, 1, t, op);
    for (int l = 2; l <= lmax; l++) {
        const double sl = level_scale(s, l);
        orc3_diffto_level(u1, u, u1, t, l - 1);
        orc3_fill_ghost(u1, t, l - 1, op->bc27);
        orc3_interp_add_level(u, u1, t, l);
        orc3_fill_ghost(u, t, l, op->bc27);
        orc3_gs_iter(u, b, omega, sl, nup, l, t, op);
        orc3_fill_ghost(u, t, l, op->bc27);
    }
}

/* fmg! (src/multigrid.jl:17-51). */
void orc3_fmg(double *u, double *b, double *r, double *u1, double s, const orc3_tree *t, const orc_operator *op,
              int ndown, int ntop, int nup, double omega) {
    int lmax = 0;
    for (int l = 1; l <= t->nlev; l++)
        if (t->npairs[l - 1] > 0) lmax = l;
    for (int l = lmax; l >= 2; l--) {
        const double sl = level_scale(s, l);
        orc3_restrict_level(u, t, l);
        orc3_fill_ghost(u, t, l - 1, op->bc27);
        orc3_residual_level(r, u, b, sl, t, l, op);
        orc3_fill_ghost(r, t, l, op->bc27);
        orc3_restrict_level(r, t, l);
        orc3_fill_ghost(r, t, l - 1, op->bc27);
        orc3_residual_postrestrict_level(b, u, r, 4 * sl, t, l, op);
    }
    for (int l = 1; l <= lmax; l++) {
        orc3_copyto_level(u1, u, t, l);
        if (l > 1) {
            orc3_diffto_level(u1, u, u1, t, l - 1);
            orc3_fill_ghost(u1, t, l - 1, op->bc27);
            orc3_interp_add_level(u, u1, t, l);
        }
        orc3_fill_ghost(u, t, l, op->bc27);
        orc3_vcycle(u, b, r, u1, s, t, op, l, ndown, ntop, nup, omega);
    }
}

/* resnorm! tail (src/multigrid.jl:400-416) for D = 3: square, restrict the squares down
 * to level 1 (each restriction divides by 8), sum the level-1 valid cells. */
static double restricted_square_sum3(double *r, const orc3_tree *t) {
    const int M = t->M, G = t->G, S = M + 2 * G;
    const int64_t total = t->nblk_alloc * S * S * S;
    for (int64_t q = 0; q < total; q++) r[q] = r[q] * r[q];
    for (int l = t->nlev - 1; l >= 1; l--) orc3_restrict_level(r, t, l + 1);
    double w = 0.0;
    for (int64_t q = 0; q < t->npairs[0]; q++) {
        const int64_t blk = t->pairs[0][q].blk;
        double part = 0.0;
        int first = 1;
        for (int k = G + 1; k <= G + M; k++)
            for (int j = G + 1; j <= G + M; j++)
                for (int i = G + 1; i <= G + M; i++) {
                    const double x = r[IX3(S, i, j, k, blk)];
                    if (first) { part = x; first = 0; } else part += x;
                }
        w += part;
    }
    return sqrt(w);
}

double orc3_resnorm(double *r, const double *b, const double *u, double s, const orc3_tree *t,
                    const orc_operator *op) {
    for (int l = t->nlev; l >= 1; l--) orc3_residual_level(r, u, b, level_scale(s, l), t, l, op);
    return restricted_square_sum3(r, t);
}

double orc3_leafnorm(double *scratch, const double *f, const orc3_tree *t) {
    const int S = t->M + 2 * t->G;
    memcpy(scratch, f, sizeof(double) * t->nblk_alloc * S * S * S);
    return restricted_square_sum3(scratch, t);
}

int orc3_solve(double *u, double *b, double *r, double *u1, double s, const orc3_tree *t, const orc_operator *op,
               int ndown, int ntop, int nup, double omega, double tol, int max_cycles, double *rel) {
    const double bn = orc3_leafnorm(r, b, t);
    const double scale = bn > 0 ? bn : 1.0;
    double x = orc3_resnorm(r, b, u, s, t, op) / scale;
    int c = 0;
    while (x > tol && c < max_cycles) {
        orc3_vcycle(u, b, r, u1, s, t, op, 0, ndown, ntop, nup, omega);
        c++;
        x = orc3_resnorm(r, b, u, s, t, op) / scale;
    }
    if (rel) *rel = x;
    return c;
}
