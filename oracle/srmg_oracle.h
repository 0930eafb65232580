/*
 * srmg_oracle.h -- CPU FP64 restatement of Steamroller.jl's multigrid field solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle that the CUDA library is checked
 * against, and the timed CPU baseline.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load it.  The product library never
 * links, calls or falls back to it.
 *
 * Parity status: UNPINNED against the reference.  Steamroller.jl ships no tests, no
 * golden vectors and no fixtures, and the reference (pure Julia) cannot run in this
 * image (no Julia toolchain).  The restatement follows the reference source op by op
 * (file:line cited on every function) and is itself checked against derived
 * known-answer tests (exact stencil identities, transfer-operator identities) in
 * tests/test_oracle_kat.py.
 *
 * Storage (src/blockfield.jl:33-40, 223-227): a field is nblk contiguous blocks of
 * S x S doubles, S = M + 2G, column-major with dim 1 (r) fastest.  Element
 * (i, j, blk) (1-based, as in Julia) lives at (i-1) + S*(j-1) + S*S*(blk-1).
 *
 * Edge structs mirror the isbits layout of the Julia structs in
 * src/connectivity.jl:6-42 and Pair{CartesianIndex{2},Int} of src/blocklayer.jl:23.
 * All indices are 1-based, as in Julia.
 */
#ifndef SRMG_ORACLE_H
#define SRMG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { int64_t coord[2]; int64_t blk; } orc_pair;
typedef struct { int64_t from, to; int64_t face[2]; } orc_neighbor;
typedef struct { int64_t block; int64_t face[2]; int64_t bnd[2]; int64_t level; } orc_boundary;
typedef struct { int64_t fine, coarse; int64_t face[2]; int64_t subblock[2]; } orc_refbnd;
typedef struct { int64_t fine, coarse; int64_t subblock[2]; } orc_child;

/* A tree plus its connectivity, one array per level (level l at index l-1). */
typedef struct {
    int M, G;
    int nlev;
    const int64_t *npairs;  const orc_pair *const *pairs;
    const int64_t *nnb;     const orc_neighbor *const *nb;
    const int64_t *nbd;     const orc_boundary *const *bd;
    const int64_t *nrb;     const orc_refbnd *const *rb;
    const int64_t *nch;     const orc_child *const *ch;
    /* blk -> coord map (index blk-1), coords 1-based; filled by orc_tree_index */
    int64_t nblk_alloc;
    int64_t *coord_of;      /* 2 * nblk_alloc entries, owned by the caller */
} orc_tree;

/* Operator: op 0 = LaplacianDiscretization{D,2}, 1 = HelmholtzDiscretization{D,2}(k2),
 * 2 = LaplacianDiscretization{D,4} (compact order 4; needs a BoxStencil connectivity).
 * geom 0 = CartesianGeometry, 1 = CylindricalGeometry{1}, 2 = CylindricalGeometry{2}
 * (D = 3: Cartesian only).  bc: the 3x3 table (D = 2), bc27: the 3x3x3 table (D = 3),
 * both column-major. */
typedef struct { int op; double k2; int geom; int8_t bc[9]; int8_t bc27[27]; } orc_operator;

/* D = 3: the isbits layouts of Pair{CartesianIndex{3},Int}, Neighbor{3}, Boundary{3},
 * RefBoundary{3}, Child{3} (src/blocklayer.jl:23, src/connectivity.jl:6-42). */
typedef struct { int64_t coord[3]; int64_t blk; } orc3_pair;
typedef struct { int64_t from, to; int64_t face[3]; } orc3_neighbor;
typedef struct { int64_t block; int64_t face[3]; int64_t bnd[3]; int64_t level; } orc3_boundary;
typedef struct { int64_t fine, coarse; int64_t face[3]; int64_t subblock[3]; } orc3_refbnd;
typedef struct { int64_t fine, coarse; int64_t subblock[3]; } orc3_child;

typedef struct {
    int M, G;
    int nlev;
    const int64_t *npairs;  const orc3_pair *const *pairs;
    const int64_t *nnb;     const orc3_neighbor *const *nb;
    const int64_t *nbd;     const orc3_boundary *const *bd;
    const int64_t *nrb;     const orc3_refbnd *const *rb;
    const int64_t *nch;     const orc3_child *const *ch;
    int64_t nblk_alloc;
    int64_t *coord_of;      /* 3 * nblk_alloc entries, owned by the caller */
} orc3_tree;

void orc3_tree_index(orc3_tree *t);
void orc3_fill_ghost_copy(double *u, const orc3_tree *t, int l);
void orc3_fill_ghost_bnd(double *u, const orc3_tree *t, int l, const int8_t bc[27]);
void orc3_fill_ghost_interp(double *u, const orc3_tree *t, int l);
void orc3_fill_ghost(double *u, const orc3_tree *t, int l, const int8_t bc[27]);
void orc3_restrict_level(double *u, const orc3_tree *t, int l);
void orc3_interp_add_level(double *u, const double *u1, const orc3_tree *t, int l);
void orc3_copyto_level(double *dst, const double *src, const orc3_tree *t, int l);
void orc3_diffto_level(double *dst, const double *a1, const double *a2, const orc3_tree *t, int l);
void orc3_gs_level(double *u, const double *b, double omega, double s, const orc3_tree *t, int l,
                   const orc_operator *op, int parity);
void orc3_gs4_level(double *u, const double *b, double omega, double s, const orc3_tree *t, int l,
                    const orc_operator *op, int P1, int P2);
void orc3_gs_iter(double *u, const double *b, double omega, double s, int n, int l, const orc3_tree *t,
                  const orc_operator *op);
void orc3_residual_level(double *r, const double *u, const double *b, double s, const orc3_tree *t, int l,
                         const orc_operator *op);
void orc3_residual_postrestrict_level(double *bfield, const double *u, const double *r, double s,
                                      const orc3_tree *t, int l, const orc_operator *op);
void orc3_rhs_level(double *q1, const double *q, const orc3_tree *t, int l, const orc_operator *op);
void orc3_vcycle(double *u, double *b, double *r, double *u1, double s, const orc3_tree *t, const orc_operator *op,
                 int lmax, int ndown, int ntop, int nup, double omega);
void orc3_fmg(double *u, double *b, double *r, double *u1, double s, const orc3_tree *t, const orc_operator *op,
              int ndown, int ntop, int nup, double omega);
double orc3_resnorm(double *r, const double *b, const double *u, double s, const orc3_tree *t,
                    const orc_operator *op);
double orc3_leafnorm(double *scratch, const double *f, const orc3_tree *t);
int orc3_solve(double *u, double *b, double *r, double *u1, double s, const orc3_tree *t, const orc_operator *op,
               int ndown, int ntop, int nup, double omega, double tol, int max_cycles, double *rel);

void orc_tree_index(orc_tree *t);

void orc_fill_ghost_copy(double *u, const orc_tree *t, int l);
void orc_fill_ghost_bnd(double *u, const orc_tree *t, int l, const int8_t bc[9]);
void orc_fill_ghost_interp(double *u, const orc_tree *t, int l);
void orc_fill_ghost(double *u, const orc_tree *t, int l, const int8_t bc[9]);

void orc_restrict_level(double *u, const orc_tree *t, int l);
void orc_restrict_full(double *u, const orc_tree *t);
void orc_interp_add_level(double *u, const double *u1, const orc_tree *t, int l);
void orc_copyto_level(double *dst, const double *src, const orc_tree *t, int l);
void orc_diffto_level(double *dst, const double *a1, const double *a2, const orc_tree *t, int l);

void orc_gs_level(double *u, const double *b, double omega, double s, const orc_tree *t, int l,
                  const orc_operator *op, int parity);
void orc_gs4_level(double *u, const double *b, double omega, double s, const orc_tree *t, int l,
                   const orc_operator *op, int p1, int p2);
void orc_gs_iter(double *u, const double *b, double omega, double s, int n, int l,
                 const orc_tree *t, const orc_operator *op);
void orc_residual_level(double *r, const double *u, const double *b, double s,
                        const orc_tree *t, int l, const orc_operator *op);
void orc_residual_postrestrict_level(double *bfield, const double *u, const double *r, double s,
                                     const orc_tree *t, int l, const orc_operator *op);

void orc_vcycle(double *u, double *b, double *r, double *u1, double s, const orc_tree *t,
                const orc_operator *op, int lmax, int ndown, int ntop, int nup, double omega);
void orc_fmg(double *u, double *b, double *r, double *u1, double s, const orc_tree *t,
             const orc_operator *op, int ndown, int ntop, int nup, double omega);
double orc_resnorm(double *r, const double *b, const double *u, double s, const orc_tree *t,
                   const orc_operator *op);
double orc_leafnorm(double *scratch, const double *f, const orc_tree *t);

/* Tolerance loop built on vcycle + resnorm (not present in the reference, which runs a
 * fixed number of cycles): cycles until resnorm(u)/leafnorm(b) <= tol or max_cycles.
 * Returns cycles run; *rel gets the final relative residual. */
int orc_solve(double *u, double *b, double *r, double *u1, double s, const orc_tree *t,
              const orc_operator *op, int ndown, int ntop, int nup, double omega,
              double tol, int max_cycles, double *rel);

/* Stage preparation and post-processing of derivs! (src/streamer.jl:309-351). */
void orc_rhs_level(double *q1, const double *q, const orc_tree *t, int l, const orc_operator *op);
void orc_netcharge(double *q, const double *ne, const double *nion, const orc_tree *t);
void orc_electric_field(double *e, double *eabs, const double *u, double h, const double e0[2],
                        const orc_tree *t);

void orc_set_threads(int n);
int orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
