/*
 * srmg.h -- C ABI of libsrmg, the B200-native (sm_100a) FAS multigrid field solve for
 * Steamroller.jl block trees.
 *
 * The library replaces the bodies of the Julia entry points
 *     vcycle!(u, b, r, u1, s, tree, conn, geometry, bc, lpldisc;
 *             lmax=0, ndown=3, ntop=5, nup=3, omega=1.0)      src/multigrid.jl:60-106
 *     fmg!(u, b, r, u1, s, tree, conn, geometry, bc, lpldisc;
 *          lmax=0, ndown=3, ntop=5, nup=3, omega=1.25)        src/multigrid.jl:17-51
 * and the helpers they call.  Julia keeps the tree and the fields; it passes them
 * through ccall as plain pointers:
 *   - fields: ScalarBlockField{2,M,G,Float64} contiguous storage
 *     (src/blockfield.jl:33-40): nblk blocks of S x S doubles, S = M + 2G, dim 1 (r)
 *     fastest; element (i, j, blk), 1-based, at (i-1) + S(j-1) + S*S(blk-1);
 *   - the tree: BlockLayer.pairs per level (src/blocklayer.jl:23);
 *   - connectivity: the four edge vectors per level (src/connectivity.jl:51-64).
 * Edge structs below are the isbits layouts of the Julia structs, so Julia vectors
 * are passed without conversion.  All block indices and coordinates are 1-based.
 *
 * Supported: D = 2, M = 16, G = 2, order-2 Laplacian / Helmholtz discretisations
 * and the compact order-4 Laplacian, Cartesian and cylindrical geometries,
 * homogeneous boundary conditions (GeneralHomogeneousBoundaryConditions,
 * src/boundary.jl:21-38), and a StarStencil or BoxStencil connectivity
 * (src/connectivity.jl:106-149; the BoxStencil one adds diagonal edges that fill the
 * 2 x 2 corner ghosts).  Anything else returns SRMG_ERR_UNSUPPORTED and the Julia shim
 * keeps the original Julia method.
 *
 * Every entry point returns SRMG_OK (0) or a negative SRMG_ERR_* code;
 * srmg_last_error() gives the message.  A context is not thread-safe; distinct
 * contexts may be used from distinct threads.
 */
#ifndef SRMG_H
#define SRMG_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SRMG_OK               0
#define SRMG_ERR_BADARG      -1
#define SRMG_ERR_BADTREE     -2
#define SRMG_ERR_CUDA        -3
#define SRMG_ERR_TIMEOUT     -4
#define SRMG_ERR_DIVERGED    -5
#define SRMG_ERR_UNSUPPORTED -6
#define SRMG_ERR_NOMEM       -7
#define SRMG_ERR_NOTREE      -8

/* lpldisc: LaplacianDiscretization{2,2} / HelmholtzDiscretization{2,2}(k2)
 * (src/laplacian.jl:14, src/helmholtz.jl:9-11), and LaplacianDiscretization{2,4}, the
 * compact order-4 scheme (src/laplacian.jl:131-209): 9-point left-hand side, 5-point
 * right-hand side applied by srmg_rhs_level, four-colour Gauss-Seidel
 * (src/multigrid.jl:206-232, 268-295).  Order 4 needs a tree set with a BoxStencil
 * connectivity and runs FP64 on the per-operation kernels (vcycle, fmg, resnorm,
 * FP64 srmg_solve); mixed precision, batches and the autotuner return
 * SRMG_ERR_UNSUPPORTED for it. */
#define SRMG_OP_LAPLACIAN 0
#define SRMG_OP_HELMHOLTZ 1
#define SRMG_OP_LAPLACIAN4 2
/* geometry: CartesianGeometry, CylindricalGeometry{1}, CylindricalGeometry{2}
 * (src/geometry.jl:14-20). */
#define SRMG_GEOM_CARTESIAN 0
#define SRMG_GEOM_CYL1      1
#define SRMG_GEOM_CYL2      2

/* Pair{CartesianIndex{2},Int}: coord => blk (src/blocklayer.jl:23). */
typedef struct { int64_t coord[2]; int64_t blk; } srmg_pair;
/* Neighbor{2} (src/connectivity.jl:14-20): ghost face -face of `to` <- `from`. */
typedef struct { int64_t from, to; int64_t face[2]; } srmg_neighbor;
/* Boundary{2} (src/connectivity.jl:6-11). */
typedef struct { int64_t block; int64_t face[2]; int64_t bnd[2]; int64_t level; } srmg_boundary;
/* RefBoundary{2} (src/connectivity.jl:23-32). */
typedef struct { int64_t fine, coarse; int64_t face[2]; int64_t subblock[2]; } srmg_refbnd;
/* Child{2} (src/connectivity.jl:36-42). */
typedef struct { int64_t fine, coarse; int64_t subblock[2]; } srmg_child;

typedef struct srmg_ctx srmg_ctx;

/* Create a context on CUDA device `device` (M = 16, G = 2; D = 2, or D = 3 for a
 * three-dimensional tree).  The context owns a CUDA stream, the device copy of the tree
 * and the device mirrors of fields passed through the host-pointer entry points.  No
 * counterpart in the reference (its state lives in Julia objects).
 * D = 3 (Cartesian, the only geometry with 3D stencils in the reference,
 * src/laplacian.jl:274-340, src/helmholtz.jl:74-100): the tree is set with
 * srmg_set_tree3; fields are 20^3 doubles per block (i fastest, then j, then k);
 * boundary tables have 27 entries (a[2+b1, 2+b2, 2+b3], column-major); ops 0, 1 and 2
 * (order 4 needs a BoxStencil{3} connectivity).  The multigrid entry points (vcycle,
 * fmg, resnorm, the ghost fills and per-level operations, rhs_level, FP64 srmg_solve)
 * run on the per-operation kernels in FP64; the other entry points return
 * SRMG_ERR_UNSUPPORTED for a D = 3 context. */
int srmg_create(srmg_ctx **ctx, int D, int M, int G, int device);
void srmg_destroy(srmg_ctx *ctx);
const char *srmg_last_error(const srmg_ctx *ctx);

/* Replace the CUDA stream the context launches on (NULL = the context's own stream).
 * The *_dev entry points are stream-ordered on it. */
int srmg_set_stream(srmg_ctx *ctx, void *cuda_stream);
int srmg_synchronize(srmg_ctx *ctx);

/* Upload tree + connectivity (replaces reading `tree`/`conn` inside vcycle!).
 * Arrays are indexed by level (level l at index l-1).  `generation` lets callers skip
 * re-uploads: the Julia shim bumps it whenever connectivity!/refine! runs
 * (src/streamer.jl:545-549).  Validates indices and nesting; a face written by two
 * edges, an index out of range or a non-star face gives SRMG_ERR_BADTREE. */
int srmg_set_tree(srmg_ctx *ctx, int nlev,
                  const int64_t *npairs, const srmg_pair *const *pairs,
                  const int64_t *nneighbor, const srmg_neighbor *const *neighbor,
                  const int64_t *nboundary, const srmg_boundary *const *boundary,
                  const int64_t *nrefbnd, const srmg_refbnd *const *refbnd,
                  const int64_t *nchild, const srmg_child *const *child,
                  uint64_t generation);
uint64_t srmg_tree_generation(const srmg_ctx *ctx);

/* D = 3: the isbits layouts of Pair{CartesianIndex{3},Int}, Neighbor{3}, Boundary{3},
 * RefBoundary{3} and Child{3} (src/blocklayer.jl:23, src/connectivity.jl:6-42). */
typedef struct { int64_t coord[3]; int64_t blk; } srmg_pair3;
typedef struct { int64_t from, to; int64_t face[3]; } srmg_neighbor3;
typedef struct { int64_t block; int64_t face[3]; int64_t bnd[3]; int64_t level; } srmg_boundary3;
typedef struct { int64_t fine, coarse; int64_t face[3]; int64_t subblock[3]; } srmg_refbnd3;
typedef struct { int64_t fine, coarse; int64_t subblock[3]; } srmg_child3;
/* srmg_set_tree for a context created with D = 3 (any face in {-1,0,1}^3 but the
 * origin: StarStencil{3} or BoxStencil{3} connectivity). */
int srmg_set_tree3(srmg_ctx *ctx, int nlev,
                   const int64_t *npairs, const srmg_pair3 *const *pairs,
                   const int64_t *nneighbor, const srmg_neighbor3 *const *neighbor,
                   const int64_t *nboundary, const srmg_boundary3 *const *boundary,
                   const int64_t *nrefbnd, const srmg_refbnd3 *const *refbnd,
                   const int64_t *nchild, const srmg_child3 *const *child,
                   uint64_t generation);

/* ---- the ccall boundary: HOST pointers (Julia-owned arrays) --------------------- */

/* `ncycles` x vcycle! (src/multigrid.jl:60-106) on host arrays of nblk_alloc blocks.
 * u is in/out exactly as in the reference, ghosts included.  b: its leaf cells are
 * never written; the reference leaves the FAS right-hand side in the covered cells of
 * the coarse levels, which none of its callers reads (derivs! re-restricts q before
 * every solve, src/streamer.jl:313-318, and vcycle! overwrites those cells before it
 * reads them), so by default b is not copied back and its covered cells keep the
 * caller's values (option "b_copy_back" 1 copies the FAS values back as the reference
 * leaves them).  r and u1 are scratch and are not written back.  Blocks until u is
 * back in host memory.  Host ranges registered with srmg_host_register are copied by
 * DMA at full bandwidth.  bc is the 3x3 Int8 table of
 * GeneralHomogeneousBoundaryConditions, column-major (src/boundary.jl:28-38). */
int srmg_vcycle(srmg_ctx *ctx, double *u, double *b, double *r, double *u1, int64_t nblk_alloc,
                double s, int op, double k2, int geom, const int8_t bc[9],
                int lmax, int ndown, int ntop, int nup, double omega, int ncycles);

/* fmg! (src/multigrid.jl:17-51) on host arrays; u in/out, b as in srmg_vcycle, r and
 * u1 scratch. */
int srmg_fmg(srmg_ctx *ctx, double *u, double *b, double *r, double *u1, int64_t nblk_alloc,
             double s, int op, double k2, int geom, const int8_t bc[9],
             int ndown, int ntop, int nup, double omega);

/* Page-lock a host range of the caller (cudaHostRegister) so that the host-array entry
 * points copy it by DMA at full bandwidth instead of staging it through the driver's
 * pageable-copy buffer.  Meant for the Julia-owned field storage (the ElasticArray
 * data of a ScalarBlockField, src/blockfield.jl:33-40) that srmg_vcycle / srmg_fmg
 * receive on every call.  The range stays registered until srmg_host_unregister or
 * srmg_destroy; the caller must not free it before (when newblock! resizes a field,
 * src/blockfield.jl:255-260, unregister the old pointer).  Registering the same
 * (ptr, bytes) twice is a no-op. */
int srmg_host_register(srmg_ctx *ctx, void *ptr, int64_t bytes);
int srmg_host_unregister(srmg_ctx *ctx, void *ptr);

/* resnorm! (src/multigrid.jl:391-417): *out = sqrt(sum over leaf cells of r^2 scaled
 * by 4^-(l-1)), with r = -(b + L u / s_l) on every level.  r is scratch. */
int srmg_resnorm(srmg_ctx *ctx, double *r, const double *b, const double *u, int64_t nblk_alloc,
                 double s, int op, double k2, int geom, const int8_t bc[9], double *out);

/* fill_ghost!(u, level, conn, bc) (src/connectivity.jl:155-159) on a host array. */
int srmg_fill_ghost(srmg_ctx *ctx, double *u, int64_t nblk_alloc, int level, const int8_t bc[9]);

/* Solve L u + s b = 0 to a relative residual: resnorm(u) / leafnorm(b) <= tol, where
 * leafnorm is the resnorm! norm applied to b.  The reference has no tolerance loop
 * (it runs poisson_iter fixed V-cycles, src/streamer.jl:322-334); this is the loop
 * built on its vcycle!/resnorm! semantics.
 *   mode SRMG_MODE_FP64 : repeated reference V-cycles in FP64 (bit-for-bit the
 *                         vcycle! algorithm), residual checked after each cycle;
 *   mode SRMG_MODE_MIXED: FP64 defect correction around FP32 V-cycles (smoothing,
 *                         restriction, prolongation in FP32), FP64 residual, FP64
 *                         coarsest-level direct solve and FP64 norms;
 *   mode SRMG_MODE_FP64_DIRECT: the FP64 V-cycles of SRMG_MODE_FP64 with the
 *                         coarsest level solved directly by the same FP64 inverse as
 *                         the mixed mode, in place of the ntop sweeps (not the
 *                         reference's algorithm: it separates the effect of the
 *                         precision from that of the coarse solve; order 2, 2D, the
 *                         persistent engine only).
 * u holds the initial guess on entry (ghosts filled) and the solution on exit
 * (ghosts filled); b is read-only in every mode. */
#define SRMG_MODE_FP64  0
#define SRMG_MODE_MIXED 1
#define SRMG_MODE_FP64_DIRECT 2
typedef struct {
    double tol;          /* relative residual target, e.g. 1e-8 */
    int max_cycles;      /* cap on V-cycles (FP64) or outer steps (mixed) */
    int mode;            /* SRMG_MODE_* */
    int ndown, ntop, nup;
    double omega;
    int inner_cycles;    /* mixed: at most this many FP32 V-cycles per defect-correction step
                            (>= 1; default 2); the engine runs one per decade between the
                            defect norm and the tolerance, up to this cap */
    int warm_start;      /* 0: start from u; 1: learned initial guess (srmg_cnn_*) */
} srmg_solve_opts;

typedef struct {
    int status;          /* SRMG_OK or an error code */
    int cycles;          /* V-cycles run (FP64 or FP32) */
    int outer;           /* defect-correction steps (mixed), 0 in FP64 mode */
    double rel_residual; /* final resnorm(u)/leafnorm(b) */
    double initial_rel;  /* before the first cycle */
    double bnorm;        /* leafnorm(b) */
    double device_ms;    /* device time of the solve (CUDA events) */
} srmg_stats;

void srmg_solve_opts_default(srmg_solve_opts *opts);
int srmg_solve(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc,
               double s, int op, double k2, int geom, const int8_t bc[9],
               const srmg_solve_opts *opts, srmg_stats *stats);

/* srmg_solve in two calls.  No counterpart in the reference, whose solves are
 * synchronous calls on host arrays: it exists for callers with several independent
 * problems, whose host-to-device and device-to-host copies (the bulk of a host-array
 * solve's time on the PCIe link) can overlap another problem's solve.
 * srmg_solve_async enqueues on the context's stream the copies of u and b in, the
 * solve, and the copy of u out, and returns without waiting; srmg_solve_wait(ctx,
 * stats) waits for them, fills stats (device_ms spans the copies and the solve) and
 * returns what srmg_solve would have returned.  u and b must stay valid and untouched
 * until the wait, and should be page-locked (srmg_host_register, or pinned memory) for
 * the copies to run asynchronously.  Between the two calls the context takes no other
 * call (SRMG_ERR_BADARG); two contexts holding the same tree give two solves in flight,
 * whose kernels run one after the other while their copies overlap.  Single 2D trees
 * on the persistent engine only (SRMG_ERR_UNSUPPORTED otherwise: use srmg_solve), no
 * learned warm start.  Results equal srmg_solve's bit for bit. */
int srmg_solve_async(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc,
                     double s, int op, double k2, int geom, const int8_t bc[9],
                     const srmg_solve_opts *opts);
int srmg_solve_wait(srmg_ctx *ctx, srmg_stats *stats);

/* ---- DEVICE pointers (fields already resident in HBM) --------------------------- */
/* Same semantics as the host entry points; pointers are device addresses of
 * nblk_alloc-block fields; work is ordered on the context's stream and these calls
 * return without synchronising (except solve/resnorm, which read a norm back). */
int srmg_vcycle_dev(srmg_ctx *ctx, double *u, double *b, double *r, double *u1,
                    int64_t nblk_alloc, double s, int op, double k2, int geom,
                    const int8_t bc[9], int lmax, int ndown, int ntop, int nup,
                    double omega, int ncycles);
int srmg_fmg_dev(srmg_ctx *ctx, double *u, double *b, double *r, double *u1, int64_t nblk_alloc,
                 double s, int op, double k2, int geom, const int8_t bc[9],
                 int ndown, int ntop, int nup, double omega);
int srmg_resnorm_dev(srmg_ctx *ctx, double *r, const double *b, const double *u,
                     int64_t nblk_alloc, double s, int op, double k2, int geom,
                     const int8_t bc[9], double *out);
int srmg_solve_dev(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc,
                   double s, int op, double k2, int geom, const int8_t bc[9],
                   const srmg_solve_opts *opts, srmg_stats *stats);

/* Single reference routines on device fields (used for per-operation parity). */
/* fill_ghost! parts (src/connectivity.jl:155-159): mask bit 0 = fill_ghost_copy!,
 * bit 1 = fill_ghost_bnd!, bit 2 = fill_ghost_interp!; 7 = fill_ghost!.  Bit 3 with bit
 * 2 makes the refinement ghosts InterpCopy ones (src/interp.jl:66-85: each coarse
 * cell's value copied into the 2 x 2 fine ghosts it covers), as derivs! fills the
 * electron density (src/streamer.jl:343); StarStencil trees only. */
int srmg_fill_ghost_dev(srmg_ctx *ctx, double *u, int64_t nblk_alloc, int level,
                        const int8_t bc[9], int mask);
/* gauss_seidel_level!(..., RedBlack{parity}) (src/multigrid.jl:238-243); for
 * SRMG_OP_LAPLACIAN4, FourColors{parity >> 1, parity & 1} with parity 0..3
 * (src/multigrid.jl:206-232). */
int srmg_gs_level_dev(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, int level,
                      double omega, double sl, int op, double k2, int geom, int parity);
/* gauss_seidel_iter! (src/multigrid.jl:250-265). */
int srmg_gs_iter_dev(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc, int level,
                     double omega, double sl, int n, int op, double k2, int geom,
                     const int8_t bc[9]);
/* residual_level! (src/multigrid.jl:349-354). */
int srmg_residual_level_dev(srmg_ctx *ctx, double *r, const double *u, const double *b,
                            int64_t nblk_alloc, int level, double sl, int op, double k2, int geom);
/* restrict_level!(u, conn.child[level]) (src/restrict.jl:31-37). */
int srmg_restrict_level_dev(srmg_ctx *ctx, double *u, int64_t nblk_alloc, int level);
/* interp_add_level!(u, u1, conn.child[level]) (src/interp.jl:107-115). */
int srmg_interp_add_level_dev(srmg_ctx *ctx, double *u, const double *u1, int64_t nblk_alloc,
                              int level);
/* residual_postrestrict_level!(b, u, r, s, tree[level-1], conn.child[level], ...)
 * (src/multigrid.jl:112-119); s is the coarse-level scale. */
int srmg_residual_postrestrict_level_dev(srmg_ctx *ctx, double *b, const double *u,
                                         const double *r, int64_t nblk_alloc, int level,
                                         double s, int op, double k2, int geom);

/* ---- stage preparation and post-processing on the device --------------------------
 * The work around the field solve inside derivs! (src/streamer.jl:309-351), so that a
 * time step can keep u, q and n on the device. */
/* netcharge!(tree, q, n, chem) (src/streamer.jl:369-373) for the NetIonization
 * chemistry (src/chemistry.jl:80: charges -1 for electrons, +1 for ions): q = -ne + nion
 * on every valid cell of every block.  For order-2 discretisations rhs_level!
 * (src/multigrid.jl:363-388) is the identity, so q is the solve's right-hand side. */
int srmg_netcharge(srmg_ctx *ctx, double *q, const double *ne, const double *nion, int64_t nblk_alloc);
int srmg_netcharge_dev(srmg_ctx *ctx, double *q, const double *ne, const double *nion, int64_t nblk_alloc);
/* restrict_full!(u, conn) (src/restrict.jl:43-47): restrict_level! for levels L..2. */
int srmg_restrict_full_dev(srmg_ctx *ctx, double *u, int64_t nblk_alloc);
/* rhs_level!(q1, q, tree[level], lpldisc, geometry) (src/multigrid.jl:363-388): q1 = R q
 * on the valid cells of every block of the level; R is the identity for order 2 and
 * the compact 5-point right-hand side (divided by 12) for SRMG_OP_LAPLACIAN4.  q's
 * ghosts must be filled.  Bit-exact.  derivs! (src/streamer.jl:314-318) calls it per
 * level between fill_ghost!(q) and fill_ghost!(q1). */
int srmg_rhs_level(srmg_ctx *ctx, double *q1, const double *q, int64_t nblk_alloc, int level, int op,
                   int geom);

/* ---- free boundary conditions on the radial boundary (FreeBC, src/freebc.jl) --------
 * derivs! (src/streamer.jl:320) solves the homogeneous potential uh (srmg_vcycle /
 * srmg_fmg with the same right-hand side), then freebc! adds boundary sources to the
 * right-hand side; after the main solve fill_ghost_free! (src/streamer.jl:348) adds the
 * boundary values to u's first outer ghost layer.  The tree of the context must be one
 * tree (not a forest) with no level above `level`.
 * srmg_freebc_set: FreeBC(CylindricalGeometry{dim}, u, level, rootsize, h)
 * (src/freebc.jl:29-53) -- dim 1 or 2 is the radial dimension, rootsize the root block
 * grid, f the transform kernel FreeBC computes (n = rootsize[other] 2^(level-1) 16
 * values).  The library keeps a copy; call again when the FreeBC changes. */
int srmg_freebc_set(srmg_ctx *ctx, int dim, int level, const int64_t rootsize[2], const double *f, int64_t n);
/* freebc!(q, u, h, s, tree, conn, conf) (src/freebc.jl:83-105): q += the boundary
 * sources computed from u's outer cells (getouter!, DST-II, times f, DST-III,
 * setouter! with its refinement-boundary corrections).  b_out (n doubles, may be NULL)
 * receives conf.b; the library keeps b for srmg_fill_ghost_free.  The transforms run
 * as direct FP64 sums (n <= 131072). */
int srmg_freebc(srmg_ctx *ctx, double *q, const double *u, int64_t nblk_alloc, double h, double s, double *b_out);
int srmg_freebc_dev(srmg_ctx *ctx, double *q, const double *u, int64_t nblk_alloc, double h, double s,
                    double *b_out);
/* fill_ghost_free!(u, conf, tree, level) (src/freebc.jl:224-243) with the b of the last
 * srmg_freebc call. */
int srmg_fill_ghost_free(srmg_ctx *ctx, double *u, int64_t nblk_alloc, int level);
int srmg_fill_ghost_free_dev(srmg_ctx *ctx, double *u, int64_t nblk_alloc, int level);
int srmg_rhs_level_dev(srmg_ctx *ctx, double *q1, const double *q, int64_t nblk_alloc, int level, int op,
                       int geom);
/* electric_field!(tree, e, eabs, u, h, t, e0) (src/multigrid.jl:421-449, the method for
 * a constant background field e0 = (e0_r, e0_z), :451).  e is a VectorBlockField{2,16,2}:
 * 21 x 21 x 2 doubles per block (component d at offset 441 d); for d = r, z and every
 * face I of validindices(e, d) (src/blockfield.jl:403-405), e[I, d] = (u[I - e_d] -
 * u[I]) / h_l + e0[d] with h_l = h / 2^(l-1); eabs (20 x 20 per block) at every valid
 * cell = sqrt(sum_d (e[I, d] + e[I + e_d, d])^2 / 4).  u's ghosts must be filled.
 * Bit-exact against the reference's arithmetic (IEEE division and square root, no
 * fused multiply-add). */
int srmg_electric_field(srmg_ctx *ctx, double *e, double *eabs, const double *u, int64_t nblk_alloc,
                        double h, const double e0[2]);
int srmg_electric_field_dev(srmg_ctx *ctx, double *e, double *eabs, const double *u, int64_t nblk_alloc,
                            double h, const double e0[2]);

/* Self-test of the failure path of the persistent kernels' grid barrier (no reference
 * counterpart): one cooperative launch in which every CTA but one enters a grid
 * barrier whose bounded wait is limited to timeout_ms (1..2000); the missing CTA makes
 * the wait run out, the kernel records it in the context's error word and returns.
 * Returns SRMG_ERR_TIMEOUT (the status a stuck barrier of a solve reports), or
 * SRMG_ERR_BADARG.  Nothing faults or hangs; the context stays usable. */
int srmg_selftest_barrier_timeout(srmg_ctx *ctx, int timeout_ms);

/* Allocation-free residual norm.  No counterpart in the reference: it exists for
 * callers that cannot call cudaMalloc when they need the norm -- hosts whose device
 * memory belongs to their own pool allocator, or loops that cannot take an
 * allocation's implicit synchronisation.  Same value as srmg_resnorm_dev up to
 * summation order, but it calls no cudaMalloc/cudaFree or allocating library routine:
 * its scratch (one partial sum per tree block) is a static device array of 65536
 * doubles (512 KiB), held by every GPU that loads the library until the process
 * exits.  Trees of more than 65536 blocks are rejected with SRMG_ERR_BADARG; 2D trees
 * only (SRMG_ERR_UNSUPPORTED for D = 3).  `out` is a DEVICE address that receives the
 * norm, stream-ordered on the context's stream; nothing is copied to the host.  The
 * array is shared by all calls and keeps the last call's contents; calls that overlap
 * on the GPU (several streams or contexts at once) race on it.  The first call on each
 * device looks up the array's device address and keeps it for the life of the process
 * (the device's primary context must outlive the calls: no use after a
 * cudaDeviceReset). */
int srmg_resnorm_noalloc(srmg_ctx *ctx, const double *b, const double *u, int64_t nblk_alloc,
                         double s, int op, double k2, int geom, double *out);

/* ---- batched solves: many independent problems in one persistent launch ----------
 * No single counterpart in the reference: it solves the Poisson potential
 * (src/streamer.jl:322-334) and each photoionization Helmholtz term (src/photo.jl,
 * one HelmholtzDiscretization per screening constant) with separate vcycle!/fmg!
 * calls, tree by tree.  A batch context holds a forest: one item per (tree,
 * operator) pair, every item with its own copy of its tree's blocks.  An item's
 * solve stops when its own relative residual reaches tol; the others continue, and
 * each item's result is the one srmg_solve_dev gives for it alone.
 * Limits: every item uses the persistent engine (option "engine" 1, sweep counts
 * >= 1, 16-byte aligned fields); at most 4 blocks on an item's level 1 for the
 * mixed mode's direct coarsest-level solve (more: smoothing at the top). */
typedef struct {
    const srmg_ctx *tree;  /* context whose uploaded tree the item solves on */
    double s;              /* scale s of L u + s b = 0 */
    int op;                /* SRMG_OP_LAPLACIAN or SRMG_OP_HELMHOLTZ */
    double k2;             /* Helmholtz k^2 (screening constant squared) */
    int8_t bc[9];          /* boundary table as in srmg_vcycle */
} srmg_item;

/* Build the forest of `batch` (a context created with srmg_create) from the items;
 * every item's tree context must stay alive only for this call (the trees are
 * copied).  All items share one geometry. */
int srmg_batch_set(srmg_ctx *batch, int nitems, const srmg_item *items, int geom);
int srmg_batch_items(const srmg_ctx *batch);
/* First block (0-based) and block count of item `item` in the forest layout: item
 * k's field occupies blocks [offset, offset + nblk) of a forest field, in its own
 * tree's block order.  -1 on a bad argument. */
int64_t srmg_batch_offset(const srmg_ctx *batch, int item);
int64_t srmg_batch_nblk(const srmg_ctx *batch, int item);
/* Solve every item.  u[k], b[k]: item k's DEVICE fields in its own tree's layout
 * (at least srmg_batch_nblk(batch, k) blocks); u in/out, b read-only.  stats: one
 * entry per item.  With option "graph" 1 the copies in and out and the solve are
 * captured in a CUDA graph on the first call and replayed by later calls with the
 * same pointers and options. */
int srmg_batch_solve_dev(srmg_ctx *batch, double *const *u, const double *const *b,
                         const srmg_solve_opts *opts, srmg_stats *stats);
/* The same on HOST fields (copied in and out inside the call). */
int srmg_batch_solve(srmg_ctx *batch, double *const *u, const double *const *b,
                     const srmg_solve_opts *opts, srmg_stats *stats);
/* The same on fields already in the forest layout (no copies). */
int srmg_batch_solve_forest_dev(srmg_ctx *batch, double *u, const double *b,
                                const srmg_solve_opts *opts, srmg_stats *stats);

/* ---- autotuner (no reference counterpart) ----------------------------------------
 * Times complete solves to opts->tol from the caller's initial guess for a set of
 * candidates, each solved twice: first the launch shape at the caller's sweeps and
 * omega -- engine_ctas (one CTA per SM or half as many: blocks per CTA) x
 * local_max_blocks (4, 16, 64: coarse levels kept inside one CTA), 6 candidates --
 * then, at the fastest shape, (ndown, nup) in {(2,2), (1,1), (1,2), (2,1), (3,3)} x the
 * Gauss-Seidel relaxation factor omega in {1, 1.1, 1.2}, 15 candidates; and for mixed
 * solves, at the fastest of those, the FP32 V-cycles per defect-correction step
 * (inner_cycles) in {1, 2, 3, 4}, 4 candidates.  The fastest candidate's options are set
 * on the context and its sweep counts, omega and inner_cycles written to *opts; u is
 * restored to its initial content.  Trials are reported in `trials` (up to max_trials).
 * Returns the number of trials run or an error code.  The tile shape is fixed: one
 * 20 x 20 block per 256-thread slot. */
typedef struct {
    int engine_ctas, local_max_blocks, ndown, nup, ntop;
    int cycles;          /* V-cycles (FP64) or defect-correction steps (mixed), worst item */
    double ms;           /* best device time of the trial, -1 if it missed the tolerance */
    double omega;        /* relaxation factor of the trial */
    int inner_cycles;    /* FP32 V-cycles per defect-correction step (mixed) */
} srmg_tune_trial;
int srmg_autotune(srmg_ctx *ctx, double *u, const double *b, int64_t nblk_alloc,
                  double s, int op, double k2, int geom, const int8_t bc[9],
                  srmg_solve_opts *opts, srmg_tune_trial *trials, int max_trials);
int srmg_batch_autotune(srmg_ctx *batch, double *const *u, const double *const *b,
                        srmg_solve_opts *opts, srmg_tune_trial *trials, int max_trials);

/* ---- learned warm start (no reference counterpart) --------------------------------
 * Successive time steps change the potential by nearly the same correction (the
 * streamer head moves a fraction of a cell per step), so the guess for step n is
 *   phi_{n-1} + delta_{n-1} + (learned change of the correction),
 * delta_{n-1} = phi_{n-1} - phi_{n-2}.  A 6-layer BF16 convolutional network (3x3
 * convolutions, 32 channels, ReLU; zero padding at the tile edge) maps, per block, the
 * 20 x 20 tile (16 x 16 cells plus the 2-cell ghost halo) of (delta_{n-1} a, g c),
 * g = b_n - 2 b_{n-1} + b_{n-2} the change of the charge change, a = 1/|delta_{n-1}|,
 * c = 1/|g| (|.| = the resnorm! leaf norm, per tree), to
 * (delta_n - delta_{n-1}) / (s_l |g|) on the block's 16 x 16 cells.  The network
 * predicts a small quantity, so BF16 precision does not limit the guess.  Forward,
 * backward and optimiser kernels run on the tensor cores; parameters are an FP32
 * master vector (per layer W [tap][co][ci], then b [co]). */
typedef struct srmg_cnn srmg_cnn;
int srmg_cnn_create(srmg_cnn **net, int device, uint64_t seed);  /* He-initialised */
void srmg_cnn_destroy(srmg_cnn *net);
const char *srmg_cnn_last_error(const srmg_cnn *net);
int srmg_cnn_nparams(void);
int srmg_cnn_get_params(srmg_cnn *net, float *host, int n);
int srmg_cnn_set_params(srmg_cnn *net, const float *host, int n);  /* resets Adam state */
int srmg_cnn_synchronize(srmg_cnn *net);
/* Samples: x DEVICE bf16 [n][400][2] (tile pixel y*20+x, channels (phi, db));
 * targets/outputs DEVICE float [n][16][16]. */
int srmg_cnn_forward(srmg_cnn *net, const uint16_t *x, float *y, int n);
/* Loss = mean over the n x 256 outputs of (y - t)^2 + lambda * mean over the 14 x 14
 * interior cells of rho^2, rho = L(y) + db channel of x: the residual the guess leaves,
 * in the output's units (L the geometry's stencil; ir0[k] = global r index before the
 * sample's first cell, DEVICE; ir0 NULL = no residual term).  Gradient in master
 * layout to grad_host if not NULL; loss to *loss (host). */
int srmg_cnn_gradients(srmg_cnn *net, const uint16_t *x, const float *t, const int *ir0,
                       float lambda, int geom, int n, float *grad_host, double *loss);
/* One Adam step (beta 0.9/0.999, eps 1e-8) on that loss over the n samples. */
int srmg_cnn_train_step(srmg_cnn *net, const uint16_t *x, const float *t, const int *ir0,
                        float lambda, int geom, int n, float lr, double *loss);
/* The same inference forward on the 5th-generation tensor cores (tcgen05 MMAs with
 * accumulators in tensor memory); srmg_cnn_tc_status synchronises and reports a timed-
 * out MMA completion wait; srmg_cnn_use_tcgen05 makes srmg_cnn_predict_dev use it. */
int srmg_cnn_forward_tc(srmg_cnn *net, const uint16_t *x, float *y, int n);
int srmg_cnn_tc_status(srmg_cnn *net);
int srmg_cnn_use_tcgen05(srmg_cnn *net, int enable);
/* Training against a loss computed by the caller: the forward pass keeps every layer's
 * activations and writes y (DEVICE float [n][256]); the backward pass takes dLoss/dy
 * (DEVICE float [n][256]) for the same n samples, and applies one Adam step when
 * lr > 0 (gradient in master layout to grad_host if not NULL). */
int srmg_cnn_forward_train(srmg_cnn *net, const uint16_t *x, int n, float *y);
int srmg_cnn_backward_step(srmg_cnn *net, const float *dy, int n, float lr, float *grad_host);
/* Tree fields -> samples, one per block holding a leaf cell (srmg_cnn_leaf_blocks of
 * them): x as above from the input fields f (ghosts filled) and g, scale[k] =
 * s_l |g| of the sample's block, blk[k] its 0-based block id.  DEVICE pointers;
 * returns the sample count. */
int srmg_cnn_leaf_blocks(const srmg_ctx *ctx);
int srmg_cnn_pack_dev(srmg_ctx *ctx, const double *f, const double *g, int64_t nblk_alloc,
                      double s, int op, double k2, int geom, const int8_t bc[9],
                      uint16_t *x, double *scale, int *blk, int max_samples);
/* Warm start for step n: u holds phi_{n-1} (ghosts filled) on entry; b = b_n,
 * b1 = b_{n-1}, phi2 = phi_{n-2}, b2 = b_{n-2}.  Three candidates -- phi_{n-1}, the
 * extrapolation phi_{n-1} + delta_{n-1}, and the extrapolation plus the network's
 * change -- are made composite-grid functions (ghosts filled); u receives the one with
 * the smallest residual norm and *which says which (0, 1, 2); resid (host, optional)
 * receives the three residual norms.  The solve then iterates to its tolerance from u
 * as usual. */
/* Blocks the network ran on in the last prediction whose `which` was read back. */
int srmg_cnn_last_active(const srmg_ctx *ctx);
int srmg_cnn_predict_dev(srmg_ctx *ctx, srmg_cnn *net, double *u, const double *b,
                         const double *b1, const double *phi2, const double *b2,
                         int64_t nblk_alloc, double s, int op, double k2, int geom,
                         const int8_t bc[9], int *which, double *resid);

/* ---- streamer transport for training data (derivs! and step!, src/streamer.jl) ----
 * The electron transport and chemistry inside derivs! (src/streamer.jl:292-366) with
 * the reference's default models, NetIonization (src/chemistry.jl:29-82, species
 * electrons and net positive ions, charges -1 and +1) over the MinimalTransportModel
 * (src/transport.jl:9-35) and a uniform gas density; no photoionization (the default
 * empty model).  The caller composes a stage as derivs! does: netcharge, restrict_full,
 * the Poisson solve, restrict_full(ne), ghost fills of ne (copy, fill_ghost_bnd! with the
 * fluid table, InterpCopy refinement ghosts: srmg_fill_ghost_dev mask 1|2|4|8) and of u,
 * srmg_electric_field_dev, fill_ghost!(eabs, ExtrapolateConst) (a table of +1 signs),
 * then srmg_streamer_flux_dev and srmg_streamer_rates_dev. */
typedef struct srmg_transport {
  double mu;   /* mobility (m^2 / V s) */
  double D;    /* diffusion coefficient (m^2 / s) */
  double ai;   /* ionisation: townsend = ai exp(-Ei / |E|) (1/m, V/m) */
  double Ei;
  double aa;   /* attachment = aa exp(-Ea / |E|) (1/m, V/m) */
  double Ea;
} srmg_transport;

/* flux!(tree, FluxSchemeKoren(), flux, ne, e, eabs, h, trans, dens, maxdt)
 * (src/fluid.jl:44-94) followed by restrict_flux!(flux, conn)
 * (src/connectivity.jl:327-360).  flux and e are VectorBlockField{2,16,2} (882
 * doubles per block, as srmg_electric_field_dev writes e); every face of every leaf
 * block is written, then each coarse face at a refinement boundary becomes the mean of
 * the two fine faces.  ne needs 2 ghost layers, eabs 1.  maxdt_blk (DEVICE, nblk_alloc
 * doubles, may be NULL) receives each leaf block's min(h/|v|, h^2/D/4, Maxwell time)
 * over its faces; maxdt_min (DEVICE, 1 double, may be NULL) their minimum over the leaf
 * blocks.  Fluxes and time steps are bit-exact against IEEE double arithmetic. */
int srmg_streamer_flux_dev(srmg_ctx *ctx, double *flux, double *maxdt_blk, double *maxdt_min,
                           const double *ne, const double *e, const double *eabs, int64_t nblk_alloc,
                           double h, const srmg_transport *tr);
/* chemderivs! (pre, init; post, add; src/chemistry.jl:29-82) and
 * fluxderivs!(tree, dne, flux, h, geom) (src/fluid.jl:8-30) on the valid cells of every
 * leaf block: dni = ionisation + attachment rate, dne = the same plus the flux
 * divergence with the geometry factors of src/geometry.jl:27-29 (geom as in
 * srmg_vcycle). */
int srmg_streamer_rates_dev(srmg_ctx *ctx, double *dne, double *dni, const double *ne, const double *eabs,
                            const double *flux, int64_t nblk_alloc, double h, int geom,
                            const srmg_transport *tr);
/* The SSPRK3 combinations of step! (src/streamer.jl:400-413), elementwise over `count`
 * doubles: stage 1 out = n + dn1 dt; stage 2 out = n + (dn1 dt/4 + dn2 dt/4); stage 3
 * out = n + ((dn1 dt/6 + dn2 dt/6) + dn3 (2 dt)/3).  Bit-exact (no fused
 * multiply-add).  out may alias n. */
int srmg_ssprk3_stage_dev(srmg_ctx *ctx, double *out, const double *n, const double *dn1, const double *dn2,
                          const double *dn3, int64_t count, double dt, int stage);

/* Tuning knobs (no reference counterpart; the autotuner drives them):
 *   "engine"           1 = persistent one-launch V-cycle (default), 0 = one kernel per
 *                      reference operation;
 *   "local_max_blocks" coarse levels whose every coarser level has at most this many
 *                      blocks run inside one CTA of the persistent kernel (default 4);
 *   "engine_ctas"      CTAs of the persistent kernel (0 = one per SM);
 *   "engine_threads"   threads per CTA of the persistent kernel: 768 (three slots, more
 *                      registers per thread) or 1024 (four slots); 0 (default) picks 768
 *                      for trees of up to 16384 blocks and 1024 above;
 *   "trace"            1 = record a %globaltimer stamp (ns) after every phase of the
 *                      persistent kernel, read back with srmg_get_trace;
 *   "graph"            1 = batched solves replay a captured CUDA graph;
 *   "op_graphs"        1 (default) = V-cycles on the per-operation kernels (3D trees,
 *                      BoxStencil trees, order 4, or "engine" 0) are captured once per
 *                      (fields, operator, sweep counts, tree, stream) into a CUDA graph
 *                      and replayed (bit-identical results; up to 8 graphs kept, all
 *                      dropped when the tree changes); 0 = launch kernel by kernel;
 *   "op_sequencer"     1 = those V-cycles are recorded once per key instead and run as
 *                      one cooperative launch that walks the recorded operations with
 *                      a grid barrier between consecutive ones (bit-identical results);
 *                      0 (default: graph replay measured faster on 2D and 3D trees);
 *   "gs_push"          1 (default) = on 2D trees off the persistent engine and on
 *                      BoxStencil{3} or order-4 octrees, every colour
 *                      sweep of gauss_seidel_iter! after its first writes the copy and
 *                      boundary ghosts of the cells it updates, instead of a fill launch
 *                      after it (bit-identical results; tables built once per tree from
 *                      the fill itself, trees whose fill the tables cannot express keep
 *                      the fill launches); 0 = a fill launch after every colour;
 *   "direct_level"     the level of the FP64 direct coarsest solve of mixed and
 *                      SRMG_MODE_FP64_DIRECT solves on the persistent kernel: 0 (default)
 *                      = level 2 for a lone tree whose level 2 holds 1..4 blocks and has no
 *                      refinement boundary (its 256..1024-row inverse is built on the host
 *                      once per operator, ~0.5 s at 1024 rows, and applied by every CTA),
 *                      else level 1 (one CTA); 1 = level 1 always (batches always use
 *                      level 1, so a solo solve matches its batched twin bit for bit only
 *                      with 1); 2 = level 2 where possible;
 *   "freebc_direct"    1 = srmg_freebc transforms by direct sums even for power-of-two
 *                      lengths (default 0: FFTs);
 *   "b_copy_back"      1 = srmg_vcycle / srmg_fmg copy b back to the host (the FAS
 *                      values in its covered cells, as the reference leaves them);
 *                      0 (default) = b is not copied back;
 *   "cnn_active_ppm"   the learned warm start runs the network only on blocks whose
 *                      share of (b_n - 2 b_{n-1} + b_{n-2})^2 is at least this many
 *                      millionths of the largest block's (default 0 = every
 *                      leaf-holding block); the others keep the extrapolation. */
int srmg_set_option(srmg_ctx *ctx, const char *key, int64_t value);

/* Phase timestamps of the last persistent-kernel launch (with option "trace" on);
 * returns the number of entries written to out (<= max_entries), or an error code. */
int srmg_get_trace(srmg_ctx *ctx, int64_t *out, int max_entries);

/* Number of CUDA kernel launches this context has issued (for launch accounting). */
int64_t srmg_launch_count(const srmg_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
