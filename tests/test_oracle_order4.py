"""The oracle's compact order-4 discretisation (LaplacianDiscretization{2,4},
src/laplacian.jl:131-209) and the BoxStencil connectivity it runs on
(src/connectivity.jl:106-149, src/stencil.jl:34-90), checked without a GPU.

The reference ships no tests for this path, so the restatement is pinned by what the
scheme must do:
  * the BoxStencil edge lists give every block exactly one edge per box direction;
  * a constant lies in the operator's kernel (all geometries, the axis row included);
  * the interior truncation error falls 16x per refinement (fourth order) for the
    Cartesian and the cylindrical stencil;
  * the Cartesian solution converges at fourth order to a manufactured solution;
  * rhs_level! is the identity at order 2 (bit-exact copy).
"""
import numpy as np
import pytest

from oracle import Oracle, lib as olib, _ptr
import ctypes
from srmg import gen
from srmg.tree import Tree, populate, connectivity, BOX2, STAR2, boundaryconditions


def uniform(level, stencil=BOX2):
    t = Tree((1, 1), level)
    populate(t, level)
    return t, connectivity(t, stencil)


def test_box_connectivity_covers_every_direction():
    p = gen.order4_problem(seed=11, geom=gen.GEOM_CYL1)
    tree, conn = p.tree, p.conn
    for l, layer in enumerate(tree, start=1):
        seen = {blk: [] for _, blk in layer.pairs}
        for e in conn.neighbor[l - 1]:
            seen[int(e["to"])].append(tuple(-int(x) for x in e["face"]))
        for e in conn.boundary[l - 1]:
            f = tuple(int(x) for x in e["face"])
            bnd = tuple(int(x) for x in e["bnd"])
            # bnd is the face restricted to the dimensions that leave the domain
            assert all(bnd[d] in (0, f[d]) for d in range(2)) and any(bnd)
            seen[int(e["block"])].append(f)
        for e in conn.refboundary[l - 1]:
            seen[int(e["fine"])].append(tuple(int(x) for x in e["face"]))
        for blk, dirs in seen.items():
            assert sorted(dirs) == sorted(BOX2), (l, blk, dirs)


def test_box_nesting_gives_diagonal_parents():
    # refining with the star stencil alone can leave a diagonal neighbour without a
    # parent; BOX2 nesting (src/streamer.jl:437) never does
    t = Tree((1, 1), 5)
    populate(t, 3)
    from srmg.tree import refine_block
    refine_block(t, 3, (3, 3), BOX2)
    refine_block(t, 4, (6, 6), BOX2)
    t.sync()
    connectivity(t, BOX2)  # raises if a diagonal parent is missing


def _problem(level, geom, op, ex, lap, bc):
    t, conn = uniform(level, BOX2 if op == 2 else STAR2)
    h1 = 1.0 / 16
    p = gen.make_problem(t, lambda r, z, l, gi, gj: -lap(r, z), 1.0, op=op, bc=bc, h1=h1, conn=conn)
    p.geom = geom
    p.s = h1 * h1  # s_l = h_l^2: the operator is then the plain Laplacian
    return p


def _rhs(o, q, nlev):
    o.fill_ghost_all(q)
    b = np.zeros_like(q)
    for l in range(1, nlev + 1):
        o.rhs_level(b, q, l)
    o.fill_ghost_all(b)
    return b


A, B = np.pi / 2, np.pi
CASES = {
    # sin(pi r) sin(pi z), all Dirichlet: the mirror ghosts are exact (odd symmetry)
    gen.GEOM_CART: (lambda r, z: np.sin(B * r) * np.sin(B * z),
                    lambda r, z: -2 * B * B * np.sin(B * r) * np.sin(B * z),
                    boundaryconditions(((-1, -1), (-1, -1)))),
    # cos(pi r / 2) sin(pi z): even about the axis, odd about r = 1
    gen.GEOM_CYL1: (lambda r, z: np.cos(A * r) * np.sin(B * z),
                    lambda r, z: (-A * A * np.cos(A * r) - A * np.sin(A * r) / r - B * B * np.cos(A * r))
                    * np.sin(B * z),
                    boundaryconditions(((1, -1), (-1, -1)))),
    # the same with the radial dimension second (CylindricalGeometry{2}): the block
    # coordinates' first component is then the axial one
    gen.GEOM_CYL2: (lambda a, r: np.cos(A * r) * np.sin(B * a),
                    lambda a, r: (-A * A * np.cos(A * r) - A * np.sin(A * r) / r - B * B * np.cos(A * r))
                    * np.sin(B * a),
                    boundaryconditions(((-1, -1), (1, -1)))),
}


@pytest.mark.parametrize("geom", [gen.GEOM_CART, gen.GEOM_CYL1, gen.GEOM_CYL2])
def test_order4_interior_truncation_is_fourth_order(geom):
    ex, lap, bc = CASES[geom]
    errs = []
    for level in (2, 3, 4):
        p = _problem(level, geom, 2, ex, lap, bc)
        o = Oracle(p)
        u = np.zeros_like(p.b)
        for l in range(1, level + 1):
            blks, r, z, _, _ = gen.block_cell_centres(p.tree, l, p.h1)
            u[blks - 1, 2:18, 2:18] = ex(r, z).reshape(len(blks), 16, 16)
        o.fill_ghost_all(u)
        b = _rhs(o, p.b.copy(), level)
        res = np.zeros_like(u)
        hl = p.h1 / 2 ** (level - 1)
        olib().orc_residual_level(_ptr(res), _ptr(u), _ptr(b), hl * hl, o.ot.ref, level, ctypes.byref(o.op))
        blks, r, z, _, _ = gen.block_cell_centres(p.tree, level, p.h1)
        rv = res[blks - 1, 2:18, 2:18].reshape(-1)
        r, z = r.reshape(-1), z.reshape(-1)
        inner = (r > 0.25) & (r < 0.75) & (z > 0.25) & (z < 0.75)
        errs.append(np.abs(rv[inner]).max())
    ratios = [errs[k] / errs[k + 1] for k in range(2)]
    assert all(x > 14.0 for x in ratios), (errs, ratios)


def test_order4_cartesian_solution_is_fourth_order():
    ex, lap, bc = CASES[gen.GEOM_CART]
    errs = []
    for level in (2, 3):
        p = _problem(level, gen.GEOM_CART, 2, ex, lap, bc)
        o = Oracle(p)
        b = _rhs(o, p.b.copy(), level)
        u = np.zeros_like(b)
        cyc, rel = o.solve(u, b, 1e-12, max_cycles=400)
        assert rel <= 1e-12
        blks, r, z, _, _ = gen.block_cell_centres(p.tree, level, p.h1)
        errs.append(np.abs(u[blks - 1, 2:18, 2:18].reshape(len(blks), -1) - ex(r, z).reshape(len(blks), -1)).max())
    assert errs[0] / errs[1] > 14.0, errs


@pytest.mark.parametrize("geom", [gen.GEOM_CART, gen.GEOM_CYL1, gen.GEOM_CYL2])
def test_order4_constant_in_kernel(geom):
    p = gen.order4_problem(seed=3, geom=geom)
    p.bc = boundaryconditions(((1, 1), (1, 1)))  # Neumann everywhere: ghosts of 1 are 1
    o = Oracle(p)
    u = np.ones_like(p.b)
    b = np.zeros_like(p.b)
    r = np.zeros_like(p.b)
    for l in range(1, len(p.tree) + 1):
        hl = p.h1 / 2 ** (l - 1)
        olib().orc_residual_level(_ptr(r), _ptr(u), _ptr(b), hl * hl, o.ot.ref, l, ctypes.byref(o.op))
    # |L 1| / s_l against the size of one term, |20 u| / (6 s_l)
    for l in range(1, len(p.tree) + 1):
        hl = p.h1 / 2 ** (l - 1)
        blks = np.array([blk for _, blk in p.tree[l - 1].pairs])
        assert np.abs(r[blks - 1, 2:18, 2:18]).max() * hl * hl <= 1e-13


def test_rhs_level_order2_is_identity():
    p = gen.order4_problem(seed=4, geom=gen.GEOM_CYL1)
    p.op = gen.OP_LAPLACIAN
    o = Oracle(p)
    q = np.random.default_rng(0).standard_normal(p.b.shape)
    q[0, 5, 5] = -0.0
    q1 = np.full_like(q, 7.0)
    for l in range(1, len(p.tree) + 1):
        o.rhs_level(q1, q, l)
    used = np.zeros(q.shape[0], dtype=bool)
    for layer in p.tree:
        for _, blk in layer.pairs:
            used[blk - 1] = True
    assert np.array_equal(q1[used][:, 2:18, 2:18].view(np.uint64), q[used][:, 2:18, 2:18].view(np.uint64))


def test_four_colours_cover_every_cell_once():
    """FourColors {0,0}, {0,1}, {1,0}, {1,1} (src/multigrid.jl:206-232): with u = 0 and
    b = 1, each colour changes a disjoint quarter of the valid cells."""
    p = gen.order4_problem(seed=12, geom=gen.GEOM_CART)
    o = Oracle(p)
    blk = p.tree[0].pairs[0][1] - 1
    seen = np.zeros((16, 16), dtype=int)
    for c in range(4):
        u = np.zeros_like(p.b)
        b = np.ones_like(p.b)
        olib().orc_gs4_level(_ptr(u), _ptr(b), 1.0, 1.0, o.ot.ref, 1, ctypes.byref(o.op), c >> 1, c & 1)
        seen += (u[blk, 2:18, 2:18] != 0)
    assert np.all(seen == 1)
