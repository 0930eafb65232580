"""The D = 3 oracle (oracle/srmg_oracle3.c), checked without a GPU.  Known answers
from the reference's 3D formulas (src/laplacian.jl:274-340, src/interp.jl:7-11,
src/restrict.jl:5-25):
  * every block of a StarStencil{3} / BoxStencil{3} tree has one edge per direction;
  * ghost fills: a mirrored boundary ghost holds sign * the valid cell it mirrors;
    interpolation with weights 1/4 reproduces linear functions; restriction of a
    constant is the constant;
  * the order-2 and order-4 solutions converge to sin(pi x) sin(pi y) sin(pi z) at
    second and fourth order;
  * V-cycles on a refined octree drive the residual norm below 1e-10.
"""
import ctypes

import numpy as np
import pytest

from oracle import Oracle3, lib as olib, _ptr
from srmg import gen3
from srmg.tree3 import Tree3, populate, connectivity, STAR3, BOX3, block_cell_centres


def test_every_block_has_one_edge_per_direction():
    for st in (STAR3, BOX3):
        p = gen3.refined3(seed=3, stencil=st)
        for l, layer in enumerate(p.tree, start=1):
            seen = {blk: [] for _, blk in layer.pairs}
            for e in p.conn.neighbor[l - 1]:
                seen[int(e["to"])].append(tuple(-int(x) for x in e["face"]))
            for e in p.conn.boundary[l - 1]:
                seen[int(e["block"])].append(tuple(int(x) for x in e["face"]))
            for e in p.conn.refboundary[l - 1]:
                seen[int(e["fine"])].append(tuple(int(x) for x in e["face"]))
            for blk, dirs in seen.items():
                assert sorted(dirs) == sorted(st), (l, blk)


def test_interp_linear_and_restrict_constant():
    p = gen3.refined3(seed=4)
    o = Oracle3(p)
    # u = linear function of the cell centre on every level, ghosts from the function too
    u = np.zeros_like(p.b)
    for l in range(1, len(p.tree) + 1):
        blks, x, y, z = block_cell_centres(p.tree, l, 1.0)
        if len(blks) == 0:
            continue
        blk = 1.0 / 2 ** (l - 1)            # block edge at level l, in level-1 block units
        ii = (np.arange(20) - 1.5) * blk / 16  # cell centres, ghosts included
        coords = np.array([p.tree[l - 1].coord[b] for b in blks])
        X = (coords[:, 0, None] - 1) * blk + ii[None, :]
        Y = (coords[:, 1, None] - 1) * blk + ii[None, :]
        Z = (coords[:, 2, None] - 1) * blk + ii[None, :]
        u[blks - 1] = (0.5 + 2 * X[:, None, None, :] - 3 * Y[:, None, :, None] + 0.25 * Z[:, :, None, None])
    for l in range(2, len(p.tree) + 1):
        w = u.copy()
        fine = np.array([b for _, b in p.tree[l - 1].pairs]) - 1
        for sl in (np.s_[:2], np.s_[18:]):  # this level's ghosts poisoned; coarse ones stay
            w[fine, sl], w[fine, :, sl], w[fine, :, :, sl] = 7, 7, 7
        olib().orc3_fill_ghost_interp(_ptr(w), o.ot.ref, l)
        for e in p.conn.refboundary[l - 1]:
            f = int(e["fine"]) - 1
            face = [int(x) for x in e["face"]]
            sl = tuple(slice(0, 2) if face[d] < 0 else slice(18, 20) if face[d] > 0 else slice(2, 18)
                       for d in (2, 1, 0))
            np.testing.assert_allclose(w[f][sl], u[f][sl], rtol=0, atol=1e-12)
    c = np.full_like(p.b, 3.25)
    for l in range(len(p.tree), 1, -1):
        olib().orc3_restrict_level(_ptr(c), o.ot.ref, l)
    assert np.all(c == 3.25)


def _sine_problem(level, op):
    t = Tree3((1, 1, 1), level)
    populate(t, level)
    conn = connectivity(t, BOX3 if op == 2 else STAR3)
    pi = np.pi
    ex = lambda x, y, z: np.sin(pi * x) * np.sin(pi * y) * np.sin(pi * z)
    p = gen3.make_problem3(t, conn, lambda x, y, z: 3 * pi * pi * ex(x, y, z), 1.0, op=op, h1=1.0 / 16)
    p.s = p.h1 ** 2
    return p, ex


@pytest.mark.parametrize("op,ratio", [(0, 3.5), (2, 14.0)])
def test_manufactured_solution_order(op, ratio):
    errs = []
    for level in (1, 2):
        p, ex = _sine_problem(level, op)
        o = Oracle3(p)
        q = p.b.copy()
        o.fill_ghost_all(q)
        b = np.zeros_like(q)
        for l in range(1, level + 1):
            o.rhs_level(b, q, l)
        o.fill_ghost_all(b)
        u = np.zeros_like(b)
        _, rel = o.solve(u, b, 1e-11, max_cycles=400)
        assert rel <= 1e-11
        blks, x, y, z = block_cell_centres(p.tree, level, p.h1)
        errs.append(np.abs(u[blks - 1, 2:18, 2:18, 2:18] - ex(x, y, z)).max())
    assert errs[0] / errs[1] > ratio, errs


@pytest.mark.parametrize("op", [0, 1, 2])
def test_vcycles_converge_on_refined_octree(op):
    p = gen3.refined3(seed=5, op=op, k2=40.0 if op == 1 else 0.0)
    o = Oracle3(p)
    q = p.b.copy()
    o.fill_ghost_all(q)
    b = np.zeros_like(q)
    for l in range(1, len(p.tree) + 1):
        o.rhs_level(b, q, l)
    o.fill_ghost_all(b)
    u = np.zeros_like(b)
    c, rel = o.solve(u, b, 1e-10, max_cycles=300)
    assert rel <= 1e-10, (c, rel)


@pytest.mark.parametrize("op", [0, 2])
def test_colours_cover_every_cell_once(op):
    """RedBlack (2 colours) and FourColors (4) for D = 3: with u = 0, b = 1 each colour
    changes a disjoint set of valid cells and together they change all of them."""
    p = gen3.refined3(seed=6, op=op)
    o = Oracle3(p)
    ncol = 4 if op == 2 else 2
    blk = p.tree[0].pairs[0][1] - 1
    seen = np.zeros((16, 16, 16), dtype=int)
    for c in range(ncol):
        u = np.zeros_like(p.b)
        b = np.ones_like(p.b)
        if op == 2:
            olib().orc3_gs4_level(_ptr(u), _ptr(b), 1.0, 1.0, o.ot.ref, 1, ctypes.byref(o.op), c >> 1, c & 1)
        else:
            olib().orc3_gs_level(_ptr(u), _ptr(b), 1.0, 1.0, o.ot.ref, 1, ctypes.byref(o.op), c)
        seen += (u[blk, 2:18, 2:18, 2:18] != 0)
    assert np.all(seen == 1)


def test_boundary_table_is_column_major():
    """boundaryconditions (src/boundary.jl:28-38) for D = 3: entry a[2+b1, 2+b2, 2+b3]
    is the product of the per-dimension signs of the nonzero b_d, at flat index
    (1+b1) + 3(1+b2) + 9(1+b3)."""
    from srmg.tree3 import boundaryconditions
    desc = ((1, -1), (-1, -1), (1, -1))
    a = boundaryconditions(desc)
    for b1 in (-1, 0, 1):
        for b2 in (-1, 0, 1):
            for b3 in (-1, 0, 1):
                want = 1
                for d, b in enumerate((b1, b2, b3)):
                    if b:
                        want *= desc[d][0] if b < 0 else desc[d][1]
                assert a[(1 + b1) + 3 * (1 + b2) + 9 * (1 + b3)] == want


def test_generator_restriction_matches_oracle():
    """The problem generator's numpy restrict_full! sums the 8 fine cells in the
    reference's order, so it matches the oracle's restriction chain bit for bit."""
    p = gen3.refined3(seed=8)
    o = Oracle3(p)
    f = np.random.default_rng(3).standard_normal(p.b.shape)
    a = f.copy()
    gen3.restrict_full3(a, p.tree, p.conn)
    b = f.copy()
    for l in range(len(p.tree), 1, -1):
        olib().orc3_restrict_level(_ptr(b), o.ot.ref, l)
    np.testing.assert_array_equal(a.view(np.uint64), b.view(np.uint64))
