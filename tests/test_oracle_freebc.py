"""The free-boundary oracle (oracle/freebc_oracle.py, restating src/freebc.jl), checked
without a GPU.  The reference has no tests for this path; the restatement is pinned by:
  * the transform pair: DST-III(DST-II(x)) = 2n x (FFTW's RODFT01 inverts RODFT10 up
    to 2n), so the middle of freebc! with f = 1 / (2n) returns its input;
  * physics: with the free boundary at r = R the potential inside R matches the one of
    a 4x wider domain with a grounded outer wall far better than the plain Dirichlet
    solution at r = R does (Malagon-Romero 2018);
  * on trees refined along the outer boundary (both radial dimensions, StarStencil and
    BoxStencil connectivity) only the outermost valid cells of outer blocks change.
"""
import numpy as np
import pytest

import freebc_oracle as fo
from oracle import Oracle
from srmg import gen
from srmg.tree import Tree, populate, connectivity, boundaryconditions, BOX2, STAR2


def test_transform_pair_inverts():
    rng = np.random.default_rng(1)
    for n in (16, 64, 512):
        x = rng.standard_normal(n)
        f = np.full(n, 1.0 / (2 * n))
        # h / 2^(level-1) / 2 = 1 for h = 2, level = 1
        np.testing.assert_allclose(fo.transform(x.copy(), f, 2.0, 1), x, rtol=0, atol=1e-13 * np.abs(x).max())


def _axis_charge(root, level):
    t = Tree(root, level)
    populate(t, level)
    conn = connectivity(t)
    h1 = 1.0 / 16
    rhs = lambda r, z, l, gi, gj: np.exp(-(r ** 2 + (z - 0.5) ** 2) / 0.08 ** 2)
    p = gen.make_problem(t, rhs, h1 * h1, bc=boundaryconditions(((1, -1), (-1, -1))), h1=h1, conn=conn)
    p.geom = gen.GEOM_CYL1
    return p


def _finest(p, u, level):
    blks, r, z, _, _ = gen.block_cell_centres(p.tree, level, p.h1)
    vals = u[blks - 1][:, 2:18, 2:18].reshape(-1)
    return dict(zip(zip(np.round(r.reshape(-1), 9), np.round(z.reshape(-1), 9)), vals))


def test_free_boundary_matches_wide_domain():
    level = 3
    p = _axis_charge((1, 1), level)
    o = Oracle(p)
    q = p.b.copy()
    o.fill_ghost_all(q)
    uh = np.zeros_like(q)
    _, rel = o.solve(uh, q.copy(), 1e-12, 2000)
    assert rel <= 1e-12
    n, H, R, f = fo.kernel(1, level, (1, 1), p.h1)
    q1 = q.copy()
    fo.freebc(q1, uh, p.h1, p.s, p.tree, p.conn, 1, level, f)
    u = np.zeros_like(q)
    _, rel = o.solve(u, q1, 1e-12, 2000)
    assert rel <= 1e-12
    wide = _axis_charge((4, 1), level)
    ow = Oracle(wide)
    qw = wide.b.copy()
    ow.fill_ghost_all(qw)
    uw = np.zeros_like(qw)
    ow.solve(uw, qw, 1e-12, 4000)
    ref = _finest(wide, uw, level)
    keys = list(_finest(p, u, level).keys())
    a = np.array([ref[k] for k in keys])
    free = np.array(list(_finest(p, u, level).values()))
    dirichlet = np.array(list(_finest(p, uh, level).values()))
    err_free = np.linalg.norm(free - a) / np.linalg.norm(a)
    err_dir = np.linalg.norm(dirichlet - a) / np.linalg.norm(a)
    assert err_dir > 1e-2 and err_free < 1e-4, (err_free, err_dir)


@pytest.mark.parametrize("dim", [1, 2])
@pytest.mark.parametrize("stencil", ["star", "box"])
def test_sources_only_on_outer_cells(dim, stencil):
    p = gen.outer_refined_problem(dim, STAR2 if stencil == "star" else BOX2)
    level = len(p.tree)
    n, H, R, f = fo.kernel(dim, level, (1, 1), p.h1)
    rng = np.random.default_rng(2)
    u = rng.standard_normal(p.b.shape)
    q = rng.standard_normal(p.b.shape)
    q0 = q.copy()
    b = fo.freebc(q, u, p.h1, p.s, p.tree, p.conn, dim, level, f)
    assert b.shape == (n,) and np.isfinite(b).all() and np.abs(b).max() > 0
    changed = np.argwhere(q != q0)
    assert len(changed) > 0
    for blk, j, i in changed:
        along = i if dim == 1 else j
        assert along == 17, (blk, j, i)
        lv = next(l for l, layer in enumerate(p.tree, start=1) if blk + 1 in layer.coord)
        c = p.tree[lv - 1].coord[blk + 1]
        assert c[dim - 1] == p.tree[lv - 1].domain[dim - 1]
