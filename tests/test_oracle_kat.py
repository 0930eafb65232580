"""Known-answer tests of the oracle, derived from the reference's formulas (the reference
ships no golden vectors or tests of its own).

  * cylindrical stencil (src/laplacian.jl:100-108): with r_i = i - 1/2 in cell units and
    w- = (2i-2)/(2i-1), w+ = 2i/(2i-1), L(r^2) = 4 at every cell (axis weight 0),
    L(z^2) = 2, L(const) = 0, L of a z-linear function = 0; Cartesian L(r^2) = 2;
  * prolongation (src/interp.jl:54-58) reproduces functions linear in (r, z);
  * restriction (src/restrict.jl:5-25) of a constant is the constant, exactly;
  * solver: the V-cycle (src/multigrid.jl:60-106) converges to a manufactured
    discrete solution u* (b := -L u* / s_l on every leaf cell, ghosts of u* filled by
    the reference's own rules), on a uniform and on a refined tree.
"""
import numpy as np
import pytest

from oracle import Oracle, OracleTree, lib as olib, make_op, _ptr
from srmg import gen

GEOM_CART, GEOM_CYL1 = 0, 1


def tree_problem(tree):
    return gen.make_problem(tree, lambda r, z, l, gi, gj: np.zeros_like(r), 1.0)


def cell_index_fields(tree, l, nblk):
    """1-based global cell indices (i along r, j along z) of every cell (ghosts too) of
    the level-l blocks, as (nblk, 20, 20) arrays; NaN outside level l."""
    I = np.full((nblk, 20, 20), np.nan)
    J = np.full((nblk, 20, 20), np.nan)
    x = np.arange(20)
    for (cr, cz), blk in tree[l - 1].index.items():
        I[blk - 1] = (x - 1 + 16 * (cr - 1))[None, :]
        J[blk - 1] = (x - 1 + 16 * (cz - 1))[:, None]
    return I, J


@pytest.fixture(scope="module")
def uniform3():
    return tree_problem(gen._uniform(3))


@pytest.mark.parametrize("geom,fn,expect", [
    (GEOM_CYL1, lambda i, j: (i - 0.5) ** 2, -4.0),
    (GEOM_CYL1, lambda i, j: (j - 0.5) ** 2, -2.0),
    (GEOM_CYL1, lambda i, j: 3.25 + 0 * i, 0.0),
    (GEOM_CYL1, lambda i, j: 0.75 * (j - 0.5) - 2.0 + 0 * i, 0.0),
    (GEOM_CART, lambda i, j: (i - 0.5) ** 2, -2.0),
])
def test_stencil_exactness(uniform3, geom, fn, expect):
    p = uniform3
    op = make_op(gen.OP_LAPLACIAN, 0.0, geom, p.bc)
    ot = OracleTree(p.tree, p.conn, p.nblk)
    for l in range(1, len(p.tree) + 1):
        I, J = cell_index_fields(p.tree, l, p.nblk)
        lev = ~np.isnan(I)
        u = np.where(lev, fn(np.nan_to_num(I), np.nan_to_num(J)), 0.0)
        b = np.zeros_like(u)
        r = np.zeros_like(u)
        olib().orc_residual_level(_ptr(r), _ptr(u), _ptr(b), 1.0, ot.ref, l, op)
        blks = [blk - 1 for blk in p.tree[l - 1].index.values()]
        got = r[blks][:, 2:18, 2:18]
        # the sums cancel values up to max|u|: allow a few ulps of that magnitude
        np.testing.assert_allclose(got, expect, rtol=0, atol=32 * np.finfo(float).eps * max(1.0, np.abs(u).max()))


def test_prolongation_reproduces_linear(uniform3):
    p = uniform3
    ot = OracleTree(p.tree, p.conn, p.nblk)
    a, b_, c = 0.37, -1.25, 4.5
    for l in range(2, len(p.tree) + 1):
        Ic, Jc = cell_index_fields(p.tree, l - 1, p.nblk)
        e = np.where(~np.isnan(Ic), a * (np.nan_to_num(Ic) - 0.5) + b_ * (np.nan_to_num(Jc) - 0.5) + c, 0.0)
        u = np.zeros_like(e)
        olib().orc_interp_add_level(_ptr(u), _ptr(e), ot.ref, l)
        If, Jf = cell_index_fields(p.tree, l, p.nblk)
        blks = [blk - 1 for blk in p.tree[l - 1].index.values()]
        expect = a * (If[blks] - 0.5) / 2 + b_ * (Jf[blks] - 0.5) / 2 + c
        np.testing.assert_allclose(u[blks][:, 2:18, 2:18], expect[:, 2:18, 2:18], rtol=1e-14, atol=1e-13)


def test_restriction_of_constant_is_exact(uniform3):
    p = uniform3
    ot = OracleTree(p.tree, p.conn, p.nblk)
    for cval in (1.0, -3.0625, 1e-300, 7.123456789):
        u = np.zeros((p.nblk, 20, 20))
        L = len(p.tree)
        for blk in p.tree[L - 1].index.values():
            u[blk - 1, 2:18, 2:18] = cval
        olib().orc_restrict_level(_ptr(u), ot.ref, L)
        for blk in p.tree[L - 2].index.values():
            assert np.all(u[blk - 1, 2:18, 2:18] == cval)


def manufactured(p, seed):
    """A discrete solution u*: smooth random leaf values, made a composite-grid function
    (restricted onto covered cells, ghosts filled level by level with the reference's
    rules), and b := -L u* / s_l on every cell."""
    orc = Oracle(p)
    rng = np.random.default_rng(seed)
    u = np.zeros((p.nblk, 20, 20))
    for l in range(1, len(p.tree) + 1):
        I, J = cell_index_fields(p.tree, l, p.nblk)
        lev = ~np.isnan(I)
        k1, k2 = rng.uniform(0.5, 2.0), rng.uniform(0.5, 2.0)
        n = 16 * 2 ** (l - 1)
        f = np.cos(np.pi * k1 * (np.nan_to_num(I) - 0.5) / n) * np.sin(np.pi * (np.nan_to_num(J) - 0.5) / n)
        f = f * np.sin(np.pi * k2 * (np.nan_to_num(J) - 0.5) / n)
        u = np.where(lev, f, u)
    olib().orc_restrict_full(_ptr(u), orc.ot.ref)
    orc.fill_ghost_all(u)
    b = np.zeros_like(u)
    r = np.zeros_like(u)
    for l in range(1, len(p.tree) + 1):
        sl = p.s / 4 ** (l - 1)
        olib().orc_residual_level(_ptr(r), _ptr(u), _ptr(b), sl, orc.ot.ref, l, orc.op)
    return orc, u, r.copy()  # r = -(0 + L u*/s_l) is the right-hand side


@pytest.mark.parametrize("which", ["uniform4", "refined"])
def test_vcycles_converge_to_manufactured_solution(which):
    if which == "uniform4":
        p = tree_problem(gen._uniform(4))
    else:
        p = gen.config2(seed=5, target_leaf=40_000, extra=3)
    orc, ustar, b = manufactured(p, 3)
    r0 = np.zeros_like(ustar)
    # u* is a fixed point: its residual vanishes to rounding
    assert orc.resnorm(r0, b, ustar) <= 1e-12 * orc.leafnorm(b)
    u = np.zeros_like(ustar)
    c, rel = orc.solve(u, b.copy(), 1e-13, max_cycles=2000)
    assert rel <= 1e-13
    leaf = np.zeros(u.shape, dtype=bool)
    for layer in p.tree:
        for cc, blk in layer.index.items():
            if p.tree.isleaf(layer.level, cc):
                leaf[blk - 1, 2:18, 2:18] = True
    err = np.linalg.norm((u - ustar)[leaf]) / np.linalg.norm(ustar[leaf])
    assert err < 1e-8, err


def test_netcharge_and_field_of_linear_potential(uniform3):
    """netcharge! (src/streamer.jl:369-373) is nion - ne exactly; electric_field!
    (src/multigrid.jl:421-449) of u = A r + B z (r, z cell centres of each level) is the
    constant field (-A + e0_r, -B + e0_z) on every face and its magnitude on every cell."""
    p = uniform3
    ot = OracleTree(p.tree, p.conn, p.nblk)
    rng = np.random.default_rng(4)
    ne = rng.uniform(0, 1e20, (p.nblk, 20, 20))
    ni = rng.uniform(0, 1e20, (p.nblk, 20, 20))
    q = np.zeros_like(ne)
    olib().orc_netcharge(_ptr(q), _ptr(ne), _ptr(ni), ot.ref)
    vm = np.zeros(q.shape, dtype=bool)
    vm[:, 2:18, 2:18] = True
    assert np.array_equal(q[vm], (ni - ne)[vm])
    assert np.all(q[~vm] == 0)

    h, A, B, e0 = 7.8125e-4, 3.0e5, -1.25e6, np.array([250.0, 1.5e6])
    u = np.zeros((p.nblk, 20, 20))
    for l in range(1, len(p.tree) + 1):
        I, J = cell_index_fields(p.tree, l, p.nblk)
        hl = h / 2 ** (l - 1)
        lev = ~np.isnan(I)
        u = np.where(lev, A * (np.nan_to_num(I) - 0.5) * hl + B * (np.nan_to_num(J) - 0.5) * hl, u)
    e = np.zeros((p.nblk, 2, 21, 21))
    eabs = np.zeros((p.nblk, 20, 20))
    olib().orc_electric_field(_ptr(e), _ptr(eabs), _ptr(u), h, _ptr(e0), ot.ref)
    er = e[:, 0, 2:18, 2:19]   # faces 3..19 along r, cells 3..18 along z (1-based)
    ez = e[:, 1, 2:19, 2:18]
    np.testing.assert_allclose(er, -A + e0[0], rtol=1e-9)
    np.testing.assert_allclose(ez, -B + e0[1], rtol=1e-9)
    np.testing.assert_allclose(eabs[vm], np.hypot(-A + e0[0], -B + e0[1]), rtol=1e-9)


def test_generator_restriction_matches_oracle():
    """The problem generators restrict right-hand sides onto parent blocks the way
    restrict_full! does (src/restrict.jl:43-47); checked bit for bit against the
    oracle's restriction chain on a refined tree."""
    import numpy as np
    from oracle import Oracle, lib as olib, _ptr
    from srmg import gen
    p = gen.order4_problem(seed=13, geom=gen.GEOM_CYL1)
    o = Oracle(p)
    f = np.random.default_rng(5).standard_normal(p.b.shape)
    a = f.copy()
    gen.restrict_full_np(a, p.tree, p.conn)
    b = f.copy()
    for l in range(len(p.tree), 1, -1):
        olib().orc_restrict_level(_ptr(b), o.ot.ref, l)
    np.testing.assert_array_equal(a.view(np.uint64), b.view(np.uint64))
