"""Parity of the free boundary conditions on the GPU (srmg_freebc, srmg_fill_ghost_free,
through the C ABI) with the oracle (oracle/freebc_oracle.py restating src/freebc.jl).

Bar: the boundary sources added to q, conf.b and the ghost values agree with the
oracle to <= 1e-12 relative L2: the GPU runs both sine transforms through its own FFT
(power-of-two lengths) or as direct FP64 sums (other lengths), the oracle through
scipy's FFTs, so the two round differently.  Every other cell is
untouched (bit-exact).  End to end (homogeneous solve, free boundary, main solve) the
potential matches the oracle's to <= 1e-10.
"""
import numpy as np
import pytest

import freebc_oracle as fo
from conftest import gpu_available
from oracle import Oracle
from srmg import gen, multigrid as mg
from srmg.tree import STAR2, BOX2

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]

REL = 1e-12
SRMG_ERR_BADARG = -1


def torch_cuda(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    torch.cuda.synchronize()
    return t


def rel_l2(a, b):
    n = np.linalg.norm(np.ravel(b))
    return np.linalg.norm(np.ravel(a - b)) / (n if n > 0 else 1.0)


CASES = [(d, st) for d in (1, 2) for st in ("star", "box")]


def setup(dim, stencil):
    p = gen.outer_refined_problem(dim, STAR2 if stencil == "star" else BOX2)
    level = len(p.tree)
    n, H, R, f = fo.kernel(dim, level, (1, 1), p.h1)
    ctx = mg.Context(0).set_tree(p.tree, p.conn)
    mg.freebc_set(ctx, dim, level, (1, 1), f)
    return p, ctx, level, f


@pytest.mark.parametrize("dim,stencil", CASES)
def test_freebc_sources_and_b(dim, stencil):
    p, ctx, level, f = setup(dim, stencil)
    rng = np.random.default_rng(3)
    u = rng.standard_normal(p.b.shape)
    q = rng.standard_normal(p.b.shape)
    qo = q.copy()
    bo = fo.freebc(qo, u, p.h1, p.s, p.tree, p.conn, dim, level, f)
    import torch
    qg, ug = torch_cuda(q), torch_cuda(u)
    bg = torch.zeros(len(f), dtype=torch.float64, device="cuda")
    l0 = ctx.launches()
    mg.freebc_(ctx, qg, ug, p.h1, p.s, b_out=bg)
    ctx.synchronize()
    # n <= 8192, a power of two: the transform pair in one CTA, then the sources of all
    # levels in one launch
    assert ctx.launches() - l0 == 2
    qn = qg.cpu().numpy()
    assert rel_l2(bg.cpu().numpy(), bo) <= REL
    changed = qo != q
    assert changed.any()
    np.testing.assert_array_equal(qn[~changed], q[~changed])
    assert rel_l2(qn[changed] - q[changed], qo[changed] - q[changed]) <= REL
    # the host-array entry point gives the same result
    qh = q.copy()
    bh = np.zeros(len(f))
    mg.freebc_(ctx, qh, u, p.h1, p.s, b_out=bh)
    np.testing.assert_array_equal(qh, qn)
    np.testing.assert_array_equal(bh, bg.cpu().numpy())
    ctx.close()


@pytest.mark.parametrize("dim,stencil", CASES)
def test_fill_ghost_free(dim, stencil):
    p, ctx, level, f = setup(dim, stencil)
    rng = np.random.default_rng(4)
    u = rng.standard_normal(p.b.shape)
    q = rng.standard_normal(p.b.shape)
    bo = fo.freebc(q.copy(), u, p.h1, p.s, p.tree, p.conn, dim, level, f)
    mg.freebc_(ctx, q.copy(), u, p.h1, p.s)
    w = rng.standard_normal(p.b.shape)
    for l in range(1, len(p.tree) + 1):
        wo = w.copy()
        fo.fill_ghost_free(wo, bo, p.tree, dim, level, l)
        wg = torch_cuda(w)
        mg.fill_ghost_free_(ctx, wg, l)
        ctx.synchronize()
        wn = wg.cpu().numpy()
        changed = wo != w
        np.testing.assert_array_equal(wn[~changed], w[~changed])
        if changed.any():
            assert rel_l2(wn[changed] - w[changed], wo[changed] - w[changed]) <= REL, l
    ctx.close()


@pytest.mark.parametrize("dim", [1, 2])
def test_free_boundary_end_to_end(dim):
    """derivs!'s sequence (src/streamer.jl:320-334): homogeneous solve, freebc!, main
    solve, on the GPU against the oracle."""
    p, ctx, level, f = setup(dim, "star")
    o = Oracle(p)
    q = p.b.copy()
    o.fill_ghost_all(q)
    uh = np.zeros_like(q)
    st = mg.solve(ctx, uh, q.copy(), p.s, p.geom, p.bc, tol=1e-12, mode=mg.MODE_FP64, max_cycles=3000)
    assert st["rel_residual"] <= 1e-12
    q1 = q.copy()
    mg.freebc_(ctx, q1, uh, p.h1, p.s)
    u = np.zeros_like(q)
    st = mg.solve(ctx, u, q1, p.s, p.geom, p.bc, tol=1e-12, mode=mg.MODE_FP64, max_cycles=3000)
    assert st["rel_residual"] <= 1e-12
    uho = np.zeros_like(q)
    o.solve(uho, q.copy(), 1e-12, 3000)
    q1o = q.copy()
    fo.freebc(q1o, uho, p.h1, p.s, p.tree, p.conn, dim, level, f)
    uo = np.zeros_like(q)
    o.solve(uo, q1o, 1e-12, 3000)
    used = np.zeros(p.nblk, dtype=bool)
    for layer in p.tree:
        for _, blk in layer.pairs:
            used[blk - 1] = True
    assert rel_l2(u[used][:, 2:18, 2:18], uo[used][:, 2:18, 2:18]) <= 1e-10
    ctx.close()


def test_freebc_refuses_bad_use():
    p = gen.outer_refined_problem(1, STAR2)
    ctx = mg.Context(0).set_tree(p.tree, p.conn)
    q = np.zeros_like(p.b)
    with pytest.raises(mg.SrmgError) as ei:           # no srmg_freebc_set yet
        mg.freebc_(ctx, q, q.copy(), p.h1, p.s)
    assert ei.value.code == SRMG_ERR_BADARG
    n, H, R, f = fo.kernel(1, 5, (1, 1), p.h1)          # level 5 < the tree's finest (6)
    mg.freebc_set(ctx, 1, 5, (1, 1), f)
    with pytest.raises(mg.SrmgError) as ei:
        mg.freebc_(ctx, q, q.copy(), p.h1, p.s)
    assert ei.value.code == SRMG_ERR_BADARG
    with pytest.raises(mg.SrmgError):                   # n does not match FreeBC's length
        mg.freebc_set(ctx, 1, 7, (1, 1), f)
    ctx.close()


@pytest.mark.parametrize("rows", [2, 3])
def test_freebc_oblong_root(rows):
    """A (1, 2) root grid: the outer column is twice as long (n = 2 * 16 * 2^(level-1)),
    a power of two (the FFT path); a (1, 3) root: n = 3 * 16 * 2^(level-1), the direct
    sums."""
    from srmg.tree import Tree, populate, connectivity, boundaryconditions, refine_block
    t = Tree((1, rows), 4)
    populate(t, 2)
    refine_block(t, 2, (2, 3))
    t.sync()
    conn = connectivity(t)
    p = gen.make_problem(t, lambda r, z, l, gi, gj: np.exp(-(r * r + (z - 0.012) ** 2) / 2e-5), gen.poisson_scale(),
                         bc=boundaryconditions(((1, -1), (-1, -1))), conn=conn)
    level = len(t)
    n, H, R, f = fo.kernel(1, level, (1, rows), p.h1)
    assert n == rows * 16 * 2 ** (level - 1)
    ctx = mg.Context(0).set_tree(p.tree, p.conn)
    mg.freebc_set(ctx, 1, level, (1, rows), f)
    rng = np.random.default_rng(8)
    u = rng.standard_normal(p.b.shape)
    q = rng.standard_normal(p.b.shape)
    qo = q.copy()
    bo = fo.freebc(qo, u, p.h1, p.s, p.tree, p.conn, 1, level, f)
    qh = q.copy()
    bh = np.zeros(n)
    mg.freebc_(ctx, qh, u, p.h1, p.s, b_out=bh)
    assert rel_l2(bh, bo) <= REL
    changed = qo != q
    np.testing.assert_array_equal(qh[~changed], q[~changed])
    assert rel_l2(qh[changed] - q[changed], qo[changed] - q[changed]) <= REL
    ctx.close()


@pytest.mark.parametrize("level", [9, 11, 13])
def test_freebc_fft_matches_direct_sums(level):
    """At the lengths of a 9-, 11- and 13-level tree (n = 4096, 16384, 65536: the last
    two through the four-step FFT) the FFT transforms give conf.b and the sources of
    the direct sums and of the oracle to <= 1e-12."""
    import torch
    p = gen.config2(seed=5, target_leaf=40_000, extra=3)
    n, H, R, f = fo.kernel(1, level, (1, 1), p.h1)
    ctx = mg.Context(0).set_tree(p.tree, p.conn)
    mg.freebc_set(ctx, 1, level, (1, 1), f)
    rng = np.random.default_rng(level)
    u = rng.standard_normal(p.b.shape)
    q = rng.standard_normal(p.b.shape)
    out = {}
    for direct in (0, 1):
        ctx.set_option("freebc_direct", direct)
        qg, ug = torch_cuda(q), torch_cuda(u)
        bg = torch.zeros(n, dtype=torch.float64, device="cuda")
        mg.freebc_(ctx, qg, ug, p.h1, p.s, b_out=bg)
        ctx.synchronize()
        out[direct] = (qg.cpu().numpy(), bg.cpu().numpy())
    qo = q.copy()
    bo = fo.freebc(qo, u, p.h1, p.s, p.tree, p.conn, 1, level, f)
    changed = qo != q
    # the FFT path rounds like the oracle's FFTs; the direct sums of n terms round to
    # within ~n ulp
    bar = {0: REL, 1: max(REL, 4 * n * np.finfo(float).eps)}
    for direct in (0, 1):
        assert rel_l2(out[direct][1], bo) <= bar[direct], direct
        assert rel_l2(out[direct][0][changed] - q[changed], qo[changed] - q[changed]) <= bar[direct], direct
    assert rel_l2(out[0][1], out[1][1]) <= bar[1]
    ctx.close()
