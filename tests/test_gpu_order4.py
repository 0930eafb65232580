"""Parity of the compact order-4 discretisation and of BoxStencil trees with the
oracle, through the C ABI on the GPU.

Bars: ghost fills (star faces and the 2 x 2 corners, each pass and fill_ghost!),
the four-colour Gauss-Seidel sweep and iteration, the residual, the FAS coarse
right-hand side and rhs_level! are bit-exact (both sides round every operation on its
own, in the reference's order); V-cycles, FMG and the residual norm agree to <= 1e-12
relative L2.  Order-2 operators on a BoxStencil tree run the per-operation kernels,
which fill the corners too, and match the oracle on every cell, ghosts included.
"""
import ctypes

import numpy as np
import pytest

from conftest import gpu_available
from oracle import Oracle, lib as olib, _ptr
from srmg import gen, multigrid as mg
from srmg.tree import connectivity, BOX2

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]

REL = 1e-12
SRMG_ERR_UNSUPPORTED = -6


def torch_cuda(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    torch.cuda.synchronize()
    return t


def to_np(t):
    return t.cpu().numpy()


def bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


def rel_l2(a, b):
    n = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (n if n > 0 else 1.0)


def permuted(p, seed):
    """Renumber blocks with gaps and shuffle every list (results must not depend on
    numbering or on the Dict order of BlockLayer.pairs, src/blocklayer.jl:48-53)."""
    rng = np.random.default_rng(seed)
    n = p.nblk
    nalloc = n + 5
    perm = rng.permutation(nalloc)[:n] + 1
    for layer in p.tree:
        idx = {c: int(perm[b - 1]) for c, b in layer.index.items()}
        layer.index = idx
        layer.coord = {b: c for c, b in idx.items()}
        layer.sync(rng)
    conn = connectivity(p.tree, BOX2)
    for lists in (conn.neighbor, conn.boundary, conn.refboundary, conn.child):
        for k, arr in enumerate(lists):
            lists[k] = arr[rng.permutation(len(arr))]
    b = np.zeros((nalloc, 20, 20))
    b[perm - 1] = p.b
    return gen.Problem(tree=p.tree, conn=conn, b=b, s=p.s, op=p.op, k2=p.k2, geom=p.geom, bc=p.bc,
                       h1=p.h1, name=p.name + "-perm")


PROBS = {
    "cart": gen.order4_problem(seed=21, geom=gen.GEOM_CART),
    "cyl1": gen.order4_problem(seed=22, geom=gen.GEOM_CYL1),
    "cyl2": gen.order4_problem(seed=23, geom=gen.GEOM_CYL2),
    "cyl1_perm": permuted(gen.order4_problem(seed=24, geom=gen.GEOM_CYL1), 5),
}


class Pair:
    def __init__(self, p):
        self.p = p
        self.ctx = mg.Context(0).set_tree(p.tree, p.conn)
        self.orc = Oracle(p)
        self.bcp = np.ascontiguousarray(p.bc, dtype=np.int8)
        self.nlev = len(p.tree)

    def rhs(self):
        """b = rhs_level!(q) on every level, q's and b's ghosts filled (src/streamer.jl:313-318)."""
        q = self.p.b.copy()
        self.orc.fill_ghost_all(q)
        b = np.zeros_like(q)
        for l in range(1, self.nlev + 1):
            self.orc.rhs_level(b, q, l)
        self.orc.fill_ghost_all(b)
        return b


@pytest.fixture(scope="module", params=list(PROBS))
def pair(request):
    return Pair(PROBS[request.param])


def rand(p, seed):
    return np.random.default_rng(seed).standard_normal((p.nblk, 20, 20))


@pytest.mark.parametrize("mask", [1, 2, 3, 4, 5, 6, 7])
def test_fill_ghost_box_bitexact(pair, mask):
    p = pair.p
    u0 = rand(p, 1)
    for l in range(1, pair.nlev + 1):
        ug = torch_cuda(u0)
        mg.fill_ghost_(pair.ctx, ug, l, p.bc, mask=mask)
        pair.ctx.synchronize()
        uo = u0.copy()
        if mask & 1:
            olib().orc_fill_ghost_copy(_ptr(uo), pair.orc.ot.ref, l)
        if mask & 2:
            olib().orc_fill_ghost_bnd(_ptr(uo), pair.orc.ot.ref, l, _ptr(pair.bcp))
        if mask & 4:
            olib().orc_fill_ghost_interp(_ptr(uo), pair.orc.ot.ref, l)
        np.testing.assert_array_equal(bits(to_np(ug)), bits(uo), err_msg=f"level {l} mask {mask}")


def test_gs4_colour_bitexact(pair):
    p = pair.p
    u0, b0 = rand(p, 2), rand(p, 3)
    for l in range(1, pair.nlev + 1):
        sl = p.s / 4 ** (l - 1)
        for c in range(4):
            ug, bg = torch_cuda(u0), torch_cuda(b0)
            pair.ctx.check(mg.lib().srmg_gs_level_dev(pair.ctx.handle, ug.data_ptr(), bg.data_ptr(), p.nblk, l,
                                                      1.25, sl, 2, 0.0, p.geom, c))
            pair.ctx.synchronize()
            uo = u0.copy()
            olib().orc_gs4_level(_ptr(uo), _ptr(b0), 1.25, sl, pair.orc.ot.ref, l, ctypes.byref(pair.orc.op),
                                 c >> 1, c & 1)
            np.testing.assert_array_equal(bits(to_np(ug)), bits(uo), err_msg=f"level {l} colour {c}")


def test_gs_iter_bitexact(pair):
    p = pair.p
    u0, b0 = rand(p, 4), pair.rhs()
    for l in range(1, pair.nlev + 1):
        sl = p.s / 4 ** (l - 1)
        ug, bg = torch_cuda(u0), torch_cuda(b0)
        pair.ctx.check(mg.lib().srmg_gs_iter_dev(pair.ctx.handle, ug.data_ptr(), bg.data_ptr(), p.nblk, l, 1.0, sl,
                                                 2, 2, 0.0, p.geom, pair.bcp.ctypes.data))
        pair.ctx.synchronize()
        uo = u0.copy()
        olib().orc_gs_iter(_ptr(uo), _ptr(b0), 1.0, sl, 2, l, pair.orc.ot.ref, ctypes.byref(pair.orc.op))
        np.testing.assert_array_equal(bits(to_np(ug)), bits(uo), err_msg=f"level {l}")


def test_residual_and_postrestrict_bitexact(pair):
    p = pair.p
    u0, b0, r0 = rand(p, 5), rand(p, 6), rand(p, 7)
    for l in range(1, pair.nlev + 1):
        sl = p.s / 4 ** (l - 1)
        ug, bg, rg = torch_cuda(u0), torch_cuda(b0), torch_cuda(r0)
        pair.ctx.check(mg.lib().srmg_residual_level_dev(pair.ctx.handle, rg.data_ptr(), ug.data_ptr(),
                                                        bg.data_ptr(), p.nblk, l, sl, 2, 0.0, p.geom))
        pair.ctx.synchronize()
        ro = r0.copy()
        olib().orc_residual_level(_ptr(ro), _ptr(u0), _ptr(b0), sl, pair.orc.ot.ref, l, ctypes.byref(pair.orc.op))
        np.testing.assert_array_equal(bits(to_np(rg)), bits(ro), err_msg=f"residual level {l}")
        if l >= 2:
            bg, r0g = torch_cuda(b0), torch_cuda(r0)  # held until the kernel has run
            pair.ctx.check(mg.lib().srmg_residual_postrestrict_level_dev(
                pair.ctx.handle, bg.data_ptr(), ug.data_ptr(), r0g.data_ptr(), p.nblk, l, 4 * sl, 2, 0.0,
                p.geom))
            pair.ctx.synchronize()
            bo = b0.copy()
            olib().orc_residual_postrestrict_level(_ptr(bo), _ptr(u0), _ptr(r0), 4 * sl, pair.orc.ot.ref, l,
                                                   ctypes.byref(pair.orc.op))
            np.testing.assert_array_equal(bits(to_np(bg)), bits(bo), err_msg=f"postrestrict level {l}")


@pytest.mark.parametrize("op", [0, 2])
def test_rhs_level_bitexact(pair, op):
    p = pair.p
    q0, q10 = rand(p, 8), rand(p, 9)
    saved = pair.orc.op.op
    pair.orc.op.op = op
    try:
        for l in range(1, pair.nlev + 1):
            qg, q1g = torch_cuda(q0), torch_cuda(q10)
            mg.rhs_level_(pair.ctx, q1g, qg, l, p.geom, "laplacian4" if op == 2 else None)
            pair.ctx.synchronize()
            q1o = q10.copy()
            pair.orc.rhs_level(q1o, q0, l)
            np.testing.assert_array_equal(bits(to_np(q1g)), bits(q1o), err_msg=f"level {l}")
        # the host-array entry point gives the same bits
        q1h = q10.copy()
        mg.rhs_level_(pair.ctx, q1h, q0, pair.nlev, p.geom, "laplacian4" if op == 2 else None)
        q1o = q10.copy()
        pair.orc.rhs_level(q1o, q0, pair.nlev)
        np.testing.assert_array_equal(bits(q1h), bits(q1o))
    finally:
        pair.orc.op.op = saved


def test_vcycle_parity(pair):
    p = pair.p
    b0 = pair.rhs()
    ug, bg = torch_cuda(np.zeros_like(b0)), torch_cuda(b0)
    rg, u1g = torch_cuda(np.zeros_like(b0)), torch_cuda(np.zeros_like(b0))
    mg.vcycle_(pair.ctx, ug, bg, rg, u1g, p.s, p.geom, p.bc, "laplacian4", ndown=2, ntop=4, nup=2, ncycles=3)
    pair.ctx.synchronize()
    uo, bo = np.zeros_like(b0), b0.copy()
    r, u1 = np.zeros_like(b0), np.zeros_like(b0)
    for _ in range(3):
        pair.orc.vcycle(uo, bo, r, u1, ndown=2, ntop=4, nup=2)
    assert rel_l2(to_np(ug), uo) <= REL
    assert rel_l2(to_np(bg), bo) <= REL


def test_fmg_parity(pair):
    p = pair.p
    b0 = pair.rhs()
    ug, bg = torch_cuda(np.zeros_like(b0)), torch_cuda(b0)
    rg, u1g = torch_cuda(np.zeros_like(b0)), torch_cuda(np.zeros_like(b0))
    mg.fmg_(pair.ctx, ug, bg, rg, u1g, p.s, p.geom, p.bc, "laplacian4", ndown=2, ntop=4, nup=2)
    pair.ctx.synchronize()
    uo, bo = np.zeros_like(b0), b0.copy()
    pair.orc.fmg(uo, bo, np.zeros_like(b0), np.zeros_like(b0), ndown=2, ntop=4, nup=2)
    assert rel_l2(to_np(ug), uo) <= REL


def test_solve_fp64_to_tolerance(pair):
    p = pair.p
    b0 = pair.rhs()
    u = np.zeros_like(b0)
    st = mg.solve(pair.ctx, u, b0, p.s, p.geom, p.bc, "laplacian4", tol=1e-9, mode=mg.MODE_FP64,
                  max_cycles=2000)
    assert st["rel_residual"] <= 1e-9
    # the oracle's norms of the returned iterate agree
    rel = pair.orc.resnorm(np.zeros_like(u), b0, u) / pair.orc.leafnorm(b0)
    assert abs(rel - st["rel_residual"]) <= 1e-9 * rel


def test_order2_helmholtz_on_box_tree(pair):
    """The photoionization terms run order 2 on the same BoxStencil connectivity
    (src/photo.jl:53, src/simulate.jl:260-262): per-operation kernels, corners filled,
    every cell (ghosts included) equal to the oracle's to rounding."""
    p = pair.p
    k2 = 2.5e5
    ctx = pair.ctx
    b0 = pair.rhs()
    ug, bg = torch_cuda(np.zeros_like(b0)), torch_cuda(b0)
    rg, u1g = torch_cuda(np.zeros_like(b0)), torch_cuda(np.zeros_like(b0))
    s = p.h1 ** 2
    mg.vcycle_(ctx, ug, bg, rg, u1g, s, p.geom, p.bc, ("helmholtz", k2), ndown=2, ntop=4, nup=2, ncycles=2)
    ctx.synchronize()
    saved = (pair.orc.op.op, pair.orc.op.k2)
    pair.orc.op.op, pair.orc.op.k2 = 1, k2
    try:
        uo, bo = np.zeros_like(b0), b0.copy()
        r, u1 = np.zeros_like(b0), np.zeros_like(b0)
        for _ in range(2):
            pair.orc.vcycle(uo, bo, r, u1, ndown=2, ntop=4, nup=2, s=s)
    finally:
        pair.orc.op.op, pair.orc.op.k2 = saved
    used = np.zeros(p.nblk, dtype=bool)
    for layer in p.tree:
        for _, blk in layer.pairs:
            used[blk - 1] = True
    assert rel_l2(to_np(ug)[used], uo[used]) <= REL
    # corner ghosts are filled on the GPU exactly where the oracle fills them
    ugn = to_np(ug)[used]
    for sl in (np.s_[:, 0:2, 0:2], np.s_[:, 0:2, 18:20], np.s_[:, 18:20, 0:2], np.s_[:, 18:20, 18:20]):
        assert rel_l2(ugn[sl], uo[used][sl]) <= REL


def test_unsupported_combinations(pair):
    p = pair.p
    b0 = pair.rhs()
    u = np.zeros_like(b0)
    with pytest.raises(mg.SrmgError) as ei:
        mg.solve(pair.ctx, u, b0, p.s, p.geom, p.bc, "laplacian4", tol=1e-8, mode=mg.MODE_MIXED)
    assert ei.value.code == SRMG_ERR_UNSUPPORTED
    # order 4 on a StarStencil tree has no corner ghosts: refused
    star = mg.Context(0).set_tree(p.tree, connectivity(p.tree))
    with pytest.raises(mg.SrmgError) as ei:
        mg.vcycle_(star, u.copy(), b0.copy(), u.copy(), u.copy(), p.s, p.geom, p.bc, "laplacian4")
    assert ei.value.code == SRMG_ERR_UNSUPPORTED
    star.close()


@pytest.mark.parametrize("root,levels,geom", [((1, 1), 1, gen.GEOM_CART), ((2, 1), 3, gen.GEOM_CYL1),
                                              ((1, 2), 3, gen.GEOM_CYL2)])
def test_small_and_oblong_trees(root, levels, geom):
    """Edge cases: a single block (every ghost, corners included, from the boundary) and
    oblong root grids, uniform trees with BoxStencil connectivity."""
    from srmg.tree import Tree, populate
    t = Tree(root, levels)
    populate(t, levels)
    conn = connectivity(t, BOX2)
    bc = {gen.GEOM_CART: gen.boundaryconditions(((-1, -1), (-1, -1))), gen.GEOM_CYL1: gen.BC_POISSON,
          gen.GEOM_CYL2: gen.boundaryconditions(((-1, -1), (1, 1)))}[geom]
    p = gen.make_problem(t, lambda r, z, l, gi, gj: np.exp(-((r - 0.004) ** 2 + (z - 0.006) ** 2) / 1e-5) * 1e18,
                         gen.poisson_scale(), op=gen.OP_LAPLACIAN4, bc=bc, conn=conn)
    p.geom = geom
    pr = Pair(p)
    b0 = pr.rhs()
    z = np.zeros_like(b0)
    ug, bg, rg, u1g = torch_cuda(z), torch_cuda(b0), torch_cuda(z), torch_cuda(z)
    mg.vcycle_(pr.ctx, ug, bg, rg, u1g, p.s, p.geom, p.bc, "laplacian4", ndown=2, ntop=4, nup=2, ncycles=2)
    pr.ctx.synchronize()
    uo, bo = z.copy(), b0.copy()
    for _ in range(2):
        pr.orc.vcycle(uo, bo, z.copy(), z.copy(), ndown=2, ntop=4, nup=2)
    assert rel_l2(to_np(ug), uo) <= REL
    pr.ctx.close()
