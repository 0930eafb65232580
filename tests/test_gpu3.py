"""Parity of the three-dimensional path (D = 3 contexts, through the C ABI) with the
3D oracle (oracle/srmg_oracle3.c).

Bars: ghost fills (every pass and the whole fill), Gauss-Seidel colour sweeps and
iterations (red-black and four-colour), the residual, the FAS coarse right-hand side,
restriction, prolongation and rhs_level! are bit-exact (both sides round every
operation on its own, in the reference's order, and fuse exactly where it calls
muladd); V-cycles and FMG agree to <= 1e-12 relative L2; the FP64 solve reaches its
tolerance with the oracle's norm of its result.
"""
import ctypes

import numpy as np
import pytest

from conftest import gpu_available
from oracle import Oracle3, lib as olib, _ptr
from srmg import gen3, multigrid as mg
from srmg.tree3 import Tree3, populate, connectivity, STAR3, BOX3

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]

REL = 1e-12
SRMG_ERR_BADARG, SRMG_ERR_UNSUPPORTED = -1, -6


def torch_cuda(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    torch.cuda.synchronize()
    return t


def bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


def rel_l2(a, b):
    n = np.linalg.norm(np.ravel(b))
    return np.linalg.norm(np.ravel(a - b)) / (n if n > 0 else 1.0)


def permuted(p, seed):
    rng = np.random.default_rng(seed)
    n = p.nblk
    nalloc = n + 3
    perm = rng.permutation(nalloc)[:n] + 1
    for layer in p.tree:
        idx = {c: int(perm[b - 1]) for c, b in layer.index.items()}
        layer.index = idx
        layer.coord = {b: c for c, b in idx.items()}
        layer.sync(rng)
    conn = connectivity(p.tree, STAR3)
    for lists in (conn.neighbor, conn.boundary, conn.refboundary, conn.child):
        for k, arr in enumerate(lists):
            lists[k] = arr[rng.permutation(len(arr))]
    b = np.zeros((nalloc, 20, 20, 20))
    b[perm - 1] = p.b
    return gen3.Problem3(tree=p.tree, conn=conn, b=b, s=p.s, op=p.op, k2=p.k2, bc=p.bc, h1=p.h1,
                         name=p.name + "-perm")


PROBS = {
    "lapl2": gen3.refined3(seed=31, op=0),
    "helm2": gen3.refined3(seed=32, op=1, k2=50.0),
    "lapl4_box": gen3.refined3(seed=33, op=2),
    "lapl2_perm": permuted(gen3.refined3(seed=34, op=0), 7),
}


def lpl(p):
    return {0: None, 1: ("helmholtz", p.k2), 2: "laplacian4"}[p.op]


class Pair:
    def __init__(self, p):
        self.p = p
        self.ctx = mg.Context(0, D=3).set_tree(p.tree, p.conn)
        self.orc = Oracle3(p)
        self.bcp = np.ascontiguousarray(p.bc, dtype=np.int8)
        self.nlev = len(p.tree)

    def rhs(self):
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
    return np.random.default_rng(seed).standard_normal(p.b.shape)


@pytest.mark.parametrize("mask", [1, 2, 3, 4, 5, 6, 7])
def test_fill_ghost_bitexact(pair, mask):
    p = pair.p
    u0 = rand(p, 1)
    for l in range(1, pair.nlev + 1):
        ug = torch_cuda(u0)
        mg.fill_ghost_(pair.ctx, ug, l, p.bc, mask=mask)
        pair.ctx.synchronize()
        uo = u0.copy()
        if mask & 1:
            olib().orc3_fill_ghost_copy(_ptr(uo), pair.orc.ot.ref, l)
        if mask & 2:
            olib().orc3_fill_ghost_bnd(_ptr(uo), pair.orc.ot.ref, l, _ptr(pair.bcp))
        if mask & 4:
            olib().orc3_fill_ghost_interp(_ptr(uo), pair.orc.ot.ref, l)
        np.testing.assert_array_equal(bits(ug.cpu().numpy()), bits(uo), err_msg=f"level {l} mask {mask}")


def test_gs_colours_bitexact(pair):
    p = pair.p
    u0, b0 = rand(p, 2), rand(p, 3)
    ncol = 4 if p.op == 2 else 2
    for l in range(1, pair.nlev + 1):
        sl = p.s / 4 ** (l - 1)
        for c in range(ncol):
            ug, bg = torch_cuda(u0), torch_cuda(b0)
            pair.ctx.check(mg.lib().srmg_gs_level_dev(pair.ctx.handle, ug.data_ptr(), bg.data_ptr(), p.nblk, l,
                                                      1.1, sl, p.op, p.k2, 0, c))
            pair.ctx.synchronize()
            uo = u0.copy()
            if p.op == 2:
                olib().orc3_gs4_level(_ptr(uo), _ptr(b0), 1.1, sl, pair.orc.ot.ref, l, ctypes.byref(pair.orc.op),
                                      c >> 1, c & 1)
            else:
                olib().orc3_gs_level(_ptr(uo), _ptr(b0), 1.1, sl, pair.orc.ot.ref, l, ctypes.byref(pair.orc.op), c)
            np.testing.assert_array_equal(bits(ug.cpu().numpy()), bits(uo), err_msg=f"level {l} colour {c}")


def test_gs_iter_bitexact(pair):
    p = pair.p
    u0, b0 = rand(p, 4), pair.rhs()
    for l in range(1, pair.nlev + 1):
        sl = p.s / 4 ** (l - 1)
        ug, bg = torch_cuda(u0), torch_cuda(b0)
        pair.ctx.check(mg.lib().srmg_gs_iter_dev(pair.ctx.handle, ug.data_ptr(), bg.data_ptr(), p.nblk, l, 1.0, sl,
                                                 2, p.op, p.k2, 0, pair.bcp.ctypes.data))
        pair.ctx.synchronize()
        uo = u0.copy()
        olib().orc3_gs_iter(_ptr(uo), _ptr(b0), 1.0, sl, 2, l, pair.orc.ot.ref, ctypes.byref(pair.orc.op))
        np.testing.assert_array_equal(bits(ug.cpu().numpy()), bits(uo), err_msg=f"level {l}")


def test_residual_postrestrict_transfers_bitexact(pair):
    p = pair.p
    u0, b0, r0 = rand(p, 5), rand(p, 6), rand(p, 7)
    L = mg.lib()
    for l in range(1, pair.nlev + 1):
        sl = p.s / 4 ** (l - 1)
        ug, bg, rg = torch_cuda(u0), torch_cuda(b0), torch_cuda(r0)
        pair.ctx.check(L.srmg_residual_level_dev(pair.ctx.handle, rg.data_ptr(), ug.data_ptr(), bg.data_ptr(),
                                                 p.nblk, l, sl, p.op, p.k2, 0))
        pair.ctx.synchronize()
        ro = r0.copy()
        olib().orc3_residual_level(_ptr(ro), _ptr(u0), _ptr(b0), sl, pair.orc.ot.ref, l, ctypes.byref(pair.orc.op))
        np.testing.assert_array_equal(bits(rg.cpu().numpy()), bits(ro), err_msg=f"residual {l}")
        if l < 2:
            continue
        bg, r0g = torch_cuda(b0), torch_cuda(r0)  # held until the kernel has run
        pair.ctx.check(L.srmg_residual_postrestrict_level_dev(pair.ctx.handle, bg.data_ptr(), ug.data_ptr(),
                                                              r0g.data_ptr(), p.nblk, l, 4 * sl, p.op,
                                                              p.k2, 0))
        pair.ctx.synchronize()
        bo = b0.copy()
        olib().orc3_residual_postrestrict_level(_ptr(bo), _ptr(u0), _ptr(r0), 4 * sl, pair.orc.ot.ref, l,
                                                ctypes.byref(pair.orc.op))
        np.testing.assert_array_equal(bits(bg.cpu().numpy()), bits(bo), err_msg=f"postrestrict {l}")
        ug = torch_cuda(u0)
        pair.ctx.check(L.srmg_restrict_level_dev(pair.ctx.handle, ug.data_ptr(), p.nblk, l))
        pair.ctx.synchronize()
        uo = u0.copy()
        olib().orc3_restrict_level(_ptr(uo), pair.orc.ot.ref, l)
        np.testing.assert_array_equal(bits(ug.cpu().numpy()), bits(uo), err_msg=f"restrict {l}")
        ug, vg = torch_cuda(u0), torch_cuda(r0)
        pair.ctx.check(L.srmg_interp_add_level_dev(pair.ctx.handle, ug.data_ptr(), vg.data_ptr(), p.nblk, l))
        pair.ctx.synchronize()
        uo = u0.copy()
        olib().orc3_interp_add_level(_ptr(uo), _ptr(r0), pair.orc.ot.ref, l)
        np.testing.assert_array_equal(bits(ug.cpu().numpy()), bits(uo), err_msg=f"interp_add {l}")


def test_rhs_level_bitexact(pair):
    p = pair.p
    q0, q10 = rand(p, 8), rand(p, 9)
    for l in range(1, pair.nlev + 1):
        qg, q1g = torch_cuda(q0), torch_cuda(q10)
        mg.rhs_level_(pair.ctx, q1g, qg, l, 0, lpl(p))
        pair.ctx.synchronize()
        q1o = q10.copy()
        pair.orc.rhs_level(q1o, q0, l)
        np.testing.assert_array_equal(bits(q1g.cpu().numpy()), bits(q1o), err_msg=f"level {l}")


def test_vcycle_and_fmg_parity(pair):
    p = pair.p
    b0 = pair.rhs()
    z = np.zeros_like(b0)
    ug, bg, rg, u1g = torch_cuda(z), torch_cuda(b0), torch_cuda(z), torch_cuda(z)
    mg.vcycle_(pair.ctx, ug, bg, rg, u1g, p.s, 0, p.bc, lpl(p), ndown=2, ntop=4, nup=2, ncycles=3)
    pair.ctx.synchronize()
    uo, bo = z.copy(), b0.copy()
    for _ in range(3):
        pair.orc.vcycle(uo, bo, z.copy(), z.copy(), ndown=2, ntop=4, nup=2)
    assert rel_l2(ug.cpu().numpy(), uo) <= REL
    assert rel_l2(bg.cpu().numpy(), bo) <= REL
    # host-array entry point and FMG
    uh, bh = z.copy(), b0.copy()
    mg.fmg_(pair.ctx, uh, bh, z.copy(), z.copy(), p.s, 0, p.bc, lpl(p), ndown=2, ntop=4, nup=2)
    uo = z.copy()
    pair.orc.fmg(uo, b0.copy(), z.copy(), z.copy(), ndown=2, ntop=4, nup=2)
    assert rel_l2(uh, uo) <= REL


def test_solve_fp64(pair):
    p = pair.p
    b0 = pair.rhs()
    u = np.zeros_like(b0)
    st = mg.solve(pair.ctx, u, b0, p.s, 0, p.bc, lpl(p), tol=1e-9, mode=mg.MODE_FP64, max_cycles=500)
    assert st["rel_residual"] <= 1e-9
    rel = pair.orc.resnorm(np.zeros_like(u), b0, u) / pair.orc.leafnorm(b0)
    assert abs(rel - st["rel_residual"]) <= 1e-9 * rel


def test_three_dimensional_limits(pair):
    p = pair.p
    b0 = pair.rhs()
    u = np.zeros_like(b0)
    with pytest.raises(mg.SrmgError) as ei:
        mg.solve(pair.ctx, u, b0, p.s, 0, p.bc, lpl(p), tol=1e-8, mode=mg.MODE_MIXED)
    assert ei.value.code == SRMG_ERR_UNSUPPORTED
    with pytest.raises(mg.SrmgError) as ei:     # a 2D-only entry point
        mg.netcharge(pair.ctx, u.copy(), u.copy(), u.copy())
    assert ei.value.code == SRMG_ERR_UNSUPPORTED
    with pytest.raises(mg.SrmgError) as ei:     # cylindrical geometry
        mg.vcycle_(pair.ctx, u.copy(), b0.copy(), u.copy(), u.copy(), p.s, 1, p.bc, lpl(p))
    assert ei.value.code == SRMG_ERR_UNSUPPORTED


def test_oblong_root_and_partial_vcycle():
    """An octree on a (2, 1, 1) root grid with refinement, and V-cycles that stop at a
    level below the finest (lmax)."""
    from srmg.tree3 import refine_block
    t = Tree3((2, 1, 1), 4)
    populate(t, 2)
    refine_block(t, 2, (3, 2, 1))
    t.sync()
    conn = connectivity(t, STAR3)
    p = gen3.make_problem3(t, conn, lambda x, y, z: np.exp(-((x - 1.2) ** 2 + (y - 0.6) ** 2 + z ** 2) / 0.05),
                           (1.0 / 16) ** 2)
    pr = Pair(p)
    b0 = pr.rhs()
    z0 = np.zeros_like(b0)
    for lmax in (0, 2):
        ug, bg, rg, u1g = torch_cuda(z0), torch_cuda(b0), torch_cuda(z0), torch_cuda(z0)
        mg.vcycle_(pr.ctx, ug, bg, rg, u1g, p.s, 0, p.bc, None, lmax=lmax, ndown=2, ntop=4, nup=2, ncycles=2)
        pr.ctx.synchronize()
        uo, bo = z0.copy(), b0.copy()
        for _ in range(2):
            pr.orc.vcycle(uo, bo, z0.copy(), z0.copy(), lmax=lmax, ndown=2, ntop=4, nup=2)
        assert rel_l2(ug.cpu().numpy(), uo) <= REL, lmax
    pr.ctx.close()
