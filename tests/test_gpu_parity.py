"""Parity of the CUDA path (called through the C ABI) with the oracle.

Bars: ghost fills, restriction and prolongation are bit-exact (integer/indexing work
plus the reference's fixed-order, non-fused arithmetic).  The per-operation kernels'
stencils round every product and sum on their own, as the oracle does (the
reference's @fastmath leaves contraction open; the oracle takes the uncontracted
reading), so GS sweeps, residuals and whole per-operation V-cycles are bit-exact too.
The persistent engine rounds the same way (its stencil is apply5's, operation by
operation), so its V-cycles are bit-exact as well, in both launch shapes: the potential
on every element (ghosts included) and the FAS right-hand sides on the valid cells (the
engine also keeps b's neighbour-copy ghosts filled, which the oracle leaves alone).
"""
import numpy as np
import pytest

from conftest import gpu_available
from oracle import Oracle, lib as olib, _ptr
from srmg import gen, multigrid as mg
from srmg.tree import connectivity

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]



def assert_bitexact(gu, uo, gb=None, bo=None):
    """u equal on every element, ghosts included; b on the valid cells."""
    assert np.array_equal(gu.view(np.uint64), uo.view(np.uint64)), \
        f"{int((gu.view(np.uint64) != uo.view(np.uint64)).sum())} elements of u differ"
    if gb is not None:
        vm = valid_mask(gu.shape)
        assert np.array_equal(gb.view(np.uint64)[vm], bo.view(np.uint64)[vm]), \
            f"{int((gb.view(np.uint64) != bo.view(np.uint64))[vm].sum())} valid cells of b differ"


def torch_cuda(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    torch.cuda.synchronize()  # the context's stream does not order after torch's
    return t


def to_np(t):
    return t.cpu().numpy()


def rel_l2(a, b, mask=None):
    if mask is not None:
        a, b = a[mask], b[mask]
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return d / n if n > 0 else d


def valid_mask(shape):
    m = np.zeros(shape, dtype=bool)
    m[:, 2:18, 2:18] = True
    return m


def permute_blocks(p, seed):
    """Renumber blocks with a random permutation (leaving gaps: nblk_alloc grows),
    shuffle every level's pairs order and every edge list: results must not depend on
    block numbering or on the Dict order of BlockLayer.pairs (src/blocklayer.jl:48-53)."""
    rng = np.random.default_rng(seed)
    n = p.nblk
    nalloc = n + 7
    perm = rng.permutation(nalloc)[:n] + 1  # old id i -> perm[i-1]
    tree = p.tree
    for layer in tree:
        new_index = {c: int(perm[b - 1]) for c, b in layer.index.items()}
        layer.index = new_index
        layer.coord = {b: c for c, b in new_index.items()}
        layer.sync(rng)
    conn = connectivity(tree)
    for lists in (conn.neighbor, conn.boundary, conn.refboundary, conn.child):
        for k, arr in enumerate(lists):
            lists[k] = arr[rng.permutation(len(arr))]
    b = np.zeros((nalloc, 20, 20))
    b[perm - 1] = p.b
    return gen.Problem(tree=tree, conn=conn, b=b, s=p.s, op=p.op, k2=p.k2, geom=p.geom,
                       bc=p.bc, h1=p.h1, name=p.name + "-permuted")


def problems():
    out = {}
    out["uniform4"] = gen.make_problem(gen._uniform(4), lambda r, z, l, gi, gj: np.sin(r * 900) * np.cos(z * 700) * 1e19,
                                       gen.poisson_scale(), name="uniform4")
    p = gen.config2(seed=5, target_leaf=40_000, extra=3)
    out["refined"] = p
    out["refined_perm"] = permute_blocks(gen.config2(seed=5, target_leaf=40_000, extra=3), 9)
    return out


PROBS = problems()


class Pair:
    """A problem with its GPU context and oracle."""

    def __init__(self, p):
        self.p = p
        self.ctx = mg.Context(0).set_tree(p.tree, p.conn)
        self.orc = Oracle(p)


@pytest.fixture(scope="module", params=list(PROBS))
def pair(request):
    return Pair(PROBS[request.param])


def random_field(p, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((p.nblk, 20, 20))


@pytest.mark.parametrize("mask", [1, 2, 4, 7])
def test_fill_ghost_bitexact(pair, mask):
    p = pair.p
    u0 = random_field(p, 1)
    for l in range(1, len(p.tree) + 1):
        ug = torch_cuda(u0)
        mg.fill_ghost_(pair.ctx, ug, l, p.bc, mask=mask)
        pair.ctx.synchronize()
        uo = u0.copy()
        bcp = np.ascontiguousarray(p.bc, dtype=np.int8)
        if mask & 1:
            olib().orc_fill_ghost_copy(_ptr(uo), pair.orc.ot.ref, l)
        if mask & 2:
            olib().orc_fill_ghost_bnd(_ptr(uo), pair.orc.ot.ref, l, _ptr(bcp))
        if mask & 4:
            olib().orc_fill_ghost_interp(_ptr(uo), pair.orc.ot.ref, l)
        np.testing.assert_array_equal(to_np(ug).view(np.uint64), uo.view(np.uint64),
                                      err_msg=f"level {l} mask {mask}")


def test_restrict_and_interp_bitexact(pair):
    p = pair.p
    u0, u1 = random_field(p, 2), random_field(p, 3)
    for l in range(2, len(p.tree) + 1):
        ug = torch_cuda(u0)
        mg.lib().srmg_restrict_level_dev(pair.ctx.handle, ug.data_ptr(), p.nblk, l)
        pair.ctx.synchronize()
        uo = u0.copy()
        olib().orc_restrict_level(_ptr(uo), pair.orc.ot.ref, l)
        assert np.array_equal(to_np(ug).view(np.uint64), uo.view(np.uint64)), f"restrict l{l}"
        ug = torch_cuda(u0)
        vg = torch_cuda(u1)
        pair.ctx.check(mg.lib().srmg_interp_add_level_dev(pair.ctx.handle, ug.data_ptr(), vg.data_ptr(), p.nblk, l))
        pair.ctx.synchronize()
        uo = u0.copy()
        olib().orc_interp_add_level(_ptr(uo), _ptr(u1), pair.orc.ot.ref, l)
        assert np.array_equal(to_np(ug).view(np.uint64), uo.view(np.uint64)), f"interp_add l{l}"


@pytest.mark.parametrize("parity", [0, 1])
def test_gs_colour_sweep(pair, parity):
    import ctypes
    p = pair.p
    u0, b0 = random_field(p, 4), random_field(p, 5)
    l = len(p.tree)
    sl = 0.3
    ug, bg = torch_cuda(u0), torch_cuda(b0)
    pair.ctx.check(mg.lib().srmg_gs_level_dev(pair.ctx.handle, ug.data_ptr(), bg.data_ptr(), p.nblk, l,
                                              1.0, sl, p.op, p.k2, p.geom, parity))
    pair.ctx.synchronize()
    uo = u0.copy()
    olib().orc_gs_level(_ptr(uo), _ptr(b0), 1.0, sl, pair.orc.ot.ref, l, ctypes.byref(pair.orc.op), parity)
    got = to_np(ug)
    assert np.array_equal(got[:, :2], uo[:, :2])  # ghosts untouched
    assert np.array_equal(got.view(np.uint64), uo.view(np.uint64))  # the reference's rounding


@pytest.mark.parametrize("n", [1, 2, 3])
def test_gs_iter_matches_oracle(pair, n):
    """gauss_seidel_iter! (red, copy+mirror fills, black, fills) n times on one level."""
    import ctypes
    p = pair.p
    u0, b0 = random_field(p, 14), random_field(p, 15)
    l = len(p.tree)
    while l > 1 and len(p.tree[l - 1]) == 0:
        l -= 1
    uo = u0.copy()
    pair.orc.fill_ghost(uo, l)
    ug, bg = torch_cuda(uo), torch_cuda(b0)
    bca = np.ascontiguousarray(p.bc, dtype=np.int8)
    pair.ctx.check(mg.lib().srmg_gs_iter_dev(pair.ctx.handle, ug.data_ptr(), bg.data_ptr(), p.nblk, l, 1.0,
                                             0.3, n, p.op, p.k2, p.geom, bca.ctypes.data))
    pair.ctx.synchronize()
    olib().orc_gs_iter(_ptr(uo), _ptr(b0), 1.0, 0.3, n, l, pair.orc.ot.ref, ctypes.byref(pair.orc.op))
    got = to_np(ug)
    assert rel_l2(got, uo) < 1e-13
    corner = np.zeros((20, 20), dtype=bool)
    corner[:2, :2] = corner[:2, 18:] = corner[18:, :2] = corner[18:, 18:] = True
    assert np.array_equal(got[:, corner], uo[:, corner])  # corner ghosts never written


def test_residual_level(pair):
    import ctypes
    p = pair.p
    u0, b0 = random_field(p, 6), random_field(p, 7)
    for l in range(1, len(p.tree) + 1):
        sl = gen.poisson_scale() / 4 ** (l - 1)
        ug, bg, rg = torch_cuda(u0), torch_cuda(b0), torch_cuda(np.zeros_like(u0))
        pair.ctx.check(mg.lib().srmg_residual_level_dev(pair.ctx.handle, rg.data_ptr(), ug.data_ptr(),
                                                        bg.data_ptr(), p.nblk, l, sl, p.op, p.k2, p.geom))
        pair.ctx.synchronize()
        ro = np.zeros_like(u0)
        olib().orc_residual_level(_ptr(ro), _ptr(u0), _ptr(b0), sl, pair.orc.ot.ref, l, ctypes.byref(pair.orc.op))
        assert np.array_equal(to_np(rg).view(np.uint64), ro.view(np.uint64)), f"level {l}"


def _prepared(pair):
    p = pair.p
    u = np.zeros_like(p.b)
    pair.orc.fill_ghost_all(u)
    return u, p.b.copy()


@pytest.mark.parametrize("threads", [768, 1024])
@pytest.mark.parametrize("ncycles", [1, 3])
def test_vcycle_matches_oracle(pair, ncycles, threads):
    """The persistent engine's V-cycles (either launch shape) == the oracle's, bit for bit."""
    p = pair.p
    u, b = _prepared(pair)
    ug, bg = torch_cuda(u), torch_cuda(b)
    rg, u1g = torch_cuda(np.zeros_like(u)), torch_cuda(np.zeros_like(u))
    pair.ctx.set_option("engine_threads", threads)
    mg.vcycle_(pair.ctx, ug, bg, rg, u1g, p.s, p.geom, p.bc, ndown=2, ntop=4, nup=2, ncycles=ncycles)
    pair.ctx.synchronize()
    pair.ctx.set_option("engine_threads", 0)
    uo, bo = u.copy(), b.copy()
    r, u1 = np.zeros_like(u), np.zeros_like(u)
    for _ in range(ncycles):
        pair.orc.vcycle(uo, bo, r, u1, ndown=2, ntop=4, nup=2)
    assert_bitexact(to_np(ug), uo, to_np(bg), bo)


def test_engine_matches_per_operation_kernels(pair):
    """The persistent one-launch V-cycle reproduces the per-operation kernel sequence bit
    for bit."""
    p = pair.p
    u, b = _prepared(pair)
    out = {}
    for engine in (0, 1):
        pair.ctx.set_option("engine", engine)
        ug, bg = torch_cuda(u), torch_cuda(b)
        mg.vcycle_(pair.ctx, ug, bg, torch_cuda(np.zeros_like(u)), torch_cuda(np.zeros_like(u)), p.s,
                   p.geom, p.bc, ndown=2, ntop=4, nup=2, ncycles=2)
        pair.ctx.synchronize()
        out[engine] = (to_np(ug), to_np(bg))
    pair.ctx.set_option("engine", 1)
    assert_bitexact(out[1][0], out[0][0], out[1][1], out[0][1])


@pytest.mark.parametrize("local_max", [0, 4, 64])
def test_engine_local_levels(local_max):
    """Coarse levels run inside one CTA or across the grid: same iterates."""
    p = PROBS["refined"]
    pr = Pair(p)
    u, b = _prepared(pr)
    pr.ctx.set_option("local_max_blocks", local_max)
    ug, bg = torch_cuda(u), torch_cuda(b)
    mg.vcycle_(pr.ctx, ug, bg, torch_cuda(np.zeros_like(u)), torch_cuda(np.zeros_like(u)), p.s, p.geom,
               p.bc, ndown=2, ntop=4, nup=2, ncycles=2)
    pr.ctx.synchronize()
    uo, bo = u.copy(), b.copy()
    r, u1 = np.zeros_like(u), np.zeros_like(u)
    for _ in range(2):
        pr.orc.vcycle(uo, bo, r, u1, ndown=2, ntop=4, nup=2)
    assert_bitexact(to_np(ug), uo, to_np(bg), bo)


def test_vcycle_host_pointer_entry_point(pair):
    """srmg_vcycle (host arrays, the ccall boundary) == the device entry point.  b is
    not copied back by default (its leaf cells are never written); with "b_copy_back"
    it returns the FAS values of the covered cells as the device path leaves them.
    Page-locked (registered) host arrays give the same results."""
    p = pair.p
    u, b = _prepared(pair)
    ug, bg = torch_cuda(u), torch_cuda(b)
    mg.vcycle_(pair.ctx, ug, bg, torch_cuda(np.zeros_like(u)), torch_cuda(np.zeros_like(u)), p.s,
               p.geom, p.bc, ndown=2, ntop=4, nup=2, ncycles=2)
    pair.ctx.synchronize()
    for copy_back, register in ((0, False), (1, False), (0, True)):
        pair.ctx.set_option("b_copy_back", copy_back)
        uh, bh = u.copy(), b.copy()
        if register:
            for a in (uh, bh):
                pair.ctx.check(mg.lib().srmg_host_register(pair.ctx.handle, a.ctypes.data, a.nbytes))
        mg.vcycle_(pair.ctx, uh, bh, np.zeros_like(u), np.zeros_like(u), p.s, p.geom, p.bc,
                   ndown=2, ntop=4, nup=2, ncycles=2)
        assert np.array_equal(uh.view(np.uint64), to_np(ug).view(np.uint64))
        want_b = to_np(bg) if copy_back else b
        assert np.array_equal(bh.view(np.uint64), want_b.view(np.uint64))
        if register:
            for a in (uh, bh):
                pair.ctx.check(mg.lib().srmg_host_unregister(pair.ctx.handle, a.ctypes.data))
    pair.ctx.set_option("b_copy_back", 0)
    # the leaf cells of b are the same either way
    leaf = leaf_mask(p)
    assert np.array_equal(to_np(bg)[leaf], b[leaf])


@pytest.mark.parametrize("variant", ["helmholtz", "cartesian", "cyl2", "default_bc", "omega"])
def test_vcycle_operator_variants(variant):
    base = PROBS["refined"]
    kw = dict(tree=base.tree, conn=base.conn, b=base.b.copy(), s=base.s, h1=base.h1, name=variant)
    omega = 1.0
    if variant == "helmholtz":
        p = gen.Problem(**kw, op=gen.OP_HELMHOLTZ, k2=3.1e6, geom=gen.GEOM_CYL1, bc=gen.BC_PHOTO)
        p.s = base.h1 ** 2
    elif variant == "cartesian":
        p = gen.Problem(**kw, geom=gen.GEOM_CART)
    elif variant == "cyl2":
        p = gen.Problem(**kw, geom=gen.GEOM_CYL2)
    elif variant == "default_bc":
        p = gen.Problem(**kw, bc=gen.BC_REFERENCE_DEFAULT)
    else:
        p = gen.Problem(**kw)
        omega = 1.25
    pr = Pair(p)
    u, b = _prepared(pr)
    ug, bg = torch_cuda(u), torch_cuda(b)
    lpl = ("helmholtz", p.k2) if p.op == 1 else None
    mg.vcycle_(pr.ctx, ug, bg, torch_cuda(np.zeros_like(u)), torch_cuda(np.zeros_like(u)), p.s, p.geom,
               p.bc, lpldisc=lpl, ndown=2, ntop=4, nup=2, omega=omega, ncycles=2)
    pr.ctx.synchronize()
    uo, bo = u.copy(), b.copy()
    r, u1 = np.zeros_like(u), np.zeros_like(u)
    for _ in range(2):
        pr.orc.vcycle(uo, bo, r, u1, ndown=2, ntop=4, nup=2, omega=omega)
    assert_bitexact(to_np(ug), uo, to_np(bg), bo)


@pytest.mark.parametrize("sequencer", [0, 1])
@pytest.mark.parametrize("variant", ["uniform4", "refined", "refined_perm", "helmholtz", "cartesian", "cyl2",
                                     "default_bc", "omega"])
def test_per_operation_vcycle_bitexact(variant, sequencer):
    """The per-operation V-cycle (engine off; kernel by kernel, or as one sequencer
    launch) reproduces the oracle's vcycle! bit for bit: every product and sum of the
    stencils is rounded on its own as in the reference, fma() stands for its muladd
    pair, and the fills, restriction and prolongation keep its operation order.  Checked
    on every element, ghosts and the FAS right-hand sides included."""
    if variant in PROBS:
        p, omega = PROBS[variant], 1.0
    else:
        base = PROBS["refined"]
        kw = dict(tree=base.tree, conn=base.conn, b=base.b.copy(), s=base.s, h1=base.h1, name=variant)
        omega = 1.25 if variant == "omega" else 1.0
        if variant == "helmholtz":
            p = gen.Problem(**kw, op=gen.OP_HELMHOLTZ, k2=3.1e6, geom=gen.GEOM_CYL1, bc=gen.BC_PHOTO)
            p.s = base.h1 ** 2
        elif variant == "cartesian":
            p = gen.Problem(**kw, geom=gen.GEOM_CART)
        elif variant == "cyl2":
            p = gen.Problem(**kw, geom=gen.GEOM_CYL2)
        elif variant == "default_bc":
            p = gen.Problem(**kw, bc=gen.BC_REFERENCE_DEFAULT)
        else:
            p = gen.Problem(**kw)
    pr = Pair(p)
    pr.ctx.set_option("engine", 0).set_option("op_graphs", 0).set_option("op_sequencer", sequencer)
    u, b = _prepared(pr)
    ug, bg = torch_cuda(u), torch_cuda(b)
    lpl = ("helmholtz", p.k2) if p.op == 1 else None
    mg.vcycle_(pr.ctx, ug, bg, torch_cuda(np.zeros_like(u)), torch_cuda(np.zeros_like(u)), p.s, p.geom,
               p.bc, lpldisc=lpl, ndown=2, ntop=4, nup=2, omega=omega, ncycles=2)
    pr.ctx.synchronize()
    uo, bo = u.copy(), b.copy()
    r, u1 = np.zeros_like(u), np.zeros_like(u)
    for _ in range(2):
        pr.orc.vcycle(uo, bo, r, u1, ndown=2, ntop=4, nup=2, omega=omega)
    assert np.array_equal(to_np(ug).view(np.uint64), uo.view(np.uint64))
    assert np.array_equal(to_np(bg).view(np.uint64), bo.view(np.uint64))
    pr.ctx.close()


def test_fmg_matches_oracle(pair):
    p = pair.p
    u, b = _prepared(pair)
    ug, bg = torch_cuda(u), torch_cuda(b)
    mg.fmg_(pair.ctx, ug, bg, torch_cuda(np.zeros_like(u)), torch_cuda(np.zeros_like(u)), p.s, p.geom,
            p.bc, ndown=2, ntop=4, nup=2)
    pair.ctx.synchronize()
    uo, bo = u.copy(), b.copy()
    pair.orc.fmg(uo, bo, np.zeros_like(u), np.zeros_like(u), ndown=2, ntop=4, nup=2)
    assert_bitexact(to_np(ug), uo, to_np(bg), bo)


def test_resnorm_matches_oracle(pair):
    p = pair.p
    u, b = _prepared(pair)
    r, u1 = np.zeros_like(u), np.zeros_like(u)
    pair.orc.vcycle(u, b.copy(), r, u1, ndown=2, ntop=4, nup=2)
    pair.orc.fill_ghost_all(u)
    got = mg.resnorm(pair.ctx, None, torch_cuda(b), torch_cuda(u), p.s, p.geom, p.bc)
    want = pair.orc.resnorm(np.zeros_like(u), b, u)
    assert abs(got - want) <= 1e-10 * abs(want)


def variant_problem(variant):
    base = PROBS["refined"]
    kw = dict(tree=base.tree, conn=base.conn, b=base.b.copy(), s=base.s, h1=base.h1, name=variant)
    if variant == "helmholtz":
        p = gen.Problem(**kw, op=gen.OP_HELMHOLTZ, k2=3.1e6, geom=gen.GEOM_CYL1, bc=gen.BC_PHOTO)
        p.s = base.h1 ** 2
        return p
    if variant == "cartesian":
        return gen.Problem(**kw, geom=gen.GEOM_CART)
    if variant == "cyl2":
        return gen.Problem(**kw, geom=gen.GEOM_CYL2)
    return base


@pytest.mark.parametrize("variant", ["poisson", "helmholtz", "cartesian", "cyl2"])
def test_fp64_solve_to_tolerance(variant):
    """The tolerance-driven FP64 solve (one persistent launch; its halo updates read the
    neighbours' b from the engine copy's ghost layer) runs the oracle's cycle count (+-1:
    the norms are summed in another order) and, with the same count, ends on its iterate
    bit for bit."""
    p = variant_problem(variant)
    pr = Pair(p)
    u, b = _prepared(pr)
    ug = torch_cuda(u)
    lpl = ("helmholtz", p.k2) if p.op == 1 else None
    st = mg.solve(pr.ctx, ug, torch_cuda(b), p.s, p.geom, p.bc, lpldisc=lpl, tol=1e-8, mode=mg.MODE_FP64,
                  max_cycles=2000)
    uo = u.copy()
    c, rel = pr.orc.solve(uo, b.copy(), 1e-8, max_cycles=2000)
    assert st["rel_residual"] <= 1e-8 and rel <= 1e-8
    assert abs(st["cycles"] - c) <= 1
    if st["cycles"] == c:
        vm = valid_mask(u.shape)
        assert np.array_equal(to_np(ug).view(np.uint64)[vm], uo.view(np.uint64)[vm])


@pytest.mark.parametrize("engine", [1, 0])
def test_mixed_solve_reaches_fp64_solution(engine):
    """Mixed precision (FP32 V-cycles, FP64 defect correction, FP64 direct coarsest
    level) reaches the FP64 solution: persistent launch per step, or per-operation kernels."""
    p = PROBS["refined"]
    pr = Pair(p)
    pr.ctx.set_option("engine", engine)
    u, b = _prepared(pr)
    ug = torch_cuda(u)
    st = mg.solve(pr.ctx, ug, torch_cuda(b), p.s, p.geom, p.bc, tol=1e-8, mode=mg.MODE_MIXED,
                  max_cycles=200)
    assert st["rel_residual"] <= 1e-8
    assert st["cycles"] < 40
    # FP64 oracle solution at a tighter tolerance
    uo = u.copy()
    c, rel = pr.orc.solve(uo, b.copy(), 1e-11, max_cycles=5000)
    leaf = leaf_mask(p)
    err = rel_l2(to_np(ug), uo, leaf)
    assert err < 1e-6, err


@pytest.mark.parametrize("variant", ["helmholtz", "cartesian", "cyl2"])
@pytest.mark.parametrize("direct_level", [1, 2])
def test_mixed_solve_direct_levels_operator_variants(variant, direct_level):
    """The mixed solve with the direct FP64 solve on level 1 (one CTA) or level 2 (every
    CTA) reaches the oracle's FP64 solution for the Helmholtz operator (photoionization
    boundary table) and the Cartesian and r = dim 2 geometries, with the autotuner's
    smoother and 3 V-cycles per defect-correction step."""
    p = variant_problem(variant)
    pr = Pair(p)
    pr.ctx.set_option("direct_level", direct_level)
    u, b = _prepared(pr)
    ug = torch_cuda(u)
    lpl = ("helmholtz", p.k2) if p.op == 1 else None
    st = mg.solve(pr.ctx, ug, torch_cuda(b), p.s, p.geom, p.bc, lpldisc=lpl, tol=1e-8, mode=mg.MODE_MIXED,
                  max_cycles=200, inner_cycles=3, **mg.TUNED)
    assert st["rel_residual"] <= 1e-8
    # the smoother was tuned on r = dim 1 trees; with r = dim 2 and the level-1 solve
    # this tree needs 49 cycles
    assert st["cycles"] < 80
    uo = u.copy()
    pr.orc.solve(uo, b.copy(), 1e-11, max_cycles=5000)
    err = rel_l2(to_np(ug), uo, leaf_mask(p))
    assert err < 1e-6, err


def leaf_mask(p):
    m = np.zeros(p.b.shape, dtype=bool)
    for layer in p.tree:
        for c, blk in layer.index.items():
            if p.tree.isleaf(layer.level, c):
                m[blk - 1, 2:18, 2:18] = True
    return m


@pytest.mark.parametrize("direct_level", [1, 2])
def test_fp64_direct_mode_reaches_the_oracle_solution(direct_level):
    """SRMG_MODE_FP64_DIRECT: FP64 V-cycles with the direct FP64 coarsest solve converge
    to the oracle's FP64 solution in far fewer cycles than the reference's 4 top sweeps,
    and to the same solution as the mixed mode; with the direct solve on level 1 (one
    CTA) and on level 2 (every CTA; the default for a lone tree)."""
    p = PROBS["refined"]
    assert len(p.tree[1]) <= 4  # level 2 can be solved directly
    pr = Pair(p)
    pr.ctx.set_option("direct_level", direct_level)
    u, b = _prepared(pr)
    out = {}
    for mode in (mg.MODE_FP64, mg.MODE_FP64_DIRECT, mg.MODE_MIXED):
        ug = torch_cuda(u)
        st = mg.solve(pr.ctx, ug, torch_cuda(b), p.s, p.geom, p.bc, tol=1e-8, mode=mode, max_cycles=2000)
        assert st["rel_residual"] <= 1e-8
        out[mode] = (st["cycles"], to_np(ug))
    assert out[mg.MODE_FP64_DIRECT][0] < out[mg.MODE_FP64][0]
    uo = u.copy()
    pr.orc.solve(uo, b.copy(), 1e-11, max_cycles=5000)
    leaf = leaf_mask(p)
    assert rel_l2(out[mg.MODE_FP64_DIRECT][1], uo, leaf) < 1e-6
    assert rel_l2(out[mg.MODE_FP64_DIRECT][1], out[mg.MODE_MIXED][1], leaf) < 1e-6
