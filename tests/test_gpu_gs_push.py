"""Gauss-Seidel sweeps that write their own ghosts (option `gs_push`, on by default) on
the per-operation path of 2D trees: every colour after the first of a
gauss_seidel_iter! call (src/multigrid.jl:250-295) writes the copy and boundary ghosts of
the cells it updates instead of being followed by a fill launch.  The results must be
the fill path's bit for bit -- V-cycles, FMG, the FP32 mixed solve at order 2 -- on BoxStencil trees
(corner ghosts, order 2 and order 4) and on a StarStencil tree with the persistent engine
off, under each boundary table of the order-4 problems, with fewer launches."""
import numpy as np
import pytest

from conftest import gpu_available
from srmg import gen, multigrid as mg

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]


def cases():
    for geom in (gen.GEOM_CYL1, gen.GEOM_CART, gen.GEOM_CYL2):
        p4 = gen.order4_problem(seed=53 + geom, geom=geom)
        yield f"box_order4_g{geom}", p4, "laplacian4", {}
    p4 = gen.order4_problem(seed=57, geom=gen.GEOM_CYL1)
    yield "box_order2", p4, None, {}
    p2 = gen.config2(seed=5, target_leaf=40_000, extra=3)
    yield "star_order2_engine_off", p2, None, {"engine": 0}
    yield "star_helmholtz_engine_off", p2, ("helmholtz", 3.0 / p2.s), {"engine": 0}


CASES = list(cases())


def _ctx(p, opts, push):
    ctx = mg.Context(0).set_tree(p.tree, p.conn)
    for k, v in dict(opts, op_graphs=0, op_sequencer=0, gs_push=push).items():
        ctx.set_option(k, v)
    return ctx


def _bits(a):
    return a.view(np.uint64)


@pytest.mark.parametrize("case", CASES, ids=lambda c: c[0])
def test_vcycle_and_fmg_push_bit_identical(case):
    import torch
    _, p, lpl, opts = case
    out, launches = {}, {}
    for push in (1, 0):
        ctx = _ctx(p, opts, push)
        b = torch.from_numpy(p.b).cuda()
        u, r, u1 = torch.zeros_like(b), torch.zeros_like(b), torch.zeros_like(b)
        torch.cuda.synchronize()
        l0 = ctx.launches()
        mg.vcycle_(ctx, u, b, r, u1, p.s, p.geom, p.bc, lpl, ndown=2, ntop=4, nup=2, ncycles=2)
        ctx.synchronize()
        launches[push] = ctx.launches() - l0
        v = u.cpu().numpy().copy()
        u.zero_()
        b.copy_(torch.from_numpy(p.b))
        mg.fmg_(ctx, u, b, r, u1, p.s, p.geom, p.bc, lpl, ndown=2, ntop=4, nup=2)
        ctx.synchronize()
        out[push] = (v, u.cpu().numpy().copy())
        ctx.close()
    for a, g, what in zip(out[1], out[0], ("vcycle", "fmg")):
        np.testing.assert_array_equal(_bits(a), _bits(g), err_msg=what)
    assert launches[1] < launches[0]


# (mixed precision takes order-2 discretisations only)
@pytest.mark.parametrize("case", [c for c in CASES if c[0] in ("box_order2", "star_order2_engine_off")],
                         ids=lambda c: c[0])
def test_mixed_solve_push_bit_identical(case):
    import torch
    _, p, lpl, opts = case
    res = {}
    for push in (1, 0):
        ctx = _ctx(p, opts, push)
        b = torch.from_numpy(p.b).cuda()
        u = torch.zeros_like(b)
        st = mg.solve(ctx, u, b, p.s, p.geom, p.bc, lpl, tol=1e-8, mode=mg.MODE_MIXED)
        ctx.synchronize()
        res[push] = (u.cpu().numpy().copy(), st["cycles"])
        ctx.close()
    np.testing.assert_array_equal(_bits(res[1][0]), _bits(res[0][0]))
    assert res[1][1] == res[0][1]


def test_gs_iter_push_with_stale_ghosts():
    """gauss_seidel_iter! on a field whose ghosts hold noise: the first colour's fill
    launch makes them consistent, so the pushes give the fill path's result."""
    import torch
    p = gen.order4_problem(seed=61, geom=gen.GEOM_CYL1)
    rng = np.random.default_rng(61)
    u0 = rng.standard_normal(p.b.shape)
    bc = np.ascontiguousarray(np.asarray(p.bc, dtype=np.int8).reshape(-1))
    for lpl_op in (2, 0):
        res = {}
        for push in (1, 0):
            ctx = _ctx(p, {}, push)
            outs = []
            for l in range(1, p.tree.finest_level() + 1):
                ug, bg = torch.from_numpy(u0).cuda(), torch.from_numpy(p.b).cuda()
                sl = p.s / 4 ** (l - 1)
                ctx.check(mg.lib().srmg_gs_iter_dev(ctx.handle, ug.data_ptr(), bg.data_ptr(), p.b.shape[0], l, 1.1,
                                                    sl, 3, lpl_op, 0.0, p.geom, bc.ctypes.data))
                ctx.synchronize()
                outs.append(ug.cpu().numpy())
            res[push] = outs
            ctx.close()
        for l, (a, g) in enumerate(zip(res[1], res[0])):
            np.testing.assert_array_equal(_bits(a), _bits(g), err_msg=f"op {lpl_op} level {l + 1}")


def cases3():
    from srmg import gen3
    from srmg.tree3 import Tree3, populate, connectivity as connectivity3, BOX3
    t = Tree3((1, 1, 1), 3)
    populate(t, 3)
    # (order 4 needs a BoxStencil{3} connectivity)
    for name, stencil, op, lpl in (("box3_order2", BOX3, 0, None), ("box3_order4", BOX3, 2, "laplacian4")):
        conn = connectivity3(t, stencil)
        p = gen3.make_problem3(t, conn, lambda x, y, z: np.cos(3 * x) * y * (1 - z), (1.0 / 16) ** 2, op=op)
        yield name, t, conn, p, lpl


@pytest.mark.parametrize("case", list(cases3()), ids=lambda c: c[0])
def test_octree_vcycle_and_fmg_push_bit_identical(case):
    """The octrees whose sweeps do not push by rule (BoxStencil{3}, order 4) push from
    tables read off their fill; V-cycles and FMG equal the fill path's bit for bit."""
    import torch
    _, t, conn, p, lpl = case
    out, launches = {}, {}
    for push in (1, 0):
        ctx = mg.Context(0, D=3).set_tree(t, conn)
        for k, v in dict(op_graphs=0, op_sequencer=0, gs_push=push).items():
            ctx.set_option(k, v)
        b = torch.from_numpy(p.b).cuda()
        u, r, u1 = torch.zeros_like(b), torch.zeros_like(b), torch.zeros_like(b)
        torch.cuda.synchronize()
        l0 = ctx.launches()
        mg.vcycle_(ctx, u, b, r, u1, p.s, 0, p.bc, lpl, ndown=2, ntop=4, nup=2, ncycles=2)
        ctx.synchronize()
        launches[push] = ctx.launches() - l0
        v = u.cpu().numpy().copy()
        u.zero_()
        b.copy_(torch.from_numpy(p.b))
        mg.fmg_(ctx, u, b, r, u1, p.s, 0, p.bc, lpl, ndown=2, ntop=4, nup=2)
        ctx.synchronize()
        out[push] = (v, u.cpu().numpy().copy())
        ctx.close()
    for a, g, what in zip(out[1], out[0], ("vcycle", "fmg")):
        np.testing.assert_array_equal(_bits(a), _bits(g), err_msg=what)
    assert launches[1] < launches[0]
