"""Batched solves: a forest of independent problems (several trees; per tree the
Poisson potential and photoionization Helmholtz terms) in one persistent launch.

Every item of a batch must end exactly where a solo solve of the same problem ends:
same V-cycle count and bit-identical potential (the engine's per-block arithmetic and
per-item norms do not depend on the other items, and a converged item is frozen while
the others iterate).  A batch solves the coarsest level directly on level 1; a lone
tree's solve uses level 2 where it can (option "direct_level"), so the solo contexts
compared here are set to level 1.  The solo solves themselves are held to the oracle
by test_gpu_parity.py.
"""
import numpy as np
import pytest

from conftest import gpu_available
from srmg import gen, multigrid as mg

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]

OPTS = dict(tol=1e-8, ndown=2, ntop=4, nup=2, max_cycles=400)


def torch_cuda(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    torch.cuda.synchronize()
    return t


def to_np(t):
    return t.cpu().numpy()


def disc(p):
    return ("helmholtz", p.k2) if p.op == gen.OP_HELMHOLTZ else None


@pytest.fixture(scope="module")
def setup():
    """Three small channel trees (Poisson + 2 Helmholtz terms each) and a uniform
    level-4 tree with fewer levels: 10 items of uneven size and depth."""
    trees = gen.config3_tree_problems(seed=11, ntrees=3, lo=2e4, hi=8e4)
    items = []
    ctxs = []
    for pois, terms in trees:
        c = mg.Context(0).set_tree(pois.tree, pois.conn).set_option("direct_level", 1)
        ctxs.append(c)
        for p in [pois] + terms[:2]:
            items.append((c, p))
    uni = gen.make_problem(gen._uniform(4), lambda r, z, l, gi, gj: np.sin(r * 900) * np.cos(z * 700) * 1e19,
                           gen.poisson_scale(), name="uniform4")
    cu = mg.Context(0).set_tree(uni.tree, uni.conn).set_option("direct_level", 1)
    ctxs.append(cu)
    items.append((cu, uni))
    batch = mg.Batch([(c, p.s, disc(p), p.bc) for c, p in items], gen.GEOM_CYL1)
    return ctxs, items, batch


def solo(c, p, mode):
    ug = torch_cuda(np.zeros_like(p.b))
    st = mg.solve(c, ug, torch_cuda(p.b), p.s, p.geom, p.bc, disc(p), mode=mode, **OPTS)
    return to_np(ug), st


@pytest.mark.parametrize("mode", [mg.MODE_FP64, mg.MODE_MIXED])
def test_batch_equals_solo(setup, mode):
    _, items, batch = setup
    us = [torch_cuda(np.zeros_like(p.b)) for _, p in items]
    bs = [torch_cuda(p.b) for _, p in items]
    sts = batch.solve(us, bs, mode=mode, **OPTS)
    cycles = []
    for k, (c, p) in enumerate(items):
        u_solo, st_solo = solo(c, p, mode)
        assert sts[k]["status"] == 0
        assert sts[k]["rel_residual"] <= OPTS["tol"], (k, sts[k])
        assert sts[k]["cycles"] == st_solo["cycles"], (k, sts[k], st_solo)
        assert sts[k]["rel_residual"] == st_solo["rel_residual"], k
        np.testing.assert_array_equal(to_np(us[k]).view(np.uint64), u_solo.view(np.uint64), err_msg=f"item {k}")
        cycles.append(sts[k]["cycles"])
    # items stop at different cycle counts: the freezing path is exercised
    assert len(set(cycles)) > 1, cycles


def test_batch_host_entry_and_forest_layout(setup):
    _, items, batch = setup
    us = [torch_cuda(np.zeros_like(p.b)) for _, p in items]
    bs = [torch_cuda(p.b) for _, p in items]
    ref = batch.solve(us, bs, mode=mg.MODE_MIXED, **OPTS)
    # host arrays
    uh = [np.zeros_like(p.b) for _, p in items]
    bh = [np.ascontiguousarray(p.b) for _, p in items]
    sth = batch.solve(uh, bh, mode=mg.MODE_MIXED, **OPTS)
    # fields already in the forest layout
    uf = np.zeros((batch.total_blocks, 20, 20))
    bf = np.zeros_like(uf)
    for k, (_, p) in enumerate(items):
        o = batch.offsets[k]
        bf[o:o + batch.nblks[k]] = p.b[:batch.nblks[k]]
    ufg, bfg = torch_cuda(uf), torch_cuda(bf)
    stf = batch.solve_forest(ufg, bfg, mode=mg.MODE_MIXED, **OPTS)
    ufn = to_np(ufg)
    for k in range(len(items)):
        u_dev = to_np(us[k])
        np.testing.assert_array_equal(uh[k].view(np.uint64), u_dev.view(np.uint64))
        o = batch.offsets[k]
        np.testing.assert_array_equal(ufn[o:o + batch.nblks[k]].view(np.uint64),
                                      u_dev[:batch.nblks[k]].view(np.uint64))
        assert sth[k]["cycles"] == ref[k]["cycles"] == stf[k]["cycles"]


@pytest.mark.parametrize("mode", [mg.MODE_FP64, mg.MODE_MIXED])
def test_batch_graph_replay(setup, mode):
    """The captured CUDA graph replays the same solve: identical results on every call,
    with fresh inputs copied into the same buffers between calls."""
    _, items, batch = setup
    us = [torch_cuda(np.zeros_like(p.b)) for _, p in items]
    bs = [torch_cuda(p.b) for _, p in items]
    ref = batch.solve(us, bs, mode=mode, **OPTS)
    ref_u = [to_np(u) for u in us]
    batch.set_option("graph", 1)
    try:
        for call in range(3):
            for u in us:
                u.zero_()
            import torch
            torch.cuda.synchronize()
            st = batch.solve(us, bs, mode=mode, **OPTS)
            for k in range(len(items)):
                assert st[k]["cycles"] == ref[k]["cycles"], (call, k)
                np.testing.assert_array_equal(to_np(us[k]).view(np.uint64), ref_u[k].view(np.uint64))
    finally:
        batch.set_option("graph", 0)


def test_batch_rejects_bad_items(setup):
    ctxs, items, _ = setup
    c, p = items[0]
    with pytest.raises(mg.SrmgError):
        mg.Batch([(c, p.s, ("helmholtz", 1.0), np.full(9, 3))], gen.GEOM_CYL1)
    empty = mg.Context(0)
    with pytest.raises(mg.SrmgError):
        mg.Batch([(empty, p.s, None, p.bc)], gen.GEOM_CYL1)


def test_autotune_single_and_batch(setup):
    """The autotuner times every candidate to the tolerance (6 launch shapes, then 15
    sweep-count and relaxation-factor pairs at the fastest shape, then for mixed solves
    4 inner-cycle counts at the fastest pair), restores the caller's initial guess, and
    leaves the fastest launch shape, sweep counts, omega and inner cycles in force; an
    FP64-direct tuning has no inner-cycle stage."""
    ctxs, items, batch = setup
    c, p = items[0]
    u0 = np.zeros_like(p.b)
    ug, bg = torch_cuda(u0), torch_cuda(p.b)
    chosen, trials = mg.autotune(c, ug, bg, p.s, p.geom, p.bc, disc(p), tol=1e-8, mode=mg.MODE_MIXED)
    assert len(trials) == 25
    assert all(t["ms"] > 0 for t in trials)
    assert {t["omega"] for t in trials[6:21]} == {1.0, 1.1, 1.2}
    assert [t["inner_cycles"] for t in trials[21:]] == [1, 2, 3, 4]
    best = min(trials, key=lambda t: t["ms"])
    assert (chosen["ndown"], chosen["nup"], chosen["omega"], chosen["inner_cycles"]) == \
        (best["ndown"], best["nup"], best["omega"], best["inner_cycles"])
    np.testing.assert_array_equal(to_np(ug), u0)  # initial guess restored
    st = mg.solve(c, ug, bg, p.s, p.geom, p.bc, disc(p), tol=1e-8, mode=mg.MODE_MIXED,
                  ndown=chosen["ndown"], nup=chosen["nup"], ntop=chosen["ntop"], omega=chosen["omega"],
                  inner_cycles=chosen["inner_cycles"])
    assert st["rel_residual"] <= 1e-8
    c.set_option("engine_ctas", 0).set_option("local_max_blocks", 4)
    _, trials_d = mg.autotune(c, ug, bg, p.s, p.geom, p.bc, disc(p), tol=1e-8, mode=mg.MODE_FP64_DIRECT)
    assert len(trials_d) == 21
    c.set_option("engine_ctas", 0).set_option("local_max_blocks", 4)
    us = [torch_cuda(np.zeros_like(q.b)) for _, q in items]
    bs = [torch_cuda(q.b) for _, q in items]
    chosen, trials = mg.batch_autotune(batch, us, bs, tol=1e-8, mode=mg.MODE_MIXED)
    assert len(trials) == 25 and all(t["ms"] > 0 for t in trials)
    sts = batch.solve(us, bs, mode=mg.MODE_MIXED, tol=1e-8, ndown=chosen["ndown"], nup=chosen["nup"],
                      ntop=chosen["ntop"], omega=chosen["omega"], inner_cycles=chosen["inner_cycles"],
                      max_cycles=400)
    assert all(s["rel_residual"] <= 1e-8 for s in sts)
    batch.set_option("engine_ctas", 0).set_option("local_max_blocks", 4)


@pytest.mark.parametrize("mode", [mg.MODE_FP64, mg.MODE_MIXED])
def test_launch_shape_independent(setup, mode):
    """The persistent kernel runs with 768 or 1024 threads per CTA (option
    "engine_threads"; by default chosen from the tree size): solo and batched results,
    cycle counts and norms are bit-identical in both shapes."""
    _, items, batch = setup
    c, p = items[0]
    out = {}
    for nt in (768, 1024):
        c.set_option("engine_threads", nt)
        batch.set_option("engine_threads", nt)
        u_solo, st_solo = solo(c, p, mode)
        us = [torch_cuda(np.zeros_like(q.b)) for _, q in items]
        sts = batch.solve(us, [torch_cuda(q.b) for _, q in items], mode=mode, **OPTS)
        out[nt] = (u_solo, st_solo, [to_np(u) for u in us], sts)
    c.set_option("engine_threads", 0)
    batch.set_option("engine_threads", 0)
    a, b = out[768], out[1024]
    np.testing.assert_array_equal(a[0].view(np.uint64), b[0].view(np.uint64))
    assert a[1]["cycles"] == b[1]["cycles"] and a[1]["rel_residual"] == b[1]["rel_residual"]
    for k in range(len(items)):
        np.testing.assert_array_equal(a[2][k].view(np.uint64), b[2][k].view(np.uint64))
        assert a[3][k]["cycles"] == b[3][k]["cycles"]
        assert a[3][k]["rel_residual"] == b[3][k]["rel_residual"]
