"""srmg_solve_async / srmg_solve_wait: the host-array solve split at its host
synchronisation, so that independent problems' copies overlap each other's solves.

Its result and statistics must equal srmg_solve's bit for bit (the same launch on the
same data), also with two contexts of one tree in flight at once on page-locked host
arrays; a context with a solve in flight takes no other call until it is waited for.
"""
import numpy as np
import pytest

from conftest import gpu_available
from srmg import gen, multigrid as mg

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]


@pytest.fixture(scope="module")
def prob():
    return gen.config2(seed=3, target_leaf=60_000, extra=3)


def _register(ctx, arrays):
    for a in arrays:
        ctx.check(mg.lib().srmg_host_register(ctx.handle, a.ctypes.data, a.nbytes))


def _unregister(ctx, arrays):
    for a in arrays:
        ctx.check(mg.lib().srmg_host_unregister(ctx.handle, a.ctypes.data))


@pytest.mark.parametrize("mode", [mg.MODE_MIXED, mg.MODE_FP64, mg.MODE_FP64_DIRECT])
def test_async_equals_sync(prob, mode):
    p = prob
    kw = dict(tol=1e-8, mode=mode, ndown=1, nup=1, ntop=4, omega=1.1, inner_cycles=3)
    ctx = mg.Context(0).set_tree(p.tree, p.conn)
    us = np.zeros_like(p.b)
    st_sync = mg.solve(ctx, us, p.b.copy(), p.s, p.geom, p.bc, **kw)
    ua, ba = np.zeros_like(p.b), p.b.copy()
    _register(ctx, (ua, ba))
    mg.solve_async(ctx, ua, ba, p.s, p.geom, p.bc, **kw)
    st = mg.solve_wait(ctx)
    _unregister(ctx, (ua, ba))
    assert np.array_equal(ua.view(np.uint64), us.view(np.uint64))
    for k in ("cycles", "outer", "rel_residual", "bnorm"):
        assert st[k] == st_sync[k], k
    assert st["rel_residual"] <= 1e-8
    ctx.close()


def test_two_contexts_in_flight(prob):
    """Two contexts on one tree alternate over four right-hand sides, two solves in
    flight at a time; every result equals its synchronous solve."""
    p = prob
    kw = dict(tol=1e-8, mode=mg.MODE_MIXED, ndown=1, nup=1, ntop=4, omega=1.1, inner_cycles=3)
    rng = np.random.default_rng(7)
    rhs = [p.b * (1.0 + 0.1 * k) + rng.standard_normal(p.b.shape) * np.abs(p.b).max() * 1e-3 for k in range(4)]
    ref_ctx = mg.Context(0).set_tree(p.tree, p.conn)
    want = []
    for b in rhs:
        u = np.zeros_like(p.b)
        mg.solve(ref_ctx, u, b.copy(), p.s, p.geom, p.bc, **kw)
        want.append(u)
    ref_ctx.close()
    ctxs = [mg.Context(0).set_tree(p.tree, p.conn) for _ in range(2)]
    us = [np.zeros_like(p.b) for _ in rhs]
    bs = [b.copy() for b in rhs]
    _register(ctxs[0], us + bs)  # page-locking is per process, not per context
    for k in range(len(rhs)):
        c = ctxs[k % 2]
        if k >= 2:
            assert mg.solve_wait(c)["rel_residual"] <= 1e-8
        mg.solve_async(c, us[k], bs[k], p.s, p.geom, p.bc, **kw)
    for c in ctxs:
        assert mg.solve_wait(c)["rel_residual"] <= 1e-8
    for k in range(len(rhs)):
        assert np.array_equal(us[k].view(np.uint64), want[k].view(np.uint64)), k
    _unregister(ctxs[0], us + bs)
    for c in ctxs:
        c.close()


def test_context_busy_until_waited(prob):
    p = prob
    ctx = mg.Context(0).set_tree(p.tree, p.conn)
    u, b = np.zeros_like(p.b), p.b.copy()
    with pytest.raises(mg.SrmgError):
        mg.solve_wait(ctx)  # nothing in flight
    mg.solve_async(ctx, u, b, p.s, p.geom, p.bc, tol=1e-8, mode=mg.MODE_MIXED)
    with pytest.raises(mg.SrmgError):
        mg.solve(ctx, np.zeros_like(p.b), p.b.copy(), p.s, p.geom, p.bc, tol=1e-8)
    with pytest.raises(mg.SrmgError):
        ctx.set_option("engine", 1)
    st = mg.solve_wait(ctx)
    assert st["rel_residual"] <= 1e-8
    # usable again
    st2 = mg.solve(ctx, np.zeros_like(p.b), p.b.copy(), p.s, p.geom, p.bc, tol=1e-8, mode=mg.MODE_MIXED)
    assert st2["rel_residual"] <= 1e-8
    ctx.close()
