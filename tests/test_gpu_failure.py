"""Failure detection on the GPU without a fault: a persistent kernel whose grid barrier
cannot complete (one CTA never arrives) gives up after its bounded wait, records the
timeout in the context's error word and returns; the host reads SRMG_ERR_TIMEOUT and
the same context then solves normally."""
import numpy as np
import pytest

from conftest import gpu_available
from srmg import gen, multigrid as mg

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]


def test_barrier_timeout_is_reported_and_the_context_recovers():
    import time
    import torch
    p = gen.config2(seed=5, target_leaf=40_000, extra=3)
    ctx = mg.Context(0).set_tree(p.tree, p.conn)
    t0 = time.perf_counter()
    rc = mg.lib().srmg_selftest_barrier_timeout(ctx.handle, 20)
    dt = time.perf_counter() - t0
    assert rc == mg.SRMG_ERR_TIMEOUT
    assert dt < 5.0  # the wait ended by itself, after about its 20 ms limit
    assert mg.lib().srmg_selftest_barrier_timeout(ctx.handle, 0) == mg.SRMG_ERR_BADARG
    # the context is usable afterwards: a mixed solve reaches its tolerance
    u = torch.zeros((p.nblk, 20, 20), dtype=torch.float64, device="cuda")
    b = torch.from_numpy(p.b).cuda()
    st = mg.solve(ctx, u, b, p.s, p.geom, p.bc, tol=1e-8, mode=mg.MODE_MIXED)
    assert st["rel_residual"] <= 1e-8
    assert np.isfinite(u.cpu().numpy()).all()
    ctx.close()
