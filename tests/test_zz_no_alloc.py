"""srmg_resnorm_noalloc: the residual norm for callers that cannot allocate.

Some callers cannot call cudaMalloc when they need a residual norm: hosts whose
device memory belongs to their own pool allocator, loops that cannot afford an
allocation's implicit synchronisation.  The
allocation-free entry point keeps its per-block partial sums in a static device
array instead.  This test calls it through the C ABI, twice in a row, and checks each
result against the existing srmg_resnorm_dev within the same tolerance the resnorm
parity test uses; it also checks that the two calls leave free device memory
unchanged and that a tree above the array's limit is rejected.

The file is named so that pytest collects it after every other test.
"""
import ctypes

import numpy as np
import pytest

from conftest import gpu_available
from srmg import gen, multigrid as mg

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]

REL_TOL = 1e-10   # as in test_gpu_parity.test_resnorm_matches_oracle


def _prepared():
    import torch
    p = gen.config2(seed=5, target_leaf=40_000, extra=3)
    ctx = mg.Context(0).set_tree(p.tree, p.conn)
    b = torch.from_numpy(p.b.copy()).cuda()
    u = torch.zeros_like(b)
    r, u1 = torch.zeros_like(b), torch.zeros_like(b)
    # one V-cycle so that the residual is a non-trivial field
    mg.vcycle_(ctx, u, b.clone(), r, u1, p.s, p.geom, p.bc, ndown=2, ntop=4, nup=2)
    ctx.synchronize()
    return p, ctx, u, b


def _noalloc(ctx, p, u, b, out):
    ctx.check(mg.lib().srmg_resnorm_noalloc(ctx.handle, b.data_ptr(), u.data_ptr(), p.nblk, p.s,
                                            p.op, p.k2, p.geom, out.data_ptr()))
    ctx.synchronize()
    return float(out.item())


def test_noalloc_resnorm_matches_resnorm_dev_twice():
    import torch
    p, ctx, u, b = _prepared()
    want = mg.resnorm(ctx, None, b, u, p.s, p.geom, p.bc)
    assert want > 0
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    first = _noalloc(ctx, p, u, b, out)           # first call on the device: set-up
    free_before = torch.cuda.mem_get_info()[0]
    second = _noalloc(ctx, p, u, b, out)
    third = _noalloc(ctx, p, u, b, out)
    free_after = torch.cuda.mem_get_info()[0]
    for got in (first, second, third):
        assert abs(got - want) <= REL_TOL * want, (got, want)
    assert second == third                        # deterministic fixed-order reduction
    assert free_after == free_before              # the calls allocated nothing
    ctx.close()


def test_noalloc_rejects_trees_above_the_limit():
    import torch
    tree = gen._uniform(9)                        # 87381 blocks > 65536
    p = gen.make_problem(tree, lambda r, z, l, gi, gj: np.ones_like(r), 1.0)
    ctx = mg.Context(0).set_tree(p.tree, p.conn)
    b = torch.zeros((p.nblk, 20, 20), dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = mg.lib().srmg_resnorm_noalloc(ctx.handle, b.data_ptr(), b.data_ptr(), p.nblk, 1.0, 0, 0.0,
                                       1, out.data_ptr())
    assert rc == -1
    assert b"65536" in mg.lib().srmg_last_error(ctx.handle)
    ctx.close()


def test_noalloc_refuses_three_dimensional_trees():
    import torch
    from srmg.tree3 import Tree3, populate, connectivity as connectivity3
    t = Tree3((1, 1, 1), 2)
    populate(t, 2)
    ctx = mg.Context(0, D=3).set_tree(t, connectivity3(t))
    n = t.nblocks_created
    f = torch.zeros((n, 20, 20, 20), dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = mg.lib().srmg_resnorm_noalloc(ctx.handle, f.data_ptr(), f.data_ptr(), n, 1.0, 0, 0.0, 0, out.data_ptr())
    assert rc == mg.SRMG_ERR_UNSUPPORTED
    ctx.close()
