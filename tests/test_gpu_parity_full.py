"""GPU-vs-oracle parity at the benchmark sizes, through the C ABI.

The refined channel tree of the benchmark (seed 2, ~1.5M leaf cells, 7829 blocks, 9
levels) and the full-size multi-branched tree (51877 blocks, 11 levels) are compared
with the oracle (the CPU FP64 restatement of src/multigrid.jl:60-106 and the routines it
calls) on the same tree and right-hand side:
  * 1 and 3 FP64 V-cycles (persistent engine): bit-exact, u on every element (ghosts
    included), b (the FAS right-hand sides) on the valid cells;
  * the tolerance-driven FP64 solve to 1e-8: the oracle's cycle count (+-1: the norms
    are summed in another order) and, with the same count, its iterate bit for bit;
  * the mixed-precision solve: its error against the oracle's FP64 solution to 1e-11.
"""
import numpy as np
import pytest

from conftest import gpu_available
from oracle import Oracle
from srmg import gen, multigrid as mg
from srmg.timestep import leaf_mask

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]

MIXED_VS_ORACLE = 1e-7   # mixed solve to 1e-8 against the oracle's FP64 solution to 1e-11


def cuda(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    torch.cuda.synchronize()
    return t


def rel_l2(a, b, mask=None):
    if mask is not None:
        a, b = a[mask], b[mask]
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def valid_mask(shape):
    m = np.zeros(shape, dtype=bool)
    m[:, 2:18, 2:18] = True
    return m


@pytest.fixture(scope="module")
def config2():
    p = gen.config2(seed=2, target_leaf=1_500_000)
    assert p.tree.nblocks() == 7829 and p.tree.finest_level() == 9
    return p, mg.Context(0).set_tree(p.tree, p.conn), Oracle(p)


@pytest.fixture(scope="module")
def config5():
    p = gen.config5()
    assert p.tree.nblocks() > 50_000
    return p, mg.Context(0).set_tree(p.tree, p.conn), Oracle(p)


def _vcycles(p, ctx, orc, ncycles):
    u = np.zeros_like(p.b)
    orc.fill_ghost_all(u)
    b = p.b.copy()
    ug, bg = cuda(u), cuda(b)
    rg, u1g = cuda(np.zeros_like(u)), cuda(np.zeros_like(u))
    mg.vcycle_(ctx, ug, bg, rg, u1g, p.s, p.geom, p.bc, ndown=2, ntop=4, nup=2, ncycles=ncycles)
    ctx.synchronize()
    r, u1 = np.zeros_like(u), np.zeros_like(u)
    for _ in range(ncycles):
        orc.vcycle(u, b, r, u1, ndown=2, ntop=4, nup=2)
    got, gb = ug.cpu().numpy(), bg.cpu().numpy()
    vm = valid_mask(u.shape)
    assert np.array_equal(got.view(np.uint64), u.view(np.uint64)), \
        f"{int((got.view(np.uint64) != u.view(np.uint64)).sum())} elements of u differ"
    assert np.array_equal(gb.view(np.uint64)[vm], b.view(np.uint64)[vm])  # FAS right-hand sides


@pytest.mark.parametrize("ncycles", [1, 3])
def test_config2_vcycles_match_oracle(config2, ncycles):
    _vcycles(*config2, ncycles)


def test_config5_vcycle_matches_oracle(config5):
    _vcycles(*config5, 1)


def test_config2_fp64_solve_matches_oracle(config2):
    """The FP64 solve to 1e-8 from a zero guess: the oracle's cycle count and iterate."""
    p, ctx, orc = config2
    ug = cuda(np.zeros_like(p.b))
    st = mg.solve(ctx, ug, cuda(p.b), p.s, p.geom, p.bc, tol=1e-8, mode=mg.MODE_FP64, max_cycles=2000)
    uo = np.zeros_like(p.b)
    c, rel = orc.solve(uo, p.b.copy(), 1e-8, max_cycles=2000)
    assert st["rel_residual"] <= 1e-8 and rel <= 1e-8
    assert abs(st["cycles"] - c) <= 1, (st["cycles"], c)
    if st["cycles"] == c:
        leaf = leaf_mask(p.tree, p.nblk)
        assert np.array_equal(ug.cpu().numpy()[leaf], uo[leaf])


def test_config2_mixed_solve_error_vs_oracle(config2):
    """The mixed-precision solve to 1e-8 against the oracle's FP64 solution to 1e-11."""
    p, ctx, orc = config2
    ug = cuda(np.zeros_like(p.b))
    st = mg.solve(ctx, ug, cuda(p.b), p.s, p.geom, p.bc, tol=1e-8, mode=mg.MODE_MIXED, max_cycles=200)
    assert st["rel_residual"] <= 1e-8
    uo = np.zeros_like(p.b)
    c, rel = orc.solve(uo, p.b.copy(), 1e-11, max_cycles=5000)
    assert rel <= 1e-11
    leaf = leaf_mask(p.tree, p.nblk)
    err = rel_l2(ug.cpu().numpy(), uo, leaf)
    assert err <= MIXED_VS_ORACLE, err
