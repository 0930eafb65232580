"""The warm-start network's inference forward on the tcgen05 tensor cores against the
mma.sync forward and the CPU oracle (oracle/cnn_oracle.py): one sample, several
samples per CTA, and the guarded tree prediction with either forward."""
import numpy as np
import pytest

from conftest import gpu_available
import cnn_oracle as co
from srmg import gen, multigrid as mg

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def inputs(n, seed):
    import torch
    rng = np.random.default_rng(seed)
    x = co.bf16_round(rng.standard_normal((n, 400, 2)).astype(np.float32)).astype(np.float32)
    xt = torch.from_numpy(x).to(torch.bfloat16).cuda()
    torch.cuda.synchronize()
    return x, xt


@pytest.fixture(scope="module")
def net():
    return mg.Cnn(0, seed=7)


@pytest.mark.parametrize("n", [1, 300])
def test_tcgen05_forward_matches_mma_sync_and_oracle(net, n):
    x, xt = inputs(n, 10 + n)
    y_tc = net.forward_tc(xt).cpu().numpy()
    y_ref = net.forward(xt).cpu().numpy()
    assert np.all(np.isfinite(y_tc))
    assert rel(y_tc, y_ref) < 2e-3, rel(y_tc, y_ref)
    yo, _ = co.forward(x, net.get_params().astype(np.float64))
    assert rel(y_tc, yo) < 2e-3, rel(y_tc, yo)


def test_tcgen05_repeated_calls_agree(net):
    x, xt = inputs(200, 3)
    a = net.forward_tc(xt).cpu().numpy()
    b = net.forward_tc(xt).cpu().numpy()
    np.testing.assert_array_equal(a, b)


def test_predict_with_tcgen05(net):
    import torch
    p = gen.config1()
    ctx = mg.Context(0).set_tree(p.tree, p.conn)
    b2 = torch.from_numpy(p.b).cuda()
    b1 = (b2 * 1.01).contiguous()
    b = (b2 * 1.025).contiguous()
    phi2, phi1 = torch.zeros_like(b2), torch.zeros_like(b2)
    mg.solve(ctx, phi2, b2, p.s, p.geom, p.bc, tol=1e-10, mode=mg.MODE_FP64)
    mg.solve(ctx, phi1, b1, p.s, p.geom, p.bc, tol=1e-10, mode=mg.MODE_FP64)
    u_a = phi1.clone()
    w_a, r_a = mg.cnn_predict(ctx, net, u_a, b, b1, phi2, b2, p.s, p.geom, p.bc, resid=True)
    net.use_tcgen05(True)
    try:
        u_b = phi1.clone()
        w_b, r_b = mg.cnn_predict(ctx, net, u_b, b, b1, phi2, b2, p.s, p.geom, p.bc, resid=True)
        net.check(mg.lib().srmg_cnn_tc_status(net.handle))
    finally:
        net.use_tcgen05(False)
    assert r_a[0] == r_b[0] and r_a[1] == r_b[1]       # previous potential, extrapolation
    assert abs(r_a[2] - r_b[2]) <= 1e-3 * r_a[2]       # learned candidate
