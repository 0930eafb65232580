"""The learned warm-start network's CUDA kernels against the CPU oracle
(oracle/cnn_oracle.py): forward outputs, the loss and every layer's weight and bias
gradient; training lowers the loss; the tree path packs samples the way the oracle
defines them and keeps a guess only when it lowers the residual."""
import numpy as np
import pytest

from conftest import gpu_available
import cnn_oracle as co
from srmg import gen, multigrid as mg

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def batch(n, seed):
    import torch
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, 400, 2)).astype(np.float32)
    x = co.bf16_round(x).astype(np.float32)
    t = (0.3 * rng.standard_normal((n, 256))).astype(np.float32)
    xt = torch.from_numpy(x).to(torch.bfloat16).cuda()
    tt = torch.from_numpy(t).cuda()
    torch.cuda.synchronize()
    return x, t, xt, tt


@pytest.fixture(scope="module")
def net():
    return mg.Cnn(0, seed=7)


def test_forward_matches_oracle(net):
    theta = net.get_params().astype(np.float64)
    x, t, xt, tt = batch(37, 1)
    y = net.forward(xt).cpu().numpy()
    yo, _ = co.forward(x, theta)
    assert rel(y, yo) < 2e-3, rel(y, yo)


def test_gradients_match_oracle(net):
    theta = net.get_params().astype(np.float64)
    x, t, xt, tt = batch(23, 2)
    loss, g = net.gradients(xt, tt)
    lo, go = co.gradients(x, t, theta)
    assert abs(loss - lo) <= 2e-3 * abs(lo)
    for l, ((w0, w1), (b0, b1)) in enumerate(co.layer_slices()):
        assert rel(g[w0:w1], go[w0:w1]) < 1e-2, (l, "W", rel(g[w0:w1], go[w0:w1]))
        assert rel(g[b0:b1], go[b0:b1]) < 1e-2, (l, "b", rel(g[b0:b1], go[b0:b1]))


def test_residual_loss_gradients_match_oracle(net):
    import torch
    theta = net.get_params().astype(np.float64)
    x, t, xt, tt = batch(19, 4)
    ir0 = np.arange(19, dtype=np.int32) * 16
    ir0t = torch.from_numpy(ir0).cuda()
    torch.cuda.synchronize()
    loss, g = net.gradients(xt, tt, ir0t, lam=0.5, geom=1)
    lo, go = co.gradients(x, t, theta, ir0=ir0, lam=0.5, geom=1)
    assert abs(loss - lo) <= 2e-3 * abs(lo)
    assert rel(g, go) < 1e-2, rel(g, go)


def test_training_lowers_loss():
    n = mg.Cnn(0, seed=3)
    x, t, xt, tt = batch(64, 3)
    # a learnable target: a smooth function of the inputs' centre
    import torch
    tgt = 0.5 * xt[:, :, 0].float().reshape(64, 20, 20)[:, 2:18, 2:18].reshape(64, 256).contiguous()
    torch.cuda.synchronize()
    l0 = n.train_step(xt, tgt, 1e-3)
    for _ in range(150):
        l = n.train_step(xt, tgt, 1e-3)
    n.synchronize()
    assert l < 0.3 * l0, (l0, l)


def test_set_get_params_roundtrip(net):
    theta = net.get_params()
    net.set_params(theta * 0.5)
    np.testing.assert_array_equal(net.get_params(), (theta * 0.5).astype(np.float32))
    net.set_params(theta)


def test_tree_pack_and_guarded_predict(net):
    """Samples of a tree match their definition; the guarded prediction never keeps a
    guess whose residual is above the previous potential's."""
    import torch
    p = gen.config1()
    ctx = mg.Context(0).set_tree(p.tree, p.conn)
    b2 = torch.from_numpy(p.b).cuda()
    b1 = (b2 * 1.01).contiguous()
    b = (b2 * 1.02).contiguous()  # a linear change: g = 0
    phi2 = torch.zeros_like(b2)
    phi1 = torch.zeros_like(b2)
    mg.solve(ctx, phi2, b2, p.s, p.geom, p.bc, tol=1e-10, mode=mg.MODE_FP64)
    mg.solve(ctx, phi1, b1, p.s, p.geom, p.bc, tol=1e-10, mode=mg.MODE_FP64)
    f = (phi1 - phi2).contiguous()
    g = (b - 2 * b1 + b2).contiguous()
    x, scale, blk = mg.cnn_pack(ctx, f, g, p.s, p.geom, p.bc)
    assert x.shape[0] == 256  # the level-5 leaves of the uniform tree
    fh = f.cpu().numpy()
    k = 17
    bk = int(blk[k])
    xs = x[k].float().cpu().numpy().reshape(20, 20, 2)
    ratio = xs[8:12, 8:12, 0] / fh[bk, 8:12, 8:12]
    assert np.allclose(ratio, ratio.flat[0], rtol=1e-2)
    u = phi1.clone()
    rn = lambda v: mg.resnorm(ctx, None, b, v, p.s, p.geom, p.bc)
    r_prev = rn(phi1)
    which = mg.cnn_predict(ctx, mg.Cnn(0, seed=11), u, b, b1, phi2, b2, p.s, p.geom, p.bc)
    assert which in (0, 1, 2)
    assert rn(u) <= r_prev
    # a linear change of b: the extrapolation is exact up to the solve tolerance
    assert which in (1, 2) and rn(u) < 1e-3 * r_prev


def test_predict_matches_separate_path(net):
    """The library's guarded prediction forms the learned candidate exactly as the
    separate pack -> forward -> scatter path does (residual norms agree)."""
    import torch
    p = gen.config1()
    ctx = mg.Context(0).set_tree(p.tree, p.conn)
    b2 = torch.from_numpy(p.b).cuda()
    b1 = (b2 * 1.01).contiguous()
    b = (b2 * 1.025).contiguous()
    phi2, phi1 = torch.zeros_like(b2), torch.zeros_like(b2)
    mg.solve(ctx, phi2, b2, p.s, p.geom, p.bc, tol=1e-10, mode=mg.MODE_FP64)
    mg.solve(ctx, phi1, b1, p.s, p.geom, p.bc, tol=1e-10, mode=mg.MODE_FP64)
    u = phi1.clone()
    which, r3 = mg.cnn_predict(ctx, net, u, b, b1, phi2, b2, p.s, p.geom, p.bc, resid=True)
    assert all(np.isfinite(r3))
    f = (phi1 - phi2).contiguous()
    g = (b - 2 * b1 + b2).contiguous()
    x, scale, blk = mg.cnn_pack(ctx, f, g, p.s, p.geom, p.bc)
    y = net.forward(x)
    lrn = (phi1 + f).contiguous()
    lrn[blk.long(), 2:18, 2:18] += (y.double() * scale[:, None]).reshape(-1, 16, 16)
    torch.cuda.synchronize()
    for l in range(len(p.tree), 1, -1):
        ctx.check(mg.lib().srmg_restrict_level_dev(ctx.handle, lrn.data_ptr(), p.nblk, l))
    for l in range(1, len(p.tree) + 1):
        mg.fill_ghost_(ctx, lrn, l, p.bc)
    ctx.synchronize()
    r_sep = mg.resnorm(ctx, None, b, lrn, p.s, p.geom, p.bc)
    assert abs(r_sep - r3[2]) <= 1e-9 * r3[2]
    assert abs(mg.resnorm(ctx, None, b, u, p.s, p.geom, p.bc) - min(r3)) <= 1e-9 * min(r3)


def test_trained_network_saves_cycles():
    """Trained on solver-generated pairs of seeded streamer runs, the learned guess
    lowers the initial residual below the time extrapolation's and needs fewer
    V-cycles to 1e-8 than the previous-step guess, on a held-out run."""
    from srmg import learn
    pairs = learn.generate(runs=2, steps=500, seed=3)
    net = mg.Cnn(0, seed=5)
    learn.train(net, pairs, steps=800, batch=4, lr=1e-3, mu=0.001)
    ev = learn.evaluate(net, runs=1, steps=400, every=40, seed=71)
    assert ev["learned"]["median_initial_rel"] < 0.5 * ev["extrapolated"]["median_initial_rel"], ev
    assert ev["learned"]["mean_cycles"] < ev["prev"]["mean_cycles"] - 1.0, ev
    assert ev["learned"]["mean_cycles"] <= ev["extrapolated"]["mean_cycles"], ev
