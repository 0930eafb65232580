"""Stage preparation and post-processing on the device against the oracle, through the
C ABI: netcharge! (src/streamer.jl:369-373), restrict_full! (src/restrict.jl:43-47) and
electric_field! (src/multigrid.jl:421-449).  All three are bit-exact: the net charge
and restriction are fixed-order sums, the field uses IEEE division and square root
with no fused multiply-add on either side."""
import numpy as np
import pytest

from conftest import gpu_available
from oracle import OracleTree, lib as olib, _ptr
from srmg import gen, multigrid as mg

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]


def torch_cuda(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    torch.cuda.synchronize()
    return t


def bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


@pytest.fixture(scope="module")
def setup():
    p = gen.config2(seed=5, target_leaf=40_000, extra=3)
    ctx = mg.Context(0).set_tree(p.tree, p.conn)
    ot = OracleTree(p.tree, p.conn, p.nblk)
    return p, ctx, ot


def test_netcharge_bit_exact(setup):
    p, ctx, ot = setup
    rng = np.random.default_rng(1)
    ne = rng.lognormal(40, 3, (p.nblk, 20, 20))
    ni = ne * rng.uniform(0.5, 1.5, ne.shape)
    q0 = rng.standard_normal(ne.shape)  # ghosts keep their values
    qo = q0.copy()
    olib().orc_netcharge(_ptr(qo), _ptr(ne), _ptr(ni), ot.ref)
    qg = torch_cuda(q0)
    mg.netcharge(ctx, qg, torch_cuda(ne), torch_cuda(ni))
    ctx.synchronize()
    assert np.array_equal(bits(qg.cpu().numpy()), bits(qo))
    qh = q0.copy()
    mg.netcharge(ctx, qh, ne, ni)
    assert np.array_equal(bits(qh), bits(qo))


def test_restrict_full_bit_exact(setup):
    p, ctx, ot = setup
    u = np.random.default_rng(2).standard_normal((p.nblk, 20, 20))
    uo = u.copy()
    olib().orc_restrict_full(_ptr(uo), ot.ref)
    ug = torch_cuda(u)
    mg.restrict_full_(ctx, ug)
    ctx.synchronize()
    assert np.array_equal(bits(ug.cpu().numpy()), bits(uo))


@pytest.mark.parametrize("seed", [3, 4])
def test_electric_field_bit_exact(setup, seed):
    p, ctx, ot = setup
    rng = np.random.default_rng(seed)
    u = rng.standard_normal((p.nblk, 20, 20)) * 1e3
    e0 = np.array([rng.uniform(-1e3, 1e3), 1.5e6])
    h = p.h1
    e_init = rng.standard_normal((p.nblk, 2, 21, 21))  # entries outside the valid faces keep their values
    eo, abso = e_init.copy(), np.zeros((p.nblk, 20, 20))
    olib().orc_electric_field(_ptr(eo), _ptr(abso), _ptr(u), h, _ptr(e0), ot.ref)
    eg, absg = torch_cuda(e_init), torch_cuda(np.zeros((p.nblk, 20, 20)))
    mg.electric_field(ctx, eg, absg, torch_cuda(u), h, e0)
    ctx.synchronize()
    assert np.array_equal(bits(eg.cpu().numpy()), bits(eo))
    assert np.array_equal(bits(absg.cpu().numpy()), bits(abso))
    eh, absh = e_init.copy(), np.zeros((p.nblk, 20, 20))
    mg.electric_field(ctx, eh, absh, u, h, e0)
    assert np.array_equal(bits(eh), bits(eo))
    assert np.array_equal(bits(absh), bits(abso))


def test_stage_rejects_bad_arguments(setup):
    p, ctx, _ = setup
    import torch
    u = torch.zeros((p.nblk, 20, 20), dtype=torch.float64, device="cuda")
    e = torch.zeros((p.nblk, 2, 21, 21), dtype=torch.float64, device="cuda")
    with pytest.raises(mg.SrmgError):
        mg.electric_field(ctx, e, u.clone(), u, 0.0, (0.0, 0.0))
    small = torch.zeros((1, 20, 20), dtype=torch.float64, device="cuda")
    with pytest.raises(mg.SrmgError):
        mg.netcharge(ctx, small, small, small)
