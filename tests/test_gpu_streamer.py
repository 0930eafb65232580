"""Parity of libsrmg's streamer-transport kernels (called through the C ABI) with the
oracle: flux! (Koren) + restrict_flux! and the per-block stable time steps bit-exact,
chemderivs! + fluxderivs! to rounding (the chemistry calls exp), the InterpCopy ghost
fill and the SSPRK3 combinations bit-exact, and one whole SSPRK3 step (three stages with
their Poisson solves) against the oracle's composition of the same step.  Uniform
(config-1) and refined trees; cylindrical and Cartesian geometry."""
import ctypes

import numpy as np
import pytest

from conftest import gpu_available
from oracle import Oracle, lib as olib, _ptr
import streamer_oracle as so
from srmg import gen, multigrid as mg
from srmg.streamer import MINIMAL, Streamer, E_BACKGROUND

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]

REL_RATES = 1e-13  # chemistry through exp(): last-bit differences only


def cuda(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    torch.cuda.synchronize()
    return t


PROBS = {"uniform": gen.config1(), "refined": gen.config2(seed=5, target_leaf=40_000, extra=3)}


@pytest.fixture(scope="module", params=list(PROBS))
def case(request):
    p = PROBS[request.param]
    return p, mg.Context(0).set_tree(p.tree, p.conn), Oracle(p)


def _inputs(p, ctx, orc, seed):
    """A positive density with filled ghosts and the field of a random potential: e,
    eabs from the oracle's electric_field! (the library's is bit-exact against it,
    test_gpu_stage.py), eabs's ghosts by fill_ghost!(ExtrapolateConst)."""
    rng = np.random.default_rng(seed)
    n = p.nblk
    ne = 1e18 * (1.0 + rng.random((n, 20, 20))) * (1.0 + 50.0 * (rng.random((n, 1, 1)) < 0.1))
    phi = 2e3 * rng.standard_normal((n, 20, 20))
    orc.fill_ghost_all(phi)
    bc1 = np.ones(9, dtype=np.int8)
    for l in range(1, len(p.tree) + 1):
        olib().orc_fill_ghost(_ptr(ne), orc.ot.ref, l, _ptr(bc1))
    e, eabs = np.zeros((n, 2, 21, 21)), np.zeros((n, 20, 20))
    e0 = np.array(E_BACKGROUND)
    olib().orc_electric_field(_ptr(e), _ptr(eabs), _ptr(phi), p.h1, _ptr(e0), orc.ot.ref)
    for l in range(1, len(p.tree) + 1):
        olib().orc_fill_ghost(_ptr(eabs), orc.ot.ref, l, _ptr(bc1))
    return ne, e, eabs


def test_flux_and_maxdt_bitexact(case):
    import torch
    p, ctx, orc = case
    ne, e, eabs = _inputs(p, ctx, orc, 1)
    tr = mg.Transport(**MINIMAL)
    fg = torch.zeros((p.nblk, 2, 21, 21), dtype=torch.float64, device="cuda")
    mdb = torch.full((p.nblk,), np.inf, dtype=torch.float64, device="cuda")
    mdm = torch.zeros(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    keep = [cuda(ne), cuda(e), cuda(eabs)]  # held until the kernel has run
    ctx.check(mg.lib().srmg_streamer_flux_dev(ctx.handle, fg.data_ptr(), mdb.data_ptr(), mdm.data_ptr(),
                                              *[x.data_ptr() for x in keep], p.nblk, p.h1, ctypes.byref(tr)))
    ctx.synchronize()
    F, md = so.flux(ne, e, eabs, p.tree, p.h1)
    so.restrict_flux(F, p.conn)
    got = fg.cpu().numpy()
    assert np.array_equal(got.view(np.uint64), F.view(np.uint64))
    assert np.array_equal(mdb.cpu().numpy(), md)
    assert float(mdm.cpu()[0]) == md.min()
    if len(p.conn.refboundary[-1]) or any(len(v) for v in p.conn.refboundary):
        # restrict_flux! changed something: the coarse faces differ from the unrestricted flux
        F0, _ = so.flux(ne, e, eabs, p.tree, p.h1)
        assert not np.array_equal(F0, F)


@pytest.mark.parametrize("geom", [gen.GEOM_CYL1, gen.GEOM_CART, gen.GEOM_CYL2])
def test_rates_match_oracle(case, geom):
    import torch
    p, ctx, orc = case
    ne, e, eabs = _inputs(p, ctx, orc, 2)
    F, _ = so.flux(ne, e, eabs, p.tree, p.h1)
    so.restrict_flux(F, p.conn)
    tr = mg.Transport(**MINIMAL)
    dne = torch.zeros((p.nblk, 20, 20), dtype=torch.float64, device="cuda")
    dni = torch.zeros_like(dne)
    torch.cuda.synchronize()
    keep = [cuda(ne), cuda(eabs), cuda(F)]  # held until the kernel has run
    ctx.check(mg.lib().srmg_streamer_rates_dev(ctx.handle, dne.data_ptr(), dni.data_ptr(),
                                               *[x.data_ptr() for x in keep], p.nblk, p.h1, geom,
                                               ctypes.byref(tr)))
    ctx.synchronize()
    wne, wni = so.rates(ne, eabs, F, p.tree, p.h1, geom)
    gne, gni = dne.cpu().numpy(), dni.cpu().numpy()
    for got, want in ((gne, wne), (gni, wni)):
        assert np.linalg.norm(got - want) <= REL_RATES * np.linalg.norm(want)
        # only the valid cells of leaf blocks are written
        assert np.array_equal(got == 0.0, want == 0.0)


def test_interp_copy_ghosts_bitexact(case):
    p, ctx, orc = case
    rng = np.random.default_rng(3)
    u0 = rng.standard_normal((p.nblk, 20, 20))
    bc1 = np.ones(9, dtype=np.int8)
    for l in range(1, len(p.tree) + 1):
        ug = cuda(u0)
        mg.fill_ghost_(ctx, ug, l, bc1, mask=15)
        ctx.synchronize()
        uo = u0.copy()
        olib().orc_fill_ghost_copy(_ptr(uo), orc.ot.ref, l)
        olib().orc_fill_ghost_bnd(_ptr(uo), orc.ot.ref, l, _ptr(bc1))
        so.interp_copy_ghosts(uo, p.conn, l)
        assert np.array_equal(ug.cpu().numpy().view(np.uint64), uo.view(np.uint64)), f"level {l}"


def test_ssprk3_stages_bitexact(case):
    p, ctx, _ = case
    rng = np.random.default_rng(4)
    n, d1, d2, d3 = (rng.standard_normal((p.nblk, 20, 20)) * 1e20 for _ in range(4))
    dt = 4.1e-12
    for stage in (1, 2, 3):
        out = cuda(np.zeros_like(n))
        keep = [cuda(n), cuda(d1), cuda(d2), cuda(d3)]  # held until the kernel has run
        ctx.check(mg.lib().srmg_ssprk3_stage_dev(ctx.handle, out.data_ptr(), *[x.data_ptr() for x in keep],
                                                 n.size, dt, stage))
        ctx.synchronize()
        want = so.ssprk3_stage(n, d1, d2, d3, dt, stage)
        assert np.array_equal(out.cpu().numpy().view(np.uint64), want.view(np.uint64)), stage


def test_refusals(case):
    p, ctx, _ = case
    tr = mg.Transport(**dict(MINIMAL, D=0.0))
    rc = mg.lib().srmg_streamer_rates_dev(ctx.handle, 1, 1, 1, 1, 1, p.nblk, p.h1, 1, ctypes.byref(tr))
    assert rc == mg.SRMG_ERR_BADARG
    rc = mg.lib().srmg_ssprk3_stage_dev(ctx.handle, 1, 1, 1, 1, 1, 10, 1e-12, 4)
    assert rc == mg.SRMG_ERR_BADARG


def _oracle_stage(p, orc, phi, ne, ni, h1, eb, tol):
    """One derivs! of the oracle: charge, restrict_full, FP64 solve from phi, then the
    density's ghosts, the field and the rates."""
    q = np.zeros_like(ne)
    olib().orc_netcharge(_ptr(q), _ptr(ne), _ptr(ni), orc.ot.ref)
    olib().orc_restrict_full(_ptr(q), orc.ot.ref)
    orc.solve(phi, q, tol, max_cycles=500)
    olib().orc_restrict_full(_ptr(ne), orc.ot.ref)
    bc1 = np.ones(9, dtype=np.int8)
    for l in range(1, len(p.tree) + 1):
        olib().orc_fill_ghost_copy(_ptr(ne), orc.ot.ref, l)
        olib().orc_fill_ghost_bnd(_ptr(ne), orc.ot.ref, l, _ptr(bc1))
        so.interp_copy_ghosts(ne, p.conn, l)
        orc.fill_ghost(phi, l)
    e, eabs = np.zeros((p.nblk, 2, 21, 21)), np.zeros_like(ne)
    e0 = np.asarray(eb, dtype=np.float64)
    olib().orc_electric_field(_ptr(e), _ptr(eabs), _ptr(phi), h1, _ptr(e0), orc.ot.ref)
    for l in range(1, len(p.tree) + 1):
        olib().orc_fill_ghost(_ptr(eabs), orc.ot.ref, l, _ptr(bc1))
    F, md = so.flux(ne, e, eabs, p.tree, h1)
    so.restrict_flux(F, p.conn)
    dne, dni = so.rates(ne, eabs, F, p.tree, h1, p.geom)
    return (dne, dni), md


def test_whole_ssprk3_step_matches_oracle():
    """Streamer.advance (three stages, each a library Poisson solve to 1e-12) against
    the oracle's step! with FP64 solves to 1e-12: densities and charge agree to the
    solves' accuracy."""
    tol = 1e-12
    s = Streamer(seed=7, device=0, tol=tol)
    # the library's stage solves in FP64 to the same tolerance as the oracle's
    s._solve = lambda: mg.solve(s.ctx, s.phi, s.b, s.s, s.geom, s.bc, tol=tol, mode=mg.MODE_FP64)
    s._solve()
    p = s.problem
    orc = Oracle(p)
    ne, ni, phi = (x.cpu().numpy().copy() for x in (s.ne, s.nion, s.phi))
    s.advance()
    # the oracle's step! (src/streamer.jl:386-425)
    (d1, md) = _oracle_stage(p, orc, phi, ne, ni, p.h1, s.eb, tol)[0:2]
    dt = 0.8 * md.min()
    assert dt == pytest.approx(s.last_dt, rel=1e-9)
    n1 = [so.ssprk3_stage(x, d1[k], None, None, dt, 1) for k, x in enumerate((ne, ni))]
    d2, _ = _oracle_stage(p, orc, phi, n1[0], n1[1], p.h1, s.eb, tol)
    n1 = [so.ssprk3_stage(x, d1[k], d2[k], None, dt, 2) for k, x in enumerate((ne, ni))]
    d3, _ = _oracle_stage(p, orc, phi, n1[0], n1[1], p.h1, s.eb, tol)
    out = [so.ssprk3_stage(x, d1[k], d2[k], d3[k], dt, 3) for k, x in enumerate((ne, ni))]
    for x in out:
        olib().orc_restrict_full(_ptr(x), orc.ot.ref)
    valid = np.zeros(ne.shape, dtype=bool)
    valid[:, 2:18, 2:18] = True
    for got, want in ((s.ne, out[0]), (s.nion, out[1])):
        g = got.cpu().numpy()
        assert np.linalg.norm((g - want)[valid]) <= 1e-9 * np.linalg.norm(want[valid])
    s.ctx.close()
