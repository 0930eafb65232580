"""The streamer-transport oracle (oracle/streamer_oracle.py) on the host: the Koren
limiter's published values, upwinding, the flux divergence's conservation on uniform
and refined trees (with restrict_flux! at refinement boundaries), the geometry factors,
and the SSPRK3 combinations.  Known answers derived from the reference's formulas
(src/fluid.jl:8-94, 265-280; src/geometry.jl:27-29; src/streamer.jl:400-413)."""
import numpy as np
import pytest

import streamer_oracle as so
from srmg import gen


def test_koren_limited_values():
    # psi(theta) b with theta = a / b: 0 for theta < 0, theta for 0 < theta <= 0.4,
    # 1/3 + theta/6 for 0.4 < theta < 4, 1 for theta >= 4 (src/fluid.jl:265-280)
    b = 1.0
    for theta, want in ((-1.0, 0.0), (0.2, 0.2), (0.4, 0.4), (1.0, 0.5), (2.0, 2.0 / 3.0), (3.9, 1.0 / 3 + 3.9 / 6),
                        (4.5, 1.0), (100.0, 1.0)):
        got = float(so.koren_limited(theta * b, b))
        assert abs(got - want * b) <= 1e-15, (theta, got, want)
    # continuity at the branch points and the sign of b
    assert float(so.koren_limited(-2.0, -1.0)) == pytest.approx(-2.0 / 3.0, abs=1e-15)
    assert float(so.koren_limited(0.0, 5.0)) == 0.0 and float(so.koren_limited(3.0, 0.0)) == 0.0


def _fields(p, seed, e0=(0.0, -1.5e6)):
    """A random positive density (ghosts included), random face fields around e0 and a
    random |E| (the field only feeds the flux here)."""
    rng = np.random.default_rng(seed)
    n = p.nblk
    ne = 1e18 * (1.0 + rng.random((n, 20, 20)))
    e = np.zeros((n, 2, 21, 21))
    e[:, 0] = e0[0] + 1e5 * rng.standard_normal((n, 21, 21))
    e[:, 1] = e0[1] + 1e5 * rng.standard_normal((n, 21, 21))
    eabs = 1.5e6 * (1.0 + 0.1 * rng.random((n, 20, 20)))
    return ne, e, eabs


def _volume_sum(dne, tree, h1, geom):
    """sum over leaf cells of the cell volume (per radian) times dne."""
    ids, lev, crd = so.leaf_blocks(tree)
    tot, mag = 0.0, 0.0
    for k, b in enumerate(ids):
        h = h1 / 2 ** (lev[k] - 1)
        i = np.arange(1, 17) + 16 * (crd[k][0] - 1)
        r = (i - 0.5) * h if geom == 1 else np.ones(16)
        v = (dne[b, 2:18, 2:18] * r[None, :]) * h * h
        tot += v.sum()
        mag += np.abs(v).sum()
    return tot, mag


@pytest.mark.parametrize("geom,refined", [(0, False), (1, False), (0, True)])
def test_flux_divergence_conserves(geom, refined):
    """With zero chemistry, the volume-weighted sum of dne over the leaf cells is the
    net flux through the domain boundary; with zero velocity at the boundary faces
    and Neumann (mirror) ghosts of ne, nothing crosses it, so the sum vanishes, across
    refinement boundaries too (restrict_flux!).  (In cylindrical geometry the
    reference's plain mean of the two fine z-face fluxes is not r-weighted, so a
    refined cylindrical tree conserves only approximately; not tested.)"""
    p = gen.config2(seed=5, target_leaf=40_000, extra=3) if refined else gen.config1()
    tree = p.tree
    ne, e, eabs = _fields(p, 3)
    # mirror ghosts (Neumann) everywhere on the domain boundary and zero normal field
    # there; interior ghosts: copies, as the fills would leave them
    conn = p.conn
    for v in conn.boundary:
        for rec in v:
            b = int(rec["block"]) - 1
            f = tuple(int(x) for x in rec["face"])
            if f == (-1, 0):
                ne[b, :, 0:2] = ne[b, :, 3:1:-1]
                e[b, 0, :, 2] = 0.0
            elif f == (1, 0):
                ne[b, :, 18:20] = ne[b, :, 17:15:-1]
                e[b, 0, :, 18] = 0.0
            elif f == (0, -1):
                ne[b, 0:2, :] = ne[b, 3:1:-1, :]
                e[b, 1, 2, :] = 0.0
            elif f == (0, 1):
                ne[b, 18:20, :] = ne[b, 17:15:-1, :]
                e[b, 1, 18, :] = 0.0
    F, _ = so.flux(ne, e, eabs, tree, p.h1)
    # faces shared by two blocks must carry one flux: make the neighbours agree by
    # averaging (the fills would make them agree exactly)
    for v in conn.neighbor:
        for rec in v:
            a, b = int(rec["from"]) - 1, int(rec["to"]) - 1
            f = tuple(int(x) for x in rec["face"])
            if f == (1, 0):
                F[b, 0, 2:18, 2] = F[a, 0, 2:18, 18]
            elif f == (0, 1):
                F[b, 1, 2, 2:18] = F[a, 1, 18, 2:18]
    so.restrict_flux(F, conn)
    tr = dict(so.MINIMAL, ai=0.0, aa=0.0)
    dne, dni = so.rates(ne, eabs, F, tree, p.h1, geom, tr)
    tot, mag = _volume_sum(dne, tree, p.h1, geom)
    assert mag > 0 and abs(tot) <= 1e-12 * mag, (tot, mag)
    assert np.all(dni == 0.0)


def test_upwinding_uses_the_upstream_cells():
    """A uniform field along +r (v < 0: electrons drift towards -r) takes the face
    value from the cell on the +r side; with a linear density profile the limiter is
    at theta = 1 and the face value is n_u + (n_d - n_u) / 2 (psi(1) = 1/2)."""
    p = gen.config1()
    n = p.nblk
    x = np.arange(20, dtype=float)
    ne = np.broadcast_to(1e18 + 1e16 * x[None, None, :], (n, 20, 20)).copy()
    e = np.zeros((n, 2, 21, 21))
    e[:, 0] = 1.0e6
    eabs = np.full((n, 20, 20), 1.0e6)
    F, md = so.flux(ne, e, eabs, p.tree, p.h1)
    mu, D = so.MINIMAL["mu"], so.MINIMAL["D"]
    ids, lev, _ = so.leaf_blocks(p.tree)
    b = ids[0]
    h = p.h1 / 2 ** (lev[0] - 1)
    xf = 5  # face between cells 4 and 5
    v = -1.0e6 * mu
    nu, nd = ne[b, 7, xf], ne[b, 7, xf - 1]
    want = v * (nu + (nd - nu) / 2) + (D * (ne[b, 7, xf - 1] - ne[b, 7, xf])) / h
    assert F[b, 0, 7, xf] == pytest.approx(want, rel=1e-15)
    assert np.all(np.isfinite(md[ids])) and np.all(md[ids] > 0)


def test_ssprk3_combinations():
    rng = np.random.default_rng(1)
    n, d1, d2, d3 = (rng.standard_normal(1000) for _ in range(4))
    dt = 3.7e-11
    assert np.array_equal(so.ssprk3_stage(n, d1, d2, d3, dt, 1), n + d1 * dt)
    assert np.array_equal(so.ssprk3_stage(n, d1, d2, d3, dt, 2), n + (d1 * (dt / 4) + d2 * (dt / 4)))
    # a constant rate: the three stages advance by exactly that rate times dt (to rounding)
    c = np.full(10, 2.5)
    out = so.ssprk3_stage(np.zeros(10), c, c, c, 1.0, 3)
    assert np.allclose(out, 2.5, rtol=1e-15)
