"""numpy restatement of the electron transport and chemistry of derivs! and of the
SSPRK3 combinations of step! (the streamer stepper that generates training pairs).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of libsrmg's stepper
kernels.  Parity with the reference is unpinned (the reference has no tests or golden
vectors and cannot run here); each routine restates the cited reference code with IEEE
double arithmetic in the same operation order, one rounding per operation.

Fields: scalar block fields as (nblk, 20, 20) arrays indexed [blk - 1, y, x] (x = r,
0-based, ghosts included); vector block fields (VectorBlockField{2,16,2},
src/blockfield.jl:84-95) as (nblk, 2, 21, 21) arrays indexed [blk - 1, d, y, x], face
(x, y) of component d lying between cell (x, y) - e_d and cell (x, y).
"""
from __future__ import annotations

import numpy as np

ELEMENTARY_CHARGE = 1.6021766208e-19   # src/constants.jl:55
EPSILON_0 = 8.854187817620389e-12     # src/constants.jl:56

# MINIMAL_TRANSPORT_MODEL (src/simulate.jl:5-10)
MINIMAL = dict(mu=0.0372193, D=0.18, ai=433200.0, Ei=2e7, aa=2000.0, Ea=3e6)


def koren_limited(a, b):
    """koren_limited(a, b) (src/fluid.jl:274-280), elementwise, branches in order."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    out = a.copy()
    mid = np.abs(10.0 * a) > np.abs(4.0 * b)
    out = np.where(mid, b / 3.0 + a / 6.0, out)
    out = np.where(np.abs(a) > np.abs(4.0 * b), b, out)
    out = np.where(a * b < 0, 0.0, out)
    return out


def leaf_blocks(tree):
    """(0-based block ids, levels, coords) of the leaf blocks (isleaf, src/tree.jl:105-115)."""
    ids, lev, crd = [], [], []
    for layer in tree:
        for c, blk in layer.pairs:
            if tree.isleaf(layer.level, c):
                ids.append(blk - 1)
                lev.append(layer.level)
                crd.append(c)
    return np.array(ids, dtype=np.int64), np.array(lev, dtype=np.int64), np.array(crd, dtype=np.int64)


def flux(ne, e, eabs, tree, h1, tr=MINIMAL):
    """flux!(tree, FluxSchemeKoren(), flux, ne, e, eabs, h, trans, dens, maxdt)
    (src/fluid.jl:44-94) for the MinimalTransportModel and a uniform gas density
    (theta = 1).  Returns (flux, maxdt per block: +inf except on leaf blocks)."""
    F = np.zeros((ne.shape[0], 2, 21, 21))
    maxdt = np.full(ne.shape[0], np.inf)
    ids, lev, _ = leaf_blocks(tree)
    maxwell = EPSILON_0 / ELEMENTARY_CHARGE
    mu, D = tr["mu"], tr["D"]
    with np.errstate(divide="ignore", invalid="ignore"):
        for l in np.unique(lev):
            b = ids[lev == l]
            h = h1 / float(1 << (int(l) - 1))
            n = ne[b]
            ea = eabs[b]
            md = np.full(len(b), np.inf)
            for d in (0, 1):
                # faces I = (x, y): d = 0 -> x 2..18, y 2..17; d = 1 -> x 2..17, y 2..18
                if d == 0:
                    ys, xs = np.meshgrid(np.arange(2, 18), np.arange(2, 19), indexing="ij")
                    sx, sy = 1, 0
                else:
                    ys, xs = np.meshgrid(np.arange(2, 19), np.arange(2, 18), indexing="ij")
                    sx, sy = 0, 1
                at = lambda f, k: f[:, ys + k * sy, xs + k * sx]
                ed = e[b][:, d, ys, xs]
                eabs1 = (at(ea, 0) + at(ea, -1)) / 2.0
                v = (-ed) * mu
                up = ~np.signbit(v)  # sv = +1
                nu = np.where(up, at(n, -1), at(n, 0))
                nu2 = np.where(up, at(n, -2), at(n, 1))
                nd = np.where(up, at(n, 0), at(n, -1))
                Fa = v * (nu + koren_limited(nu - nu2, nd - nu))
                tmax = (maxwell * eabs1) / np.abs(Fa)
                Ff = Fa + (D * (at(n, -1) - at(n, 0))) / h
                F[b[:, None, None], d, ys[None], xs[None]] = Ff
                m = np.fmin(np.fmin(h / np.abs(v), ((h * h) / D) / 4.0), tmax)
                md = np.fmin(md, m.reshape(len(b), -1).min(axis=1))
            maxdt[b] = md
    return F, maxdt


def restrict_flux(F, conn):
    """restrict_flux!(flux, conn) (src/connectivity.jl:327-360, the generated kernel
    src/restrict.jl:55-78): at every star refinement face, the coarse block's face on
    the half `subblock` covers = ((0 + f_2k) + f_2k+1) / 2 of the fine faces."""
    for v in conn.refboundary:
        for rec in v:
            face = tuple(int(x) for x in rec["face"])
            if sum(abs(x) for x in face) != 1:
                continue  # isaxis
            dim = 0 if face[0] != 0 else 1
            fine, coarse = int(rec["fine"]) - 1, int(rec["coarse"]) - 1
            sb = int(rec["subblock"][1 - dim])
            fn = 2 if face[dim] == -1 else 18     # bndindex(f, face[dim]) - 1
            cn = 18 if face[dim] == -1 else 2     # bndindex(f, -face[dim]) - 1
            for k in range(8):
                ft, ct = 2 + 2 * k, 2 + 8 * (sb - 1) + k
                if dim == 0:
                    a, b_ = F[fine, 0, ft, fn], F[fine, 0, ft + 1, fn]
                    F[coarse, 0, ct, cn] = ((0.0 + a) + b_) / 2.0
                else:
                    a, b_ = F[fine, 1, fn, ft], F[fine, 1, fn, ft + 1]
                    F[coarse, 1, cn, ct] = ((0.0 + a) + b_) / 2.0
    return F


def rates(ne, eabs, F, tree, h1, geom, tr=MINIMAL):
    """chemderivs! (NetIonization over the MinimalTransportModel, src/chemistry.jl:29-82,
    src/transport.jl:30-35; pre then post) and fluxderivs! (src/fluid.jl:8-30) on the
    valid cells of the leaf blocks.  Returns (dne, dni), zero elsewhere."""
    dne, dni = np.zeros_like(ne), np.zeros_like(ne)
    ids, lev, crd = leaf_blocks(tree)
    mu = tr["mu"]
    ys, xs = np.meshgrid(np.arange(2, 18), np.arange(2, 18), indexing="ij")
    for k, b in enumerate(ids):
        h = h1 / float(1 << (int(lev[k]) - 1))
        n1 = ne[b, 2:18, 2:18]
        E = eabs[b, 2:18, 2:18]
        pre = ((mu * E) * n1) * (tr["ai"] * np.exp((-tr["Ei"]) / E))
        post = (((-mu) * E) * n1) * (tr["aa"] * np.exp((-tr["Ea"]) / E))
        chem = pre + post
        dni[b, 2:18, 2:18] = chem
        Jr = 16 * (crd[k][0] - 1) + xs - 1
        Jz = 16 * (crd[k][1] - 1) + ys - 1

        def fac(dim, delta):
            radial = (geom == 1 and dim == 0) or (geom == 2 and dim == 1)
            if geom == 0 or not radial:
                return 1.0
            J = Jr if dim == 0 else Jz
            return np.abs(1.0 + float(delta) / (2.0 * J - 1.0))

        fb = F[b]
        v = chem
        v = v + (fac(0, -1) * fb[0, ys, xs]) / h
        v = v - (fac(0, 1) * fb[0, ys, xs + 1]) / h
        v = v + (fac(1, -1) * fb[1, ys, xs]) / h
        v = v - (fac(1, 1) * fb[1, ys + 1, xs]) / h
        dne[b, 2:18, 2:18] = v
    return dne, dni


def interp_copy_ghosts(u, conn, level):
    """fill_ghost_interp!(u, conn.refboundary[level], InterpCopy()) (src/connectivity.jl:
    251-258, src/interp.jl:66-85): each coarse cell of subblockbnd(subblock, -face)
    copied into the 2 x 2 fine ghost cells it covers."""
    for rec in conn.refboundary[level - 1]:
        face = tuple(int(x) for x in rec["face"])
        if sum(abs(x) for x in face) != 1:
            continue
        fine, coarse = int(rec["fine"]) - 1, int(rec["coarse"]) - 1
        sbr, sbz = int(rec["subblock"][0]), int(rec["subblock"][1])
        for g in range(2):
            for k in range(16):
                if face[0] != 0:
                    x = g if face[0] == -1 else 18 + g
                    y = 2 + k
                    jr = 1 + 8 * sbr if face[0] == -1 else 2 + 8 * (sbr - 1)
                    jz = 2 + 8 * (sbz - 1) + (k >> 1)
                else:
                    y = g if face[1] == -1 else 18 + g
                    x = 2 + k
                    jz = 1 + 8 * sbz if face[1] == -1 else 2 + 8 * (sbz - 1)
                    jr = 2 + 8 * (sbr - 1) + (k >> 1)
                u[fine, y, x] = u[coarse, jz, jr]
    return u


def ssprk3_stage(n, d1, d2, d3, dt, stage):
    """The combinations of step! (src/streamer.jl:400-413)."""
    if stage == 1:
        return n + d1 * dt
    if stage == 2:
        dt1 = dt / 4.0
        return n + (d1 * dt1 + d2 * dt1)
    return n + ((d1 * (dt / 6.0) + d2 * (dt / 6.0)) + d3 * ((2.0 * dt) / 3.0))
