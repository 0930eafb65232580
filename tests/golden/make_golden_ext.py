"""Generate tests/golden/ext_hashes.json: a second, independent restatement in plain
Python loops of the compact order-4 discretisation (2D, BoxStencil tree) and of the
three-dimensional operations, run on tiny trees; the SHA-256 of every output's bytes
pins the C oracle (tests/test_oracle_golden_ext.py) bit for bit.

Why: as for mg_tiny.npz (make_golden.py), the reference ships no golden vectors and
cannot run here, so the oracle is pinned to an independently written restatement of
the same reference lines.  Exact IEEE doubles (Python floats, no contraction); the
reference's muladd is a correctly rounded fused multiply-add computed with exact
rationals.  Inputs come from seeded numpy generators, so only hashes are stored.

Run:  python tests/golden/make_golden_ext.py   (writes tests/golden/ext_hashes.json)
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "steamroller.jl_b200"))
sys.path.insert(0, HERE)

import make_golden as g2  # noqa: E402  (the 2D fill helpers take any face in {-1,0,1}^2)
from srmg.tree import Tree, populate, refine_block, connectivity, boundaryconditions, BOX2  # noqa: E402
from srmg import tree3 as t3  # noqa: E402

M, G = 16, 2
S = M + 2 * G


def fma(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


# ---------------------------------------------------------------- order 4, 2D

def order4_tree():
    t = Tree((1, 1), 3)
    populate(t, 2)
    refine_block(t, 2, (1, 1), BOX2)
    refine_block(t, 2, (2, 2), BOX2)
    t.sync()
    return t


def lap4(u, blk, i, j, gi, geom):
    """applystencil for LaplacianDiscretization{2,4} (src/laplacian.jl:133-202): the 3x3
    literal (rows: offset along dimension 1, columns: along dimension 2) walked
    column-major, literal zeros skipped, then / 6.  gi is the radial 1-based global
    index (unused for Cartesian)."""
    if geom == 0:
        lit = [[1, 4, 1], [4, -20, 4], [1, 4, 1]]
    else:
        n = gi
        lo = 2 * (n - 1) / (2 * n - 1)
        hi = 2 * n / (2 * n - 1)
        edge_lo = 4 * (-2 + 9 * n - 16 * n ** 2 + 8 * n ** 3) / (2 * n - 1) ** 3
        centre = -16 * (1 - 5 * n + 5 * n ** 2) / (1 - 2 * n) ** 2
        edge_hi = 4 * (1 + n - 8 * n ** 2 + 8 * n ** 3) / (2 * n - 1) ** 3
        if geom == 1:
            lit = [[lo, edge_lo, lo], [4, centre, 4], [hi, edge_hi, hi]]
        else:
            lit = [[lo, 4, hi], [edge_lo, centre, edge_hi], [lo, 4, hi]]
    v = 0.0
    for col in range(3):          # column-major: the row index runs fastest
        for row in range(3):
            c = lit[row][col]
            v += c * g2.at(u, blk, i + row - 1, j + col - 1)
    return v / 6


def diag4(gi, geom):
    if geom == 0:
        return -20 / 6
    n = gi
    return -16 * (1 - 5 * n + 5 * n ** 2) / (1 - 2 * n) ** 2 / 6


def radial_index(c, i, j, geom):
    """1-based global index along the radial dimension of local 1-based cell (i, j)."""
    if geom == 1:
        return i - G + M * (c[0] - 1)
    if geom == 2:
        return j - G + M * (c[1] - 1)
    return 0


def gs4_level(u, b, omega, s, tree, l, P1, P2, geom):
    for (c, blk) in tree[l - 1].pairs:
        for i2 in range(G + 1, G + M + 1, 2):
            for i1 in range(G + 1, G + M + 1, 2):
                I1, I2 = i1 + P1, i2 + P2
                gi = radial_index(c, I1, I2, geom)
                Lu = lap4(u, blk, I1, I2, gi, geom)
                upd = omega * (Lu + s * g2.at(b, blk, I1, I2)) / diag4(gi, geom)
                g2.put(u, blk, I1, I2, g2.at(u, blk, I1, I2) - upd)


def gs4_iter(u, b, omega, s, n, l, tree, conn, bc, geom):
    for _ in range(n):
        for P1, P2 in ((0, 0), (0, 1), (1, 0), (1, 1)):
            gs4_level(u, b, omega, s, tree, l, P1, P2, geom)
            g2.fill_copy(u, conn.neighbor[l - 1])
            g2.fill_bnd(u, conn.boundary[l - 1], bc)


def residual4(r, u, b, s, tree, l, geom):
    for (c, blk) in tree[l - 1].pairs:
        for I2 in range(G + 1, G + M + 1):
            for I1 in range(G + 1, G + M + 1):
                Lu = lap4(u, blk, I1, I2, radial_index(c, I1, I2, geom), geom)
                g2.put(r, blk, I1, I2, -(g2.at(b, blk, I1, I2) + Lu / s))


def rhs4(q1, q, tree, l, geom):
    """rhs! for order 4 (src/laplacian.jl:141-148, 166-173): the literal's nonzero
    entries in column-major order, then / 12."""
    for (c, blk) in tree[l - 1].pairs:
        for I2 in range(G + 1, G + M + 1):
            for I1 in range(G + 1, G + M + 1):
                n = radial_index(c, I1, I2, geom)
                if geom == 1:
                    lit = [[0, (2 * n - 2) / (2 * n - 1), 0], [1, 8, 1], [0, 2 * n / (2 * n - 1), 0]]
                elif geom == 2:
                    lit = [[0, 1, 0], [(2 * n - 2) / (2 * n - 1), 8, 2 * n / (2 * n - 1)], [0, 1, 0]]
                else:
                    lit = [[0, 1, 0], [1, 8, 1], [0, 1, 0]]
                v = 0.0
                for col in range(3):
                    for row in range(3):
                        if lit[row][col] == 0:
                            continue
                        v += lit[row][col] * g2.at(q, blk, I1 + row - 1, I2 + col - 1)
                g2.put(q1, blk, I1, I2, v / 12)


# ---------------------------------------------------------------- three dimensions

S3 = S * S * S


def a3(f, blk, i, j, k):
    return f[blk - 1, k - 1, j - 1, i - 1]


def p3(f, blk, i, j, k, v):
    f[blk - 1, k - 1, j - 1, i - 1] = v


def rng3(face):
    return g2.grange(face)


def fill3_copy(u, nb):
    for e in nb:
        frm, to = int(e["from"]), int(e["to"])
        f = [int(x) for x in e["face"]]
        cnt = [M if f[d] == 0 else G for d in range(3)]
        for i3 in range(1, cnt[2] + 1):
            for i2 in range(1, cnt[1] + 1):
                for i1 in range(1, cnt[0] + 1):
                    ii = (i1, i2, i3)
                    a = [G + ii[d] if f[d] == 0 else (ii[d] + G if f[d] == -1 else ii[d] + M) for d in range(3)]
                    b = [G + ii[d] if f[d] == 0 else (ii[d] if f[d] == 1 else ii[d] + M + G) for d in range(3)]
                    p3(u, to, *b, a3(u, frm, *a))


def fill3_bnd(u, bd, bc27):
    for e in bd:
        blk = int(e["block"])
        face = [int(x) for x in e["face"]]
        bnd = [int(x) for x in e["bnd"]]
        s = float(int(bc27[(1 + bnd[0]) + 3 * (1 + bnd[1]) + 9 * (1 + bnd[2])]))
        for k in rng3(face[2]):
            for j in rng3(face[1]):
                for i in rng3(face[0]):
                    p3(u, blk, i, j, k, s * a3(u, blk, g2.mir(i, bnd[0]), g2.mir(j, bnd[1]), g2.mir(k, bnd[2])))


def interp3(dest, dblk, dlo, src, sblk, srng, add):
    """interp!(InterpLinear) for D = 3 (src/interp.jl:24-63), weights 1/4 (:10-11)."""
    for k3, s3 in enumerate(srng[2]):
        for k2, s2 in enumerate(srng[1]):
            for k1, s1 in enumerate(srng[0]):
                for i3 in (0, 1):
                    for i2 in (0, 1):
                        for i1 in (0, 1):
                            d = (dlo[0] + 2 * k1 + i1, dlo[1] + 2 * k2 + i2, dlo[2] + 2 * k3 + i3)
                            f = 0.25 * a3(src, sblk, s1, s2, s3)
                            f += 0.25 * a3(src, sblk, s1 + 2 * i1 - 1, s2, s3)
                            f += 0.25 * a3(src, sblk, s1, s2 + 2 * i2 - 1, s3)
                            f += 0.25 * a3(src, sblk, s1, s2, s3 + 2 * i3 - 1)
                            if add:
                                f = f + a3(dest, dblk, *d)
                            p3(dest, dblk, *d, f)


def fill3_interp(u, rb):
    gh = G // 2
    for e in rb:
        face = [int(x) for x in e["face"]]
        sb = [int(x) for x in e["subblock"]]
        srng, dlo = [], []
        for d in range(3):
            r = g2.sbrange(sb[d])
            if -face[d] == -1:
                r = range(r.start, r.start + gh)
            elif -face[d] == 1:
                r = range(r.stop - gh, r.stop)
            srng.append(r)
            dlo.append(rng3(face[d]).start)
        interp3(u, int(e["fine"]), dlo, u, int(e["coarse"]), srng, False)


def fill3(u, conn, l, bc27):
    fill3_copy(u, conn.neighbor[l - 1])
    fill3_bnd(u, conn.boundary[l - 1], bc27)
    fill3_interp(u, conn.refboundary[l - 1])


def restrict3(u, ch):
    for e in ch:
        fine, coarse = int(e["fine"]), int(e["coarse"])
        d0 = [g2.sbrange(int(x)).start for x in e["subblock"]]
        for c3 in range(M // 2):
            for c2 in range(M // 2):
                for c1 in range(M // 2):
                    f = 0.0
                    for i3 in (0, 1):
                        for i2 in (0, 1):
                            for i1 in (0, 1):
                                f += a3(u, fine, G + 1 + 2 * c1 + i1, G + 1 + 2 * c2 + i2, G + 1 + 2 * c3 + i3)
                    p3(u, coarse, d0[0] + c1, d0[1] + c2, d0[2] + c3, f / 8)


def interp3_add(u, u1, ch):
    for e in ch:
        sb = [int(x) for x in e["subblock"]]
        interp3(u, int(e["fine"]), (G + 1, G + 1, G + 1), u1, int(e["coarse"]), [g2.sbrange(x) for x in sb], True)


def lap3(u, blk, i, j, k, op, s, k2):
    """3D stencils (src/laplacian.jl:274-340, src/helmholtz.jl:74-89): the 3x3x3
    literal, first offset fastest, slab slowest, literal zeros skipped."""
    v = 0.0
    for d3 in (-1, 0, 1):
        for d2 in (-1, 0, 1):
            for d1 in (-1, 0, 1):
                nz = abs(d1) + abs(d2) + abs(d3)
                if op == 2:
                    c = {0: -24, 1: 2, 2: 1, 3: 0}[nz]
                else:
                    c = {0: (-6 - s * k2) if op == 1 else -6, 1: 1, 2: 0, 3: 0}[nz]
                if c == 0:
                    continue
                v += c * a3(u, blk, i + d1, j + d2, k + d3)
    return v / 6 if op == 2 else v


def gs3_rb(u, b, omega, s, tree, l, P, op, k2):
    c = (-6 - s * k2) if op == 1 else -6
    for (_, blk) in tree[l - 1].pairs:
        for i3 in range(G + 1, G + M + 1):
            for i2 in range(G + 1, G + M + 1):
                for i1 in range(G + 1, G + M + 1, 2):
                    I1 = i1 + (P ^ (i2 & 1) ^ (i3 & 1))
                    Lu = lap3(u, blk, I1, i2, i3, op, s, k2)
                    v = fma(s, a3(b, blk, I1, i2, i3), Lu)
                    p3(u, blk, I1, i2, i3, fma(-(omega / c), v, a3(u, blk, I1, i2, i3)))


def gs3_iter(u, b, omega, s, n, l, tree, conn, bc27, op, k2):
    for _ in range(n):
        for P in (0, 1):
            gs3_rb(u, b, omega, s, tree, l, P, op, k2)
            fill3_copy(u, conn.neighbor[l - 1])
            fill3_bnd(u, conn.boundary[l - 1], bc27)


def residual3(r, u, b, s, tree, l, op, k2):
    for (_, blk) in tree[l - 1].pairs:
        for k in range(G + 1, G + M + 1):
            for j in range(G + 1, G + M + 1):
                for i in range(G + 1, G + M + 1):
                    p3(r, blk, i, j, k, -(a3(b, blk, i, j, k) + lap3(u, blk, i, j, k, op, s, k2) / s))


def postrestrict3(bf, u, r, s, tree, l, ch, op, k2):
    for e in ch:
        blk = int(e["coarse"])
        rr = [g2.sbrange(int(x)) for x in e["subblock"]]
        for k in rr[2]:
            for j in rr[1]:
                for i in rr[0]:
                    p3(bf, blk, i, j, k, -(a3(r, blk, i, j, k) + lap3(u, blk, i, j, k, op, s, k2) / s))


def vcycle3(u, b, r, u1, s, tree, conn, bc27, ndown, ntop, nup, op=0, k2=0.0):
    lmax = len(tree)
    for l in range(lmax, 1, -1):
        sl = s / (1 << (l - 1)) ** 2
        gs3_iter(u, b, 1.0, sl, ndown, l, tree, conn, bc27, op, k2)
        restrict3(u, conn.child[l - 1])
        fill3(u, conn, l - 1, bc27)
        for (_, blk) in tree[l - 2].pairs:
            u1[blk - 1] = u[blk - 1]
        residual3(r, u, b, sl, tree, l, op, k2)
        fill3(r, conn, l, bc27)
        restrict3(r, conn.child[l - 1])
        fill3(r, conn, l - 1, bc27)
        postrestrict3(b, u, r, 4 * sl, tree, l, conn.child[l - 1], op, k2)
    gs3_iter(u, b, 1.0, s, ntop, 1, tree, conn, bc27, op, k2)
    for l in range(2, lmax + 1):
        sl = s / (1 << (l - 1)) ** 2
        for (_, blk) in tree[l - 2].pairs:
            u1[blk - 1] = u[blk - 1] - u1[blk - 1]
        fill3(u1, conn, l - 1, bc27)
        interp3_add(u, u1, conn.child[l - 1])
        fill3(u, conn, l, bc27)
        gs3_iter(u, b, 1.0, sl, nup, l, tree, conn, bc27, op, k2)
        fill3(u, conn, l, bc27)


def tiny_octree():
    t = t3.Tree3((1, 1, 1), 3)
    t3.populate(t, 2)
    t3.refine_block(t, 2, (2, 1, 2))
    t.sync()
    return t


# ---------------------------------------------------------------- main

def inputs2(nblk):
    rng = np.random.default_rng(4401)
    return rng.standard_normal((nblk, S, S)), rng.standard_normal((nblk, S, S))


def inputs3(nblk):
    rng = np.random.default_rng(4402)
    return rng.standard_normal((nblk, S, S, S)), rng.standard_normal((nblk, S, S, S))


BC2 = boundaryconditions(((1, -1), (-1, 1)))
BC3 = t3.boundaryconditions(((1, -1), (-1, 1), (-1, -1)))


def main():
    out = {}
    tree = order4_tree()
    conn = connectivity(tree, BOX2)
    u0, b0 = inputs2(tree.nblocks_created)
    for l in (1, 2, 3):
        u = u0.copy()
        g2.fill_ghost(u, conn, l, BC2)
        out[f"o4_fill_l{l}"] = digest(u)
    for geom in (0, 1, 2):
        u = u0.copy()
        gs4_iter(u, b0, 1.0, 0.37, 2, 3, tree, conn, BC2, geom)
        out[f"o4_gs_iter_l3_g{geom}"] = digest(u)
        r = np.zeros_like(u0)
        residual4(r, u0, b0, 0.37, tree, 3, geom)
        out[f"o4_residual_l3_g{geom}"] = digest(r)
        q1 = np.zeros_like(u0)
        rhs4(q1, u0, tree, 3, geom)
        out[f"o4_rhs_l3_g{geom}"] = digest(q1)
    t = tiny_octree()
    c3 = t3.connectivity(t, t3.STAR3)
    cb = t3.connectivity(t, t3.BOX3)
    v0, w0 = inputs3(t.nblocks_created)
    for name, cc in (("star", c3), ("box", cb)):
        for l in (1, 2, 3):
            u = v0.copy()
            fill3(u, cc, l, BC3)
            out[f"d3_fill_{name}_l{l}"] = digest(u)
    u = v0.copy()
    restrict3(u, c3.child[2])
    out["d3_restrict_l3"] = digest(u)
    u = v0.copy()
    interp3_add(u, w0, c3.child[2])
    out["d3_interp_add_l3"] = digest(u)
    for op, k2 in ((0, 0.0), (1, 30.0)):
        u = v0.copy()
        gs3_iter(u, w0, 1.0, 0.37, 1, 3, t, c3, BC3, op, k2)
        out[f"d3_gs_iter_l3_op{op}"] = digest(u)
        r = np.zeros_like(v0)
        residual3(r, v0, w0, 0.37, t, 3, op, k2)
        out[f"d3_residual_l3_op{op}"] = digest(r)
    r = np.zeros_like(v0)
    residual3(r, v0, w0, 0.37, t, 3, 2, 0.0)
    out["d3_residual_l3_op2"] = digest(r)
    u, b, r, u1 = v0.copy(), w0.copy(), np.zeros_like(v0), np.zeros_like(v0)
    for l in (1, 2, 3):
        fill3(u, c3, l, BC3)
    vcycle3(u, b, r, u1, 0.5, t, c3, BC3, 1, 2, 1)
    out["d3_vcycle_u"] = digest(u)
    out["d3_vcycle_b"] = digest(b)
    with open(os.path.join(HERE, "ext_hashes.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", len(out), "hashes")


if __name__ == "__main__":
    main()
