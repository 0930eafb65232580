"""Generate tests/golden/*.npz: a second, independent restatement of the reference's
multigrid arithmetic in plain Python loops, run on tiny trees.

Why: Steamroller.jl ships no tests or golden vectors and cannot run here (no Julia),
so the C oracle cannot be pinned to reference outputs.  These fixtures pin it to an
independently written restatement instead: same reference lines, different code,
exact IEEE double arithmetic (Python floats; muladd as a correctly rounded fused
multiply-add computed with exact rationals).  tests/test_oracle_golden.py checks the
C oracle against them bit for bit.

Run:  python tests/golden/make_golden.py   (writes tests/golden/mg_tiny.npz)
"""
from __future__ import annotations

import os
import sys
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "steamroller.jl_b200"))

from srmg.tree import Tree, populate, refine_block, connectivity, boundaryconditions  # noqa: E402

M, G = 16, 2
S = M + 2 * G


def fma(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def at(f, blk, i, j):
    """1-based (i, j) of 1-based block blk; f is (nblk, S, S) [blk, j, i]."""
    return f[blk - 1, j - 1, i - 1]


def put(f, blk, i, j, v):
    f[blk - 1, j - 1, i - 1] = v


# -- src/connectivity.jl:184-198
def fill_copy(u, nb):
    for e in nb:
        frm, to = int(e["from"]), int(e["to"])
        f = [int(e["face"][0]), int(e["face"][1])]
        rng = [range(1, (M if f[d] == 0 else G) + 1) for d in range(2)]
        for i2 in rng[1]:
            for i1 in rng[0]:
                ii = [i1, i2]
                a = [G + ii[d] if f[d] == 0 else (ii[d] + G if f[d] == -1 else ii[d] + M) for d in range(2)]
                b = [G + ii[d] if f[d] == 0 else (ii[d] if f[d] == 1 else ii[d] + M + G) for d in range(2)]
                put(u, to, b[0], b[1], at(u, frm, a[0], a[1]))


def grange(face):
    if face == 0:
        return range(G + 1, G + M + 1)
    if face == -1:
        return range(1, G + 1)
    return range(M + G + 1, M + 2 * G + 1)


def mir(i, d):
    if d == -1:
        return 2 * G - i + 1
    if d == 1:
        return 2 * (G + M) - i + 1
    return i


# -- src/connectivity.jl:217-231, src/boundary.jl:45-47
def fill_bnd(u, bd, bc):
    for e in bd:
        blk = int(e["block"])
        face = [int(e["face"][0]), int(e["face"][1])]
        bnd = [int(e["bnd"][0]), int(e["bnd"][1])]
        a = float(int(bc[(1 + bnd[0]) + 3 * (1 + bnd[1])]))
        for j in grange(face[1]):
            for i in grange(face[0]):
                put(u, blk, i, j, a * at(u, blk, mir(i, bnd[0]), mir(j, bnd[1])))


def sbrange(sb):
    return range(G + 1 + (sb - 1) * (M // 2), G + sb * (M // 2) + 1)


# -- src/interp.jl:24-63
def interp(dest_f, dblk, dlo, src_f, sblk, srng, add):
    for k2, js2 in enumerate(srng[1]):
        for k1, js1 in enumerate(srng[0]):
            jd0 = (dlo[0] + 2 * k1, dlo[1] + 2 * k2)
            for i2 in (0, 1):
                for i1 in (0, 1):
                    jd = (jd0[0] + i1, jd0[1] + i2)
                    f = 0.5 * at(src_f, sblk, js1, js2)
                    f += 0.25 * at(src_f, sblk, js1 + 2 * i1 - 1, js2)
                    f += 0.25 * at(src_f, sblk, js1, js2 + 2 * i2 - 1)
                    if add:
                        f = f + at(dest_f, dblk, jd[0], jd[1])
                    put(dest_f, dblk, jd[0], jd[1], f)


# -- src/connectivity.jl:251-258, src/blockfield.jl:416-434
def fill_interp(u, rb):
    gh = G // 2
    for e in rb:
        face = [int(e["face"][0]), int(e["face"][1])]
        sb = [int(e["subblock"][0]), int(e["subblock"][1])]
        srng = []
        dlo = []
        for d in range(2):
            r = sbrange(sb[d])
            mf = -face[d]
            if mf == -1:
                r = range(r.start, r.start + gh)
            elif mf == 1:
                r = range(r.stop - gh, r.stop)
            srng.append(r)
            dlo.append(grange(face[d]).start)
        interp(u, int(e["fine"]), dlo, u, int(e["coarse"]), srng, False)


def fill_ghost(u, conn, l, bc):
    fill_copy(u, conn.neighbor[l - 1])
    fill_bnd(u, conn.boundary[l - 1], bc)
    fill_interp(u, conn.refboundary[l - 1])


# -- src/restrict.jl:5-37
def restrict(u, ch):
    for e in ch:
        fine, coarse = int(e["fine"]), int(e["coarse"])
        sb = [int(e["subblock"][0]), int(e["subblock"][1])]
        d0 = (sbrange(sb[0]).start, sbrange(sb[1]).start)
        for k2 in range(M // 2):
            for k1 in range(M // 2):
                js = (G + 1 + 2 * k1, G + 1 + 2 * k2)
                f = 0.0
                for i2 in (0, 1):
                    for i1 in (0, 1):
                        f += at(u, fine, js[0] + i1, js[1] + i2)
                put(u, coarse, d0[0] + k1, d0[1] + k2, f / 4)


# -- src/interp.jl:107-115
def interp_add(u, u1, ch):
    for e in ch:
        sb = [int(e["subblock"][0]), int(e["subblock"][1])]
        interp(u, int(e["fine"]), (G + 1, G + 1), u1, int(e["coarse"]),
               [sbrange(sb[0]), sbrange(sb[1])], True)


# -- src/laplacian.jl:100-108 (cylindrical, r = dim 1), :25-49 order of terms
def lap(u, blk, i, j, gi):
    wm = (2 * gi - 2) / (2 * gi - 1)
    wp = (2 * gi) / (2 * gi - 1)
    v = 0.0
    v += 1 * at(u, blk, i, j - 1)
    v += wm * at(u, blk, i - 1, j)
    v += -4 * at(u, blk, i, j)
    v += wp * at(u, blk, i + 1, j)
    v += 1 * at(u, blk, i, j + 1)
    return v


# -- src/multigrid.jl:153-180, 238-243
def gs_level(u, b, omega, s, tree, l, P):
    for (c, blk) in tree[l - 1].pairs:
        g0 = M * (c[0] - 1) + 1
        for i2 in range(G + 1, G + M + 1):
            for i1 in range(G + 1, G + M + 1, 2):
                p = P ^ (i2 & 1)
                I1 = i1 + p
                gi = I1 - G + g0 - 1
                Lu = lap(u, blk, I1, i2, gi)
                v = fma(s, at(b, blk, I1, i2), Lu)
                put(u, blk, I1, i2, fma(-(omega / -4), v, at(u, blk, I1, i2)))


def gs_iter(u, b, omega, s, n, l, tree, conn, bc):
    for _ in range(n):
        gs_level(u, b, omega, s, tree, l, 0)
        fill_copy(u, conn.neighbor[l - 1])
        fill_bnd(u, conn.boundary[l - 1], bc)
        gs_level(u, b, omega, s, tree, l, 1)
        fill_copy(u, conn.neighbor[l - 1])
        fill_bnd(u, conn.boundary[l - 1], bc)


# -- src/multigrid.jl:309-354
def residual_level(r, u, b, s, tree, l):
    for (c, blk) in tree[l - 1].pairs:
        g0 = M * (c[0] - 1) + 1
        for I2 in range(G + 1, G + M + 1):
            for I1 in range(G + 1, G + M + 1):
                Lu = lap(u, blk, I1, I2, I1 - G + g0 - 1)
                put(r, blk, I1, I2, -(at(b, blk, I1, I2) + Lu / s))


# -- src/multigrid.jl:112-119, 331-344
def postrestrict(bf, u, r, s, tree, l, ch):
    coord = tree[l - 2].coord
    for e in ch:
        blk = int(e["coarse"])
        c = coord[blk]
        g0 = M * (c[0] - 1) + 1
        sb = [int(e["subblock"][0]), int(e["subblock"][1])]
        for I2 in sbrange(sb[1]):
            for I1 in sbrange(sb[0]):
                Lu = lap(u, blk, I1, I2, I1 - G + g0 - 1)
                put(bf, blk, I1, I2, -(at(r, blk, I1, I2) + Lu / s))


def copyto(dst, src, tree, l):
    for (_, blk) in tree[l - 1].pairs:
        dst[blk - 1] = src[blk - 1]


def diffto(dst, a1, a2, tree, l):
    for (_, blk) in tree[l - 1].pairs:
        dst[blk - 1] = a1[blk - 1] - a2[blk - 1]


# -- src/multigrid.jl:60-106
def vcycle(u, b, r, u1, s, tree, conn, bc, ndown, ntop, nup, omega=1.0):
    lmax = len(tree)
    for l in range(lmax, 1, -1):
        sl = s / (1 << (l - 1)) ** 2
        gs_iter(u, b, omega, sl, ndown, l, tree, conn, bc)
        restrict(u, conn.child[l - 1])
        fill_ghost(u, conn, l - 1, bc)
        copyto(u1, u, tree, l - 1)
        residual_level(r, u, b, sl, tree, l)
        fill_ghost(r, conn, l, bc)
        restrict(r, conn.child[l - 1])
        fill_ghost(r, conn, l - 1, bc)
        postrestrict(b, u, r, 4 * sl, tree, l, conn.child[l - 1])
    gs_iter(u, b, omega, s, ntop, 1, tree, conn, bc)
    for l in range(2, lmax + 1):
        sl = s / (1 << (l - 1)) ** 2
        diffto(u1, u, u1, tree, l - 1)
        fill_ghost(u1, conn, l - 1, bc)
        interp_add(u, u1, conn.child[l - 1])
        fill_ghost(u, conn, l, bc)
        gs_iter(u, b, omega, sl, nup, l, tree, conn, bc)
        fill_ghost(u, conn, l, bc)


def tiny_tree():
    """Root block, level 2 full, two level-3 refinements (with the nesting they force)."""
    t = Tree((1, 1), 3)
    populate(t, 2)
    refine_block(t, 2, (1, 2))
    refine_block(t, 2, (2, 2))
    t.sync()
    return t


def main():
    rng = np.random.default_rng(20261203)
    tree = tiny_tree()
    conn = connectivity(tree)
    nblk = tree.nblocks_created
    bc = boundaryconditions(((1, -1), (-1, 1)))
    u0 = rng.standard_normal((nblk, S, S))
    b0 = rng.standard_normal((nblk, S, S))
    out = {"u0": u0, "b0": b0, "bc": bc}
    # per-operation outputs
    for l in (1, 2, 3):
        u = u0.copy()
        fill_ghost(u, conn, l, bc)
        out[f"fill_ghost_l{l}"] = u
    u = u0.copy()
    restrict(u, conn.child[2])
    out["restrict_l3"] = u
    u = u0.copy()
    interp_add(u, b0, conn.child[2])
    out["interp_add_l3"] = u
    u = u0.copy()
    gs_iter(u, b0, 1.0, 0.37, 2, 3, tree, conn, bc)
    out["gs_iter_l3"] = u
    r = np.zeros_like(u0)
    residual_level(r, u0, b0, 0.37, tree, 3)
    out["residual_l3"] = r
    # one full V-cycle (2,2,4) from filled ghosts
    u, b, r, u1 = u0.copy(), b0.copy(), np.zeros_like(u0), np.zeros_like(u0)
    for l in (1, 2, 3):
        fill_ghost(u, conn, l, bc)
    out["vcycle_u_in"] = u.copy()
    vcycle(u, b, r, u1, 0.5, tree, conn, bc, 2, 4, 2)
    out["vcycle_u"] = u
    out["vcycle_b"] = b
    np.savez_compressed(os.path.join(HERE, "mg_tiny.npz"), **out)
    print("wrote", os.path.join(HERE, "mg_tiny.npz"), {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
