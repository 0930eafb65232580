"""Free boundary conditions (FreeBC, src/freebc.jl) restated in numpy: the checker for
libsrmg's srmg_freebc / srmg_fill_ghost_free.

TEST INFRASTRUCTURE ONLY (the oracle): imported by tests/ and nowhere in the product.

Parity: unpinned (the reference ships no tests for this path and cannot run here); the
restatement is pinned by its own known-answer tests (the transform pair inverts, and
the free-space boundary moves the potential at r = R towards the one of a much larger
domain).

The reference's transforms are FFTW's RODFT10 (DST-II) and RODFT01 (DST-III),
unnormalised; scipy.fft.dst types 2 and 3 with norm=None have the same definitions.
The kernel f uses the modified Bessel functions I_0, I_1, K_0, K_1 through their
exponentially scaled forms (ratios are unchanged by the scaling), as FreeBC does with
besselix / besselkx (src/freebc.jl:39-41).
"""
from __future__ import annotations

import numpy as np
import scipy.fft
import scipy.special

M, G = 16, 2


def other(dim: int) -> int:
    """mod1(dim + 1, 2) for D = 2."""
    return 2 if dim == 1 else 1


def kernel(dim: int, level: int, rootsize, h: float):
    """FreeBC(geom, u, level, rootsize, h) fields (src/freebc.jl:29-53): n, H, R, f."""
    od = other(dim)
    n = rootsize[od - 1] * 2 ** (level - 1) * M
    H = rootsize[od - 1] * h * M
    R = rootsize[dim - 1] * h * M
    k = (np.pi / H) * np.arange(1, n + 1)
    x = k * R
    f = (2 / H) / (k * (scipy.special.i1e(x) / scipy.special.i0e(x) + scipy.special.k1e(x) / scipy.special.k0e(x)))
    return n, H, R, f


def _coord(tree, l, blk):
    return tree[l - 1].coord[blk]


def _cell(dim, along_dim, along_other):
    """0-based [blk, j, i] index tuple (j along dimension 2, i along dimension 1)."""
    return (along_other, along_dim) if dim == 1 else (along_dim, along_other)


def getouter(u, tree, dim, level, h, n):
    """getouter!(u1, u, tree, dim, level, h) (src/freebc.jl:108-140): the outermost
    valid cells along `dim` of every block on the outer boundary, divided by h_l,
    repeated p = 2^(level-l) times; finer levels overwrite."""
    u1 = np.zeros(n)
    od = other(dim)
    for l in range(1, min(level, len(tree)) + 1):
        layer = tree[l - 1]
        k = layer.domain[dim - 1]
        hl = h / 2 ** (l - 1)
        p = 2 ** (level - l)
        for c, blk in layer.pairs:
            if c[dim - 1] != k:
                continue
            i0 = (c[od - 1] - 1) * M
            for i in range(1, M + 1):
                j, ii = _cell(dim, G + M - 1, G + i - 1)
                u1[p * (i0 + i - 1): p * (i0 + i)] = u[blk - 1, j, ii] / hl
    return u1


def transform(u1, f, h, level):
    """The middle of freebc! (src/freebc.jl:93-102): DST-II, times f, DST-III, scaled.
    (`am[end] *= 3` there is overwritten by the next line and has no effect.)"""
    u1 = scipy.fft.dst(u1, type=2)
    am = f * u1
    am = scipy.fft.dst(am, type=3)
    return am * h / 2 ** (level - 1) / 2


def factor(J):
    """factor(CylindricalGeometry{D}, c, delta) with delta along D (src/geometry.jl:27-29)."""
    return abs(1 + 1 / (2 * J - 1))


def setouter(q, b, tree, conn, dim, level, s):
    """setouter!(q, b, tree, conn, dim, level, s, geom) (src/freebc.jl:147-221), in place."""
    od = other(dim)
    face0 = (1, 0) if dim == 1 else (0, 1)
    for l in range(1, min(level, len(tree)) + 1):
        layer = tree[l - 1]
        sl = s / (1 << (l - 1)) ** 2
        p = 2 ** (level - l)
        k = layer.domain[dim - 1]
        for e in conn.boundary[l - 1]:
            if tuple(int(x) for x in e["face"]) != face0:
                continue
            blk = int(e["block"])
            B = _coord(tree, l, blk)
            i0 = (B[od - 1] - 1) * M
            for i in range(1, M + 1):
                Jd = M * (B[dim - 1] - 1) + M
                bmean = _seqsum(b[p * (i0 + i - 1): p * (i0 + i)]) / p
                j, ii = _cell(dim, G + M - 1, G + i - 1)
                q[blk - 1, j, ii] += 2 * factor(Jd) * bmean / sl
        for e in conn.refboundary[l - 1]:
            blk = int(e["fine"])
            B = _coord(tree, l, blk)
            if B[dim - 1] != k:
                continue
            d = int(e["face"][od - 1])
            i = G + 1 if d == -1 else M + G
            jg = (B[od - 1] - 1) * M + i - G
            Jd = M * (B[dim - 1] - 1) + M
            J1d = (Jd - 1) // 2 + 1
            if d == 1:
                seg = b[p * jg: p * (jg + 2)]
            else:
                # b[p (j - 3) : p (j - 1) - 1] in 1-based indices, as written
                seg = b[p * (jg - 3) - 1: p * (jg - 1) - 1]
            bmean = _seqsum(seg) / (2 * p)
            jj, ii = _cell(dim, G + M - 1, i - 1)
            q[blk - 1, jj, ii] += 2 * 0.25 * factor(J1d) * bmean / sl


def fill_ghost_free(u, b, tree, dim, level, l):
    """fill_ghost_free!(u, conf, tree, l) (src/freebc.jl:224-243), in place: the first
    ghost layer beyond the outer boundary gains 2 bmean."""
    od = other(dim)
    layer = tree[l - 1]
    k = layer.domain[dim - 1]
    p = 2 ** (level - l)
    for c, blk in layer.pairs:
        if c[dim - 1] != k:
            continue
        i0 = (c[od - 1] - 1) * M
        for i in range(1, M + 1):
            bmean = _seqsum(b[p * (i0 + i - 1): p * (i0 + i)]) / p
            j, ii = _cell(dim, G + M, G + i - 1)
            u[blk - 1, j, ii] += 2 * bmean


def freebc(q, u, h, s, tree, conn, dim, level, f):
    """freebc!(q, u, h, s, tree, conn, conf) (src/freebc.jl:83-105): returns b; q in place."""
    n = len(f)
    u1 = getouter(u, tree, dim, level, h, n)
    b = transform(u1, f, h, level)
    setouter(q, b, tree, conn, dim, level, s)
    return b


def _seqsum(a):
    v = 0.0
    for x in a:
        v += float(x)
    return v
