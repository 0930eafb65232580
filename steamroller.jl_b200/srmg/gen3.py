"""Seeded three-dimensional field-solve problems (D = 3, CartesianGeometry, the only
geometry the reference defines 3D stencils for: src/laplacian.jl:274-340,
src/helmholtz.jl:74-100).  Fields are [nblk, 20, 20, 20] float64 arrays indexed
[blk, k, j, i], i.e. Julia's (i, j, k, blk)."""
from __future__ import annotations

import dataclasses

import numpy as np

from .tree3 import (Tree3, Connectivity3, STAR3, BOX3, boundaryconditions, block_cell_centres, connectivity,
                    populate, refine_block)

S3 = 20


@dataclasses.dataclass
class Problem3:
    tree: Tree3
    conn: Connectivity3
    b: np.ndarray
    s: float
    op: int = 0
    k2: float = 0.0
    bc: np.ndarray = dataclasses.field(default_factory=lambda: boundaryconditions(((-1, -1),) * 3))
    h1: float = 1.0 / 16
    geom: int = 0
    name: str = ""

    @property
    def nblk(self) -> int:
        return self.b.shape[0]


def restrict_full3(b, tree, conn):
    """restrict_full! (src/restrict.jl:43-47) in numpy: coarse = (sum of 8 fine) / 8."""
    for l in range(len(tree), 1, -1):
        for e in conn.child[l - 1]:
            f, c = int(e["fine"]), int(e["coarse"])
            sb = [int(x) for x in e["subblock"]]
            src = b[f - 1, 2:18, 2:18, 2:18]
            acc = np.zeros((8, 8, 8))
            for i3 in (0, 1):
                for i2 in (0, 1):
                    for i1 in (0, 1):
                        acc = acc + src[i3::2, i2::2, i1::2]
            z0, y0, x0 = (2 + 8 * (sb[2] - 1), 2 + 8 * (sb[1] - 1), 2 + 8 * (sb[0] - 1))
            b[c - 1, z0:z0 + 8, y0:y0 + 8, x0:x0 + 8] = acc / 8


def make_problem3(tree, conn, rhs_fn, s, op=0, k2=0.0, bc=None, h1=1.0 / 16, name=""):
    b = np.zeros((tree.nblocks_created, S3, S3, S3))
    for l in range(1, len(tree) + 1):
        blks, x, y, z = block_cell_centres(tree, l, h1)
        if len(blks):
            b[blks - 1, 2:18, 2:18, 2:18] = rhs_fn(x, y, z)
    restrict_full3(b, tree, conn)
    return Problem3(tree=tree, conn=conn, b=b, s=s, op=op, k2=k2,
                    bc=boundaryconditions(((-1, -1),) * 3) if bc is None else bc, h1=h1, name=name)


def refined3(seed: int = 1, op: int = 0, k2: float = 0.0, stencil=None, levels=4) -> Problem3:
    """Uniform to level 2 (8 blocks), then seeded refinement of a few blocks to levels 3
    and 4 with BoxStencil nesting; a Gaussian charge near the refined corner."""
    rng = np.random.default_rng(seed)
    st = stencil if stencil is not None else (BOX3 if op == 2 else STAR3)
    t = Tree3((1, 1, 1), levels)
    populate(t, 2)
    c2 = tuple(int(x) for x in rng.integers(1, 3, size=3))
    refine_block(t, 2, c2, BOX3)
    kids = [c for c in t[2].index if tuple((x - 1) // 2 + 1 for x in c) == c2]
    refine_block(t, 3, kids[int(rng.integers(len(kids)))], BOX3)
    t.sync()
    conn = connectivity(t, st)
    centre = (np.array(c2) - 0.5) / 2.0
    w = 0.15

    def rhs(x, y, z):
        return np.exp(-((x - centre[0]) ** 2 + (y - centre[1]) ** 2 + (z - centre[2]) ** 2) / w ** 2)

    h1 = 1.0 / 16
    return make_problem3(t, conn, rhs, h1 * h1, op=op, k2=k2, h1=h1, name=f"refined3-op{op}")
