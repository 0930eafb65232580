"""Host-side mirror of Steamroller.jl's block tree and connectivity in three dimensions
(D = 3): ``BlockLayer{3}``, ``Tree{3}``, ``populate!``, nesting-preserving refinement and
``connectivity!`` with a StarStencil{3} or BoxStencil{3}.  Layouts are the isbits
layouts of the Julia structs for D = 3; indices are 1-based.

Reference (dimension-generic code, written out for D = 3):
  * ``BlockLayer`` / ``Tree`` / ``populate!``   src/blocklayer.jl:9-53, src/tree.jl:6-44
  * ``parentcoord`` / ``subcoord``              src/mesh.jl:48-61
  * edge structs / ``connectivity!``           src/connectivity.jl:6-42, 106-149
  * Star/Box stencil iteration orders          src/stencil.jl:16-90
"""
from __future__ import annotations

import itertools

import numpy as np

PAIR3_DTYPE = np.dtype([("coord", "<i8", (3,)), ("blk", "<i8")])
NEIGHBOR3_DTYPE = np.dtype([("from", "<i8"), ("to", "<i8"), ("face", "<i8", (3,))])
BOUNDARY3_DTYPE = np.dtype([("block", "<i8"), ("face", "<i8", (3,)), ("bnd", "<i8", (3,)), ("level", "<i8")])
REFBND3_DTYPE = np.dtype([("fine", "<i8"), ("coarse", "<i8"), ("face", "<i8", (3,)), ("subblock", "<i8", (3,))])
CHILD3_DTYPE = np.dtype([("fine", "<i8"), ("coarse", "<i8"), ("subblock", "<i8", (3,))])

# StarStencil{3}: -e1, +e1, -e2, +e2, -e3, +e3 (src/stencil.jl:16-32)
STAR3 = ((-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1))
# BoxStencil{3}: every offset in {-1,0,1}^3 but the origin, dimension 1 fastest (__incbox)
BOX3 = tuple((a, b, c) for c, b, a in itertools.product((-1, 0, 1), repeat=3) if (a, b, c) != (0, 0, 0))


class BlockLayer3:
    def __init__(self, level: int, domain):
        self.level = level
        self.domain = tuple(domain)
        self.index: dict[tuple, int] = {}
        self.coord: dict[int, tuple] = {}
        self.pairs: list = []

    def __len__(self):
        return len(self.pairs)

    def in_domain(self, c) -> bool:
        return all(1 <= c[d] <= self.domain[d] for d in range(3))

    def add(self, c, blk):
        self.index[c] = blk
        self.coord[blk] = c

    def sync(self, order=None):
        self.pairs = list(self.index.items())
        if order is not None:
            perm = order.permutation(len(self.pairs))
            self.pairs = [self.pairs[i] for i in perm]

    def pairs_array(self) -> np.ndarray:
        a = np.zeros(len(self.pairs), dtype=PAIR3_DTYPE)
        if self.pairs:
            a["coord"] = np.array([c for c, _ in self.pairs], dtype=np.int64)
            a["blk"] = np.array([b for _, b in self.pairs], dtype=np.int64)
        return a


def parentcoord(c):
    return tuple((x - 1) // 2 + 1 for x in c)


def subcoord(c):
    return tuple((x - 1) % 2 + 1 for x in c)


def subblocks(c):
    """Children in CartesianIndices order (dimension 1 fastest)."""
    return [(2 * c[0] - 1 + a, 2 * c[1] - 1 + b, 2 * c[2] - 1 + d)
            for d in (0, 1) for b in (0, 1) for a in (0, 1)]


class Tree3(list):
    """``Tree{3}`` (src/tree.jl:6-15)."""

    D = 3

    def __init__(self, rootsize=(1, 1, 1), levels=8):
        super().__init__(BlockLayer3(l, tuple(r << (l - 1) for r in rootsize)) for l in range(1, levels + 1))
        self.rootsize = tuple(rootsize)
        self.nblocks_created = 0

    def nblocks(self) -> int:
        return sum(len(layer.index) for layer in self)

    def sync(self, rng=None):
        for layer in self:
            layer.sync(rng)

    def new_block(self) -> int:
        self.nblocks_created += 1
        return self.nblocks_created

    def isleaf(self, lvl, c) -> bool:
        if lvl >= len(self):
            return True
        return not any(cc in self[lvl].index for cc in subblocks(c))


def populate(tree: Tree3, level: int) -> int:
    """``populate!`` (src/tree.jl:31-44): every block of levels 1..level, numbered level by
    level in CartesianIndices order."""
    for l in range(1, level + 1):
        layer = tree[l - 1]
        n1, n2, n3 = layer.domain
        for k in range(1, n3 + 1):
            for j in range(1, n2 + 1):
                for i in range(1, n1 + 1):
                    layer.add((i, j, k), tree.new_block())
    tree.sync()
    return tree.nblocks_created


def refine_block(tree: Tree3, l: int, c, stencil=BOX3) -> None:
    """Refine leaf block ``c`` of level ``l``, first making every in-domain neighbour of
    ``c`` along ``stencil`` exist (proper nesting, src/refinement.jl:286-311; the
    reference refines with a BoxStencil, src/streamer.jl:437)."""
    layer = tree[l - 1]
    if c not in layer.index:
        raise KeyError(c)
    if not tree.isleaf(l, c):
        return
    for s in stencil:
        n = tuple(c[d] + s[d] for d in range(3))
        if layer.in_domain(n) and n not in layer.index:
            refine_block(tree, l - 1, parentcoord(n), stencil)
    nxt = tree[l]
    for cc in subblocks(c):
        if cc not in nxt.index:
            nxt.add(cc, tree.new_block())


class Connectivity3:
    def __init__(self, boundary, neighbor, refboundary, child):
        self.boundary = boundary
        self.neighbor = neighbor
        self.refboundary = refboundary
        self.child = child


def connectivity(tree: Tree3, stencil=STAR3) -> Connectivity3:
    """``connectivity!`` (src/connectivity.jl:106-149) for D = 3."""
    nlev = len(tree)
    bd, nb, rb, ch = ([[] for _ in range(nlev)] for _ in range(4))
    for layer in tree:
        lv = layer.level
        for c, blk in layer.pairs:
            for s in stencil:
                n = tuple(c[d] + s[d] for d in range(3))
                if not layer.in_domain(n):
                    bnd = tuple(0 if 1 <= n[d] <= layer.domain[d] else s[d] for d in range(3))
                    bd[lv - 1].append((blk, s, bnd, lv))
                    continue
                other = layer.index.get(n, 0)
                if other != 0:
                    nb[lv - 1].append((blk, other, s))
                elif lv > 1:
                    pblk = tree[lv - 2].index.get(parentcoord(n), 0)
                    if pblk == 0:
                        raise ValueError(f"Proper nesting broken at level {lv}, {n}")
                    rb[lv - 1].append((blk, pblk, s, subcoord(n)))
            if lv > 1:
                pblk = tree[lv - 2].index.get(parentcoord(c), 0)
                if pblk == 0:
                    raise ValueError("Malformed tree")
                ch[lv - 1].append((blk, pblk, subcoord(c)))

    def arr(rows, dtype, fields):
        a = np.zeros(len(rows), dtype=dtype)
        for k, name in enumerate(fields):
            if rows:
                a[name] = np.array([r[k] for r in rows], dtype=np.int64)
        return a

    return Connectivity3(
        [arr(x, BOUNDARY3_DTYPE, ("block", "face", "bnd", "level")) for x in bd],
        [arr(x, NEIGHBOR3_DTYPE, ("from", "to", "face")) for x in nb],
        [arr(x, REFBND3_DTYPE, ("fine", "coarse", "face", "subblock")) for x in rb],
        [arr(x, CHILD3_DTYPE, ("fine", "coarse", "subblock")) for x in ch],
    )


def boundaryconditions(desc) -> np.ndarray:
    """``boundaryconditions`` (src/boundary.jl:28-38) for D = 3: the 3x3x3 Int8 table,
    flattened column-major (a[i, j, k] at (i-1) + 3(j-1) + 9(k-1))."""
    a = np.ones((3, 3, 3), dtype=np.int8)
    for i, (lo, hi) in enumerate(desc):
        sl_lo = [slice(None)] * 3
        sl_hi = [slice(None)] * 3
        sl_lo[i] = slice(0, 1)
        sl_hi[i] = slice(2, 3)
        a[tuple(sl_lo)] *= lo
        a[tuple(sl_hi)] *= hi
    return np.ascontiguousarray(a.transpose(2, 1, 0)).reshape(27)


def block_cell_centres(tree: Tree3, level: int, h1: float):
    """Blocks of a level and the (x, y, z) of their valid cells, [blk][k][j][i] order."""
    layer = tree[level - 1]
    blks = np.array([b for _, b in layer.pairs], dtype=np.int64)
    h = h1 / 2 ** (level - 1)
    if len(blks) == 0:
        return blks, np.zeros((0, 16, 16, 16)), np.zeros((0, 16, 16, 16)), np.zeros((0, 16, 16, 16))
    coords = np.array([c for c, _ in layer.pairs], dtype=np.int64)
    idx = np.arange(16)
    x = ((coords[:, 0, None] - 1) * 16 + idx[None, :] + 0.5) * h
    y = ((coords[:, 1, None] - 1) * 16 + idx[None, :] + 0.5) * h
    z = ((coords[:, 2, None] - 1) * 16 + idx[None, :] + 0.5) * h
    X = np.broadcast_to(x[:, None, None, :], (len(blks), 16, 16, 16))
    Y = np.broadcast_to(y[:, None, :, None], (len(blks), 16, 16, 16))
    Z = np.broadcast_to(z[:, :, None, None], (len(blks), 16, 16, 16))
    return blks, X, Y, Z
