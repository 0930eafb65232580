"""Host-side mirror of Steamroller.jl's block-tree types and connectivity builder.

The drop-in boundary receives exactly these structures from Julia: per-level block
lists (``BlockLayer.pairs``) and the four edge lists of ``Connectivity``.  This module
rebuilds them in Python so that tests and benchmarks can drive the C ABI the way the
Julia shim does.  Layouts are the isbits layouts of the Julia structs; indices are
1-based, as in Julia.

Reference:
  * ``BlockLayer`` / ``sync!``            src/blocklayer.jl:9-24, 48-53
  * ``Tree`` / ``populate!`` / ``isleaf`` src/tree.jl:6-44, 105-115
  * ``parentcoord`` / ``subcoord``         src/mesh.jl:48-61
  * edge structs / ``connectivity!``      src/connectivity.jl:6-42, 106-149
  * ``StarStencil`` / ``BoxStencil`` order src/stencil.jl:16-55
"""
from __future__ import annotations

import numpy as np

# Pair{CartesianIndex{2}, Int}: 24 bytes (src/blocklayer.jl:23)
PAIR_DTYPE = np.dtype([("coord", "<i8", (2,)), ("blk", "<i8")])
# Neighbor{2}(from, to, face): 32 bytes (src/connectivity.jl:14-20)
NEIGHBOR_DTYPE = np.dtype([("from", "<i8"), ("to", "<i8"), ("face", "<i8", (2,))])
# Boundary{2}(block, face, bnd, level): 48 bytes (src/connectivity.jl:6-11)
BOUNDARY_DTYPE = np.dtype([("block", "<i8"), ("face", "<i8", (2,)), ("bnd", "<i8", (2,)),
                           ("level", "<i8")])
# RefBoundary{2}(fine, coarse, face, subblock): 48 bytes (src/connectivity.jl:23-32)
REFBND_DTYPE = np.dtype([("fine", "<i8"), ("coarse", "<i8"), ("face", "<i8", (2,)),
                         ("subblock", "<i8", (2,))])
# Child{2}(fine, coarse, subblock): 32 bytes (src/connectivity.jl:36-42)
CHILD_DTYPE = np.dtype([("fine", "<i8"), ("coarse", "<i8"), ("subblock", "<i8", (2,))])

# StarStencil{2} iteration order: (-1,0), (1,0), (0,-1), (0,1)  (src/stencil.jl:16-32)
STAR2 = ((-1, 0), (1, 0), (0, -1), (0, 1))
# BoxStencil{2} iteration order (src/stencil.jl:34-55, __incbox :72-90): dimension 1
# fastest from (-1,-1), the origin skipped
BOX2 = ((-1, -1), (0, -1), (1, -1), (-1, 0), (1, 0), (-1, 1), (0, 1), (1, 1))


class BlockLayer:
    """One level of the tree: coordinate <-> block maps plus the ``pairs`` list.

    ``domain`` is the level's extent in blocks, ``(n1, n2)``: coordinates run over
    ``1..n1`` x ``1..n2`` (``multiplyindices``, src/blocklayer.jl:111-115).
    """

    def __init__(self, level: int, domain: tuple[int, int]):
        self.level = level
        self.domain = domain
        self.index: dict[tuple[int, int], int] = {}
        self.coord: dict[int, tuple[int, int]] = {}
        self.pairs: list[tuple[tuple[int, int], int]] = []

    def __len__(self):
        return len(self.pairs)

    def __contains__(self, c):
        return c in self.index

    def in_domain(self, c) -> bool:
        return 1 <= c[0] <= self.domain[0] and 1 <= c[1] <= self.domain[1]

    def get(self, c, default=0) -> int:
        return self.index.get(c, default)

    def add(self, c, blk):
        self.index[c] = blk
        self.coord[blk] = c

    def sync(self, order=None):
        """Rebuild ``pairs`` (src/blocklayer.jl:48-53).  Julia's order is Dict order,
        i.e. unspecified; ``order`` may be an RNG to shuffle it."""
        self.pairs = list(self.index.items())
        if order is not None:
            perm = order.permutation(len(self.pairs))
            self.pairs = [self.pairs[i] for i in perm]

    def pairs_array(self) -> np.ndarray:
        a = np.zeros(len(self.pairs), dtype=PAIR_DTYPE)
        if self.pairs:
            a["coord"] = np.array([c for c, _ in self.pairs], dtype=np.int64)
            a["blk"] = np.array([b for _, b in self.pairs], dtype=np.int64)
        return a


class Tree(list):
    """``Tree{D} = Vector{BlockLayer{D}}`` (src/tree.jl:6-15)."""

    def __init__(self, rootsize=(1, 1), levels=16):
        super().__init__(BlockLayer(l, (rootsize[0] << (l - 1), rootsize[1] << (l - 1)))
                         for l in range(1, levels + 1))
        self.rootsize = tuple(rootsize)
        self.nblocks_created = 0

    def nblocks(self) -> int:
        return sum(len(layer.index) for layer in self)

    def finest_level(self) -> int:
        return max((l.level for l in self if l.index), default=0)

    def sync(self, rng=None):
        for layer in self:
            layer.sync(rng)

    def new_block(self) -> int:
        self.nblocks_created += 1
        return self.nblocks_created

    def isleaf(self, lvl: int, c) -> bool:
        """``isleaf`` (src/tree.jl:105-115)."""
        if lvl >= len(self):
            return True
        nxt = self[lvl]  # level lvl+1
        i, j = c
        for cc in ((2 * i - 1, 2 * j - 1), (2 * i, 2 * j - 1), (2 * i - 1, 2 * j), (2 * i, 2 * j)):
            if cc in nxt.index:
                return False
        return True


def parentcoord(c):
    """``parentcoord`` (src/mesh.jl:48-50)."""
    return ((c[0] - 1) // 2 + 1, (c[1] - 1) // 2 + 1)


def subcoord(c):
    """``subcoord`` (src/mesh.jl:59-61)."""
    return ((c[0] - 1) % 2 + 1, (c[1] - 1) % 2 + 1)


def subblocks(c):
    """Children coordinates in CartesianIndices order (dim 1 fastest), src/mesh.jl:40-42."""
    i, j = c
    return [(2 * i - 1, 2 * j - 1), (2 * i, 2 * j - 1), (2 * i - 1, 2 * j), (2 * i, 2 * j)]


def populate(tree: Tree, level: int) -> int:
    """``populate!`` (src/tree.jl:31-44): every block of levels 1..level, numbered
    level by level in CartesianIndices order."""
    for l in range(1, level + 1):
        layer = tree[l - 1]
        for j in range(1, layer.domain[1] + 1):
            for i in range(1, layer.domain[0] + 1):
                layer.add((i, j), tree.new_block())
    tree.sync()
    return tree.nblocks_created


def refine_block(tree: Tree, l: int, c, stencil=STAR2) -> None:
    """Refine leaf block ``c`` of level ``l`` keeping proper nesting: every in-domain
    neighbour of ``c`` along ``stencil`` must exist at level ``l`` first, so that the
    children's missing neighbours always have a parent (the invariant asserted by
    src/connectivity.jl:129,141 and maintained by ensure_proper_refine!,
    src/refinement.jl:286-311).  The reference refines with a BoxStencil
    (src/streamer.jl:437); ``BOX2`` reproduces that nesting, which a BoxStencil
    connectivity needs."""
    if l >= len(tree):
        raise ValueError("cannot refine beyond the tree's maximum level")
    layer = tree[l - 1]
    if c not in layer.index:
        raise KeyError(c)
    if not tree.isleaf(l, c):
        return
    for s in stencil:
        n = (c[0] + s[0], c[1] + s[1])
        if layer.in_domain(n) and n not in layer.index:
            refine_block(tree, l - 1, parentcoord(n), stencil)
    nxt = tree[l]
    for cc in subblocks(c):
        if cc not in nxt.index:
            nxt.add(cc, tree.new_block())


class Connectivity:
    """Per-level edge lists (src/connectivity.jl:51-64), as numpy structured arrays."""

    def __init__(self, boundary, neighbor, refboundary, child):
        self.boundary = boundary
        self.neighbor = neighbor
        self.refboundary = refboundary
        self.child = child


def connectivity(tree: Tree, stencil=STAR2) -> Connectivity:
    """``connectivity!`` (src/connectivity.jl:106-149) with a StarStencil (``STAR2``,
    order-2 discretisations) or a BoxStencil (``BOX2``, the order-4 compact
    discretisation, src/simulate.jl:260-262), whose diagonal edges fill the 2 x 2
    corner ghosts.  A diagonal step out of the domain along one dimension only gives a
    Boundary whose ``bnd`` is zero along the other (src/connectivity.jl:112-115)."""
    nlev = len(tree)
    bd, nb, rb, ch = ([[] for _ in range(nlev)] for _ in range(4))
    for layer in tree:
        lv = layer.level
        for c, blk in layer.pairs:
            for s in stencil:
                n = (c[0] + s[0], c[1] + s[1])
                if not layer.in_domain(n):
                    bnd = tuple(0 if 1 <= n[d] <= layer.domain[d] else s[d] for d in range(2))
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

    return Connectivity(
        [arr(x, BOUNDARY_DTYPE, ("block", "face", "bnd", "level")) for x in bd],
        [arr(x, NEIGHBOR_DTYPE, ("from", "to", "face")) for x in nb],
        [arr(x, REFBND_DTYPE, ("fine", "coarse", "face", "subblock")) for x in rb],
        [arr(x, CHILD_DTYPE, ("fine", "coarse", "subblock")) for x in ch],
    )


def boundaryconditions(desc) -> np.ndarray:
    """``boundaryconditions`` (src/boundary.jl:28-38): the 3x3 Int8 sign table,
    returned flattened in Julia's column-major order (a[i, j] at (i-1) + 3(j-1))."""
    a = np.ones((3, 3), dtype=np.int8)
    for i, (lo, hi) in enumerate(desc):
        if i == 0:
            a[0, :] *= lo
            a[2, :] *= hi
        else:
            a[:, 0] *= lo
            a[:, 2] *= hi
    return np.ascontiguousarray(a.T).reshape(9)  # column-major flattening


def level_cells(tree: Tree, M: int = 16) -> list[int]:
    """Valid cells per level (all blocks of the level, leaves and parents)."""
    return [len(layer.index) * M * M for layer in tree]


def leaf_cells(tree: Tree, M: int = 16) -> int:
    n = 0
    for layer in tree:
        for c in layer.index:
            if tree.isleaf(layer.level, c):
                n += M * M
    return n
