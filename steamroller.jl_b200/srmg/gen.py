"""Seeded synthetic field-solve problems: trees, right-hand sides and operators.

The reference publishes no benchmark data, so every workload here is synthetic and
seeded.  Shapes follow the reference's own defaults: rootsize (1,1)
(src/simulate.jl:27), L = 1.25e-2 m and M = 16, G = 2 (src/simulate.jl:235-238,
samples/bagheri.in.jl:42), CylindricalGeometry{1} (src/simulate.jl:257), order-2
stencils, s = h^2 e/eps0 for Poisson (src/streamer.jl:328,331) and s = h^2 for the
photoionization Helmholtz terms (src/photo.jl:55).

Refined trees are grown around seeded conducting channels.  The refinement
indicator is a field-magnitude proxy |E|(x) = E0 + sum_seg V/max(dist(x, seg), r_c)
* (1 + 2 exp(-dist(x, tip)/(5 r_c))) -- the 1/distance fall-off of a charged line
with a tip enhancement -- and the threshold is bisected until the tree holds the
requested number of leaf cells.  Right-hand sides are net charge n_ion - n_e of the
channel (Gaussian profile, log-uniform per-cell noise), restricted onto parent
blocks the way derivs! does (restrict_full!, src/streamer.jl:313).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .tree import (Tree, Connectivity, boundaryconditions, connectivity, populate,
                   refine_block, leaf_cells, STAR2, BOX2)

ELEMENTARY_CHARGE = 1.6021766208e-19   # src/constants.jl:55
EPSILON_0 = 8.854187817620389e-12      # src/constants.jl:56
L_DOMAIN = 1.25e-2                     # samples/bagheri.in.jl:42
M_BLOCK = 16
G_GHOST = 2
S_BLOCK = M_BLOCK + 2 * G_GHOST

OP_LAPLACIAN, OP_HELMHOLTZ, OP_LAPLACIAN4 = 0, 1, 2
GEOM_CART, GEOM_CYL1, GEOM_CYL2 = 0, 1, 2

# Poisson BCs for the benchmark: Neumann on the axis and outer radius, Dirichlet at the
# z electrodes; the photoionization BC of src/photo.jl:108-110 is the same table.
BC_POISSON = boundaryconditions(((1, 1), (-1, -1)))
BC_REFERENCE_DEFAULT = boundaryconditions(((1, -1), (-1, -1)))  # src/simulate.jl:245-246
BC_PHOTO = boundaryconditions(((1, 1), (-1, -1)))


@dataclasses.dataclass
class Problem:
    """One field solve: L u + s b = 0 on a tree (multigrid.jl:6-16)."""
    tree: Tree
    conn: Connectivity
    b: np.ndarray            # (nblk, S, S) float64, [blk, j, i] == Julia (i, j, blk)
    s: float
    op: int = OP_LAPLACIAN
    k2: float = 0.0
    geom: int = GEOM_CYL1
    bc: np.ndarray = dataclasses.field(default_factory=lambda: BC_POISSON.copy())
    h1: float = L_DOMAIN / M_BLOCK
    name: str = ""

    @property
    def nblk(self) -> int:
        return self.b.shape[0]

    def zeros(self) -> np.ndarray:
        return np.zeros_like(self.b)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """Vectorised splitmix64 finaliser (uint64 in, uint64 out)."""
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)).astype(np.uint64)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def cell_hash01(seed: int, level: int, gi: np.ndarray, gj: np.ndarray) -> np.ndarray:
    """Deterministic U[0,1) per global cell, independent of block numbering."""
    with np.errstate(over="ignore"):
        key = (np.uint64(seed) * np.uint64(0x100000001B3)
               ^ (np.uint64(level) << np.uint64(58))
               ^ (gi.astype(np.uint64) << np.uint64(29)) ^ gj.astype(np.uint64))
    return (splitmix64(key) >> np.uint64(11)).astype(np.float64) / float(1 << 53)


def block_cell_centres(tree: Tree, level: int, h1: float):
    """(blk[n], r[n,16,16], z[n,16,16], gi, gj) for every block of a level; arrays
    are indexed [block, j, i] (cell_centers, src/mesh.jl:111-116)."""
    layer = tree[level - 1]
    if not layer.index:
        e = np.zeros((0, M_BLOCK, M_BLOCK))
        return np.zeros(0, np.int64), e, e, e.astype(np.int64), e.astype(np.int64)
    coords = np.array(list(layer.index.keys()), dtype=np.int64)
    blks = np.array(list(layer.index.values()), dtype=np.int64)
    hl = h1 / (1 << (level - 1))
    k = np.arange(1, M_BLOCK + 1, dtype=np.int64)
    gi = M_BLOCK * (coords[:, 0, None, None] - 1) + k[None, None, :]
    gj = M_BLOCK * (coords[:, 1, None, None] - 1) + k[None, :, None]
    gi = np.broadcast_to(gi, (len(blks), M_BLOCK, M_BLOCK))
    gj = np.broadcast_to(gj, (len(blks), M_BLOCK, M_BLOCK))
    return blks, (gi - 0.5) * hl, (gj - 0.5) * hl, gi, gj


def restrict_full_np(f: np.ndarray, tree: Tree, conn: Connectivity) -> None:
    """restrict_full! (src/restrict.jl:43-47) in numpy: parents' covered subblocks
    become the 2x2 average of their children's valid cells (same summation order)."""
    G, M, mh = G_GHOST, M_BLOCK, M_BLOCK // 2
    for l in range(len(tree), 1, -1):
        ch = conn.child[l - 1]
        if len(ch) == 0:
            continue
        fine = ch["fine"] - 1
        v = f[fine, G:G + M, G:G + M]
        acc = 0.0 + v[:, 0::2, 0::2]
        acc = acc + v[:, 0::2, 1::2]
        acc = acc + v[:, 1::2, 0::2]
        acc = acc + v[:, 1::2, 1::2]
        acc = acc / 4
        for q in range(len(ch)):
            sb = ch["subblock"][q]
            i0 = G + (sb[0] - 1) * mh
            j0 = G + (sb[1] - 1) * mh
            f[ch["coarse"][q] - 1, j0:j0 + mh, i0:i0 + mh] = acc[q]


@dataclasses.dataclass
class Channel:
    """A straight conducting segment in the (r, z) plane."""
    r0: float
    z0: float
    r1: float
    z1: float          # (r1, z1) is the tip
    radius: float
    density: float
    volt: float


def _seg_dist(r, z, ch: Channel):
    dr, dz = ch.r1 - ch.r0, ch.z1 - ch.z0
    ll = dr * dr + dz * dz
    t = np.clip(((r - ch.r0) * dr + (z - ch.z0) * dz) / ll, 0.0, 1.0)
    pr, pz = ch.r0 + t * dr - r, ch.z0 + t * dz - z
    return np.sqrt(pr * pr + pz * pz), t


def field_proxy(r, z, channels, e0=1.5e6):
    out = np.full(np.shape(r), e0)
    for ch in channels:
        d, _ = _seg_dist(r, z, ch)
        dt = np.hypot(r - ch.r1, z - ch.z1)
        out = out + ch.volt / np.maximum(d, ch.radius) * (1 + 2 * np.exp(-dt / (5 * ch.radius)))
    return out


def channel_density(r, z, channels):
    n = np.zeros(np.shape(r))
    for ch in channels:
        d, t = _seg_dist(r, z, ch)
        n = n + ch.density * np.exp(-(d / ch.radius) ** 2)
    return n


def grow_tree(base_level: int, extra_levels: int, indicator, thr: float,
              h1: float = L_DOMAIN / M_BLOCK, rootsize=(1, 1), stencil=STAR2) -> Tree:
    """Uniform tree to ``base_level`` then refine, level by level, every leaf block
    whose max indicator over its cells exceeds ``thr`` (with proper nesting along
    ``stencil``)."""
    tree = Tree(rootsize, base_level + extra_levels)
    populate(tree, base_level)
    for l in range(base_level, base_level + extra_levels):
        blks, r, z, _, _ = block_cell_centres(tree, l, h1)
        if len(blks) == 0:
            break
        mx = indicator(r, z).reshape(len(blks), -1).max(axis=1)
        coords = list(tree[l - 1].index.keys())
        for q in np.nonzero(mx > thr)[0]:
            c = coords[q]
            if tree.isleaf(l, c):
                refine_block(tree, l, c, stencil)
    tree.sync()
    return tree


def tree_for_leaf_target(base_level, extra_levels, indicator, target_leaf, h1=L_DOMAIN / M_BLOCK,
                         iters=18):
    """Bisect the indicator threshold (in log space) for ~target_leaf leaf cells."""
    blks, r, z, _, _ = block_cell_centres(_uniform(base_level), base_level, h1)
    vals = indicator(r, z)
    hi, lo = math.log(float(vals.max())), math.log(float(np.median(vals)))
    best = None
    for _ in range(iters):
        mid = 0.5 * (lo + hi)
        tree = grow_tree(base_level, extra_levels, indicator, math.exp(mid), h1)
        n = leaf_cells(tree)
        if best is None or abs(math.log(n / target_leaf)) < abs(math.log(best[1] / target_leaf)):
            best = (tree, n)
        if abs(n / target_leaf - 1) < 0.03:
            break
        if n > target_leaf:
            lo = mid
        else:
            hi = mid
    return best[0]


def _uniform(level):
    t = Tree((1, 1), level)
    populate(t, level)
    return t


def make_problem(tree: Tree, rhs_fn, s, op=OP_LAPLACIAN, k2=0.0, bc=None, name="",
                 h1=L_DOMAIN / M_BLOCK, conn=None) -> Problem:
    """Evaluate ``rhs_fn(r, z, level, gi, gj)`` on every block, restrict onto parents."""
    if conn is None:
        conn = connectivity(tree)
    nblk = tree.nblocks_created
    b = np.zeros((nblk, S_BLOCK, S_BLOCK))
    for l in range(1, len(tree) + 1):
        blks, r, z, gi, gj = block_cell_centres(tree, l, h1)
        if len(blks):
            b[blks - 1, G_GHOST:G_GHOST + M_BLOCK, G_GHOST:G_GHOST + M_BLOCK] = rhs_fn(r, z, l, gi, gj)
    restrict_full_np(b, tree, conn)
    return Problem(tree=tree, conn=conn, b=b, s=s, op=op, k2=k2,
                   bc=(BC_POISSON if bc is None else bc).copy(), h1=h1, name=name)


def poisson_scale(h1=L_DOMAIN / M_BLOCK):
    return h1 * h1 * (ELEMENTARY_CHARGE / EPSILON_0)


# ----------------------------------------------------------------------------- configs

def config1(seed: int = 1) -> Problem:
    """Uniform tree to level 5 (341 blocks, 256x256 finest cells), Gaussian ion seed
    (peak 1e20 m^-3, sigma 0.2 mm read as a standard deviation, w = sqrt(2) sigma,
    src/initcond.jl:52-60) on the axis at mid-height with seeded jitter, over a 1e9
    m^-3 background that cancels in n_ion - n_e."""
    rng = np.random.default_rng(seed)
    tree = _uniform(5)
    h5 = L_DOMAIN / M_BLOCK / 16
    z0 = L_DOMAIN / 2 + rng.uniform(-h5 / 2, h5 / 2)
    w = math.sqrt(2) * 0.2e-3

    def rhs(r, z, l, gi, gj):
        n_ion = 1e9 + 1e20 * np.exp(-(r * r + (z - z0) ** 2) / (w * w))
        return n_ion - 1e9

    return make_problem(tree, rhs, poisson_scale(), name="config1-uniform-l5")


def seeded_channel(rng, main=True) -> Channel:
    length = rng.uniform(0.2, 0.6) * L_DOMAIN
    return Channel(r0=0.0, z0=L_DOMAIN, r1=0.0, z1=L_DOMAIN - length,
                   radius=rng.uniform(0.1e-3, 0.3e-3), density=10 ** rng.uniform(19, 20),
                   volt=1.0)


def channel_rhs(channels, seed):
    def rhs(r, z, l, gi, gj):
        n = channel_density(r, z, channels)
        noise = 10 ** (0.2 * cell_hash01(seed, l, gi, gj) - 0.1)   # log-uniform +-0.1 dex
        head = np.zeros_like(n)
        for ch in channels:
            dt = np.hypot(r - ch.r1, z - ch.z1)
            head += 0.1 * ch.density * np.exp(-(dt / (2 * ch.radius)) ** 2)
        return (n + head) - n * noise
    return rhs


def config2(seed: int = 2, target_leaf: int = 1_500_000, base_level=5, extra=4) -> Problem:
    """Config-1 base tree plus 4 refined levels (6-9) around a seeded thin conducting
    channel (radius 0.1-0.3 mm, length 20-60% of the gap, density 1e19-1e20 m^-3,
    log-uniform noise); about 1.5M leaf cells."""
    rng = np.random.default_rng(seed)
    ch = seeded_channel(rng)
    ind = lambda r, z: field_proxy(r, z, [ch])
    tree = tree_for_leaf_target(base_level, extra, ind, target_leaf)
    return make_problem(tree, channel_rhs([ch], seed), poisson_scale(),
                        name=f"config2-channel-{leaf_cells(tree)}leaf")


def branched_channels(rng, nbranch=4):
    main = seeded_channel(rng)
    chans = [main]
    for _ in range(nbranch):
        t = rng.uniform(0.3, 0.9)
        zb = main.z0 + t * (main.z1 - main.z0)
        ang = rng.uniform(0.15, 0.6)
        ln = rng.uniform(0.1, 0.3) * L_DOMAIN
        chans.append(Channel(r0=0.0, z0=zb, r1=ln * math.sin(ang), z1=zb - ln * math.cos(ang),
                             radius=main.radius * rng.uniform(0.6, 1.0),
                             density=main.density * rng.uniform(0.3, 1.0), volt=0.7))
    return chans


def config5(seed: int = 5, target_leaf: int = 10_000_000) -> Problem:
    """Uniform to level 6 (1024 blocks) plus 5 refined levels around a multi-branched
    seeded channel; 8-12M leaf cells."""
    rng = np.random.default_rng(seed)
    chans = branched_channels(rng)
    ind = lambda r, z: field_proxy(r, z, chans)
    tree = tree_for_leaf_target(6, 5, ind, target_leaf)
    return make_problem(tree, channel_rhs(chans, seed), poisson_scale(),
                        name=f"config5-branched-{leaf_cells(tree)}leaf")


def townsend_alpha(e):
    """Effective ionisation coefficient of air, alpha = A exp(-B/E) (m^-1)."""
    return 4.332e5 * np.exp(-1.41e7 / np.maximum(e, 1.0))


def config3_tree_problems(seed: int = 3, ntrees: int = 16, lo=1e5, hi=3e6):
    """16 independent trees with leaf cells log-uniform in [1e5, 3e6]; per tree one
    Poisson RHS (channel charge) and 3 Helmholtz photoionization terms with
    lambda_j = 10^U(2,4) m^-1, s = h^2, source = mu |E| n_e alpha(|E|)."""
    rng = np.random.default_rng(seed)
    out = []
    for t in range(ntrees):
        target = int(math.exp(rng.uniform(math.log(lo), math.log(hi))))
        ch = seeded_channel(rng)
        ind = lambda r, z, ch=ch: field_proxy(r, z, [ch])
        tree = tree_for_leaf_target(4 if target < 4e5 else 5, 5, ind, target)
        conn = connectivity(tree)
        pois = make_problem(tree, channel_rhs([ch], seed * 100 + t), poisson_scale(),
                            name=f"cfg3-tree{t}-poisson", conn=conn)
        scale = 1e6 / ch.volt

        def src(r, z, l, gi, gj, ch=ch, scale=scale):
            e = field_proxy(r, z, [ch]) * scale / 1e6 * 3e6
            ne = channel_density(r, z, [ch])
            return 0.0372 * e * ne * townsend_alpha(e)

        terms = []
        for j in range(3):
            lam = 10 ** rng.uniform(2, 4)
            h1 = L_DOMAIN / M_BLOCK
            terms.append(make_problem(tree, src, h1 * h1, op=OP_HELMHOLTZ, k2=lam * lam,
                                      bc=BC_PHOTO, name=f"cfg3-tree{t}-helm{j}", conn=conn))
        out.append((pois, terms))
    return out


def order4_problem(seed: int = 7, geom: int = GEOM_CYL1, base_level: int = 3, extra: int = 3,
                   thr_frac: float = 0.35) -> Problem:
    """The compact order-4 Laplacian (LaplacianDiscretization{2,4}) on a refined tree
    grown around a seeded channel with BoxStencil nesting and connectivity
    (src/simulate.jl:258-262, src/streamer.jl:437).  ``b`` holds the net charge q; the
    solve's right-hand side is rhs_level!(q1, q) of it (src/streamer.jl:313-318)."""
    rng = np.random.default_rng(seed)
    ch = seeded_channel(rng)
    ind = lambda r, z: field_proxy(r, z, [ch])
    blks, r, z, _, _ = block_cell_centres(_uniform(base_level), base_level, L_DOMAIN / M_BLOCK)
    vals = ind(r, z)
    thr = float(np.exp(np.log(vals.min()) + thr_frac * (np.log(vals.max()) - np.log(vals.min()))))
    tree = grow_tree(base_level, extra, ind, thr, stencil=BOX2)
    conn = connectivity(tree, BOX2)
    # Neumann on the axis and the outer radius, Dirichlet at the electrodes, with the
    # radial dimension chosen by the geometry; all Dirichlet for Cartesian
    bc = {GEOM_CART: boundaryconditions(((-1, -1), (-1, -1))), GEOM_CYL1: BC_POISSON,
          GEOM_CYL2: boundaryconditions(((-1, -1), (1, 1)))}[geom]
    pr = make_problem(tree, channel_rhs([ch], seed), poisson_scale(), op=OP_LAPLACIAN4, bc=bc,
                      name=f"order4-g{geom}-l{base_level}+{extra}", conn=conn)
    pr.geom = geom
    return pr


def outer_refined_problem(dim: int = 1, stencil=STAR2, seed: int = 9) -> Problem:
    """A tree refined at the outer radial boundary, for the free boundary conditions
    (FreeBC, src/freebc.jl): uniform to level 4 (8 x 8 blocks), two outer-edge blocks
    refined to level 5 and one of their outer-edge children to level 6, so that the
    outer boundary has refinement boundaries along it (the corrections of setouter!,
    src/freebc.jl:178-219).  ``dim`` is the radial dimension (CylindricalGeometry{dim});
    b is a seeded Gaussian charge on the axis."""
    rng = np.random.default_rng(seed)
    t = Tree((1, 1), 7)
    populate(t, 4)

    def at(r, z):
        return (r, z) if dim == 1 else (z, r)
    refine_block(t, 4, at(8, 4), stencil)
    refine_block(t, 4, at(8, 5), stencil)
    refine_block(t, 5, at(16, 9), stencil)
    t.sync()
    conn = connectivity(t, stencil)
    z0 = L_DOMAIN * rng.uniform(0.35, 0.65)
    w = 0.08 * L_DOMAIN

    def rhs(r, z, l, gi, gj):
        rr, zz = (r, z) if dim == 1 else (z, r)
        return 1e18 * np.exp(-(rr * rr + (zz - z0) ** 2) / (w * w))

    bc = boundaryconditions(((1, -1), (-1, -1))) if dim == 1 else boundaryconditions(((-1, -1), (1, -1)))
    pr = make_problem(t, rhs, poisson_scale(), bc=bc, name=f"outer-refined-dim{dim}", conn=conn)
    pr.geom = GEOM_CYL1 if dim == 1 else GEOM_CYL2
    return pr
