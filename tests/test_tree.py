"""Host-side tree and connectivity logic (mirror of src/tree.jl, src/connectivity.jl)."""
import numpy as np
import pytest

from srmg.tree import (Tree, populate, refine_block, connectivity, boundaryconditions,
                       parentcoord, subcoord, leaf_cells)
from srmg import gen


def uniform(level):
    t = Tree((1, 1), level)
    populate(t, level)
    return t


def test_populate_numbering_and_counts():
    t = uniform(5)
    assert [len(l) for l in t] == [1, 4, 16, 64, 256]
    assert t.nblocks() == 341
    # populate! numbers level by level, CartesianIndices order (dim 1 fastest)
    assert t[1].index[(1, 1)] == 2 and t[1].index[(2, 1)] == 3 and t[1].index[(1, 2)] == 4


def test_uniform_connectivity_counts():
    t = uniform(4)
    c = connectivity(t)
    for l, layer in enumerate(t, start=1):
        n = layer.domain[0]
        assert len(c.neighbor[l - 1]) == 4 * n * (n - 1)
        assert len(c.boundary[l - 1]) == 4 * n
        assert len(c.refboundary[l - 1]) == 0
        assert len(c.child[l - 1]) == (0 if l == 1 else n * n)


def test_every_face_has_exactly_one_edge():
    p = gen.config2(seed=7, target_leaf=120_000)
    t, c = p.tree, p.conn
    for l, layer in enumerate(t, start=1):
        seen = {}
        for e in c.neighbor[l - 1]:
            key = (int(e["to"]), (-int(e["face"][0]), -int(e["face"][1])))
            assert key not in seen
            seen[key] = "n"
        for e in c.boundary[l - 1]:
            key = (int(e["block"]), tuple(int(v) for v in e["face"]))
            assert key not in seen and tuple(e["bnd"]) == tuple(e["face"])
            seen[key] = "b"
        for e in c.refboundary[l - 1]:
            key = (int(e["fine"]), tuple(int(v) for v in e["face"]))
            assert key not in seen
            seen[key] = "r"
        assert len(seen) == 4 * len(layer)


def test_proper_nesting_after_refinement():
    t = Tree((1, 1), 5)
    populate(t, 3)
    refine_block(t, 3, (4, 4))  # corner block: forces no extra refinement at level 3
    refine_block(t, 4, (7, 7))  # needs (6,7) and (7,6): forces refining their parents
    t.sync()
    c = connectivity(t)  # raises if nesting is broken
    assert len(c.refboundary[3]) > 0
    # children of refined blocks cover their parent's subblocks exactly once
    for l in range(2, len(t) + 1):
        cover = {}
        for e in c.child[l - 1]:
            k = (int(e["coarse"]), tuple(e["subblock"]))
            assert k not in cover
            cover[k] = 1


def test_parent_and_subcoord():
    assert parentcoord((3, 4)) == (2, 2)
    assert subcoord((3, 4)) == (1, 2)
    assert parentcoord((1, 1)) == (1, 1) and subcoord((2, 1)) == (2, 1)


def test_boundaryconditions_table():
    # src/boundary.jl:28-38, column-major flattening, a[2+b1, 2+b2]
    bc = boundaryconditions(((1, -1), (-1, -1)))
    a = bc.reshape(3, 3, order="F")
    assert a[0, 1] == 1 and a[2, 1] == -1 and a[1, 0] == -1 and a[1, 2] == -1
    assert a[0, 0] == -1 and a[2, 2] == 1  # corners multiply


def test_generators_are_deterministic():
    a = gen.config2(seed=3, target_leaf=60_000)
    b = gen.config2(seed=3, target_leaf=60_000)
    assert a.nblk == b.nblk
    np.testing.assert_array_equal(a.b, b.b)
    assert leaf_cells(a.tree) == leaf_cells(b.tree)


def test_config1_shape():
    p = gen.config1()
    assert p.nblk == 341 and len(p.tree) == 5
    assert leaf_cells(p.tree) == 65536
    assert p.b.max() > 1e19


@pytest.mark.parametrize("target", [150_000, 400_000])
def test_leaf_target_is_met(target):
    p = gen.config2(seed=11, target_leaf=target)
    n = leaf_cells(p.tree)
    assert 0.7 * target < n < 1.4 * target
