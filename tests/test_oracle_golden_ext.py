"""The C oracle's order-4 (2D, BoxStencil tree) and three-dimensional operations
reproduce, bit for bit, an independent pure-Python restatement of the same reference
lines (tests/golden/make_golden_ext.py -> ext_hashes.json: SHA-256 of each output).
Inputs are regenerated from the generator's seeds."""
import ctypes
import json
import os
import sys

import numpy as np
import pytest

from conftest import ROOT
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_golden_ext as mk  # noqa: E402
from oracle import Oracle, Oracle3, lib as olib, _ptr  # noqa: E402
from srmg import gen, gen3  # noqa: E402
from srmg.tree import connectivity, BOX2  # noqa: E402
from srmg import tree3 as t3  # noqa: E402

HASHES = json.load(open(os.path.join(ROOT, "tests", "golden", "ext_hashes.json")))


@pytest.fixture(scope="module")
def o4():
    tree = mk.order4_tree()
    conn = connectivity(tree, BOX2)
    u0, b0 = mk.inputs2(tree.nblocks_created)
    p = gen.Problem(tree=tree, conn=conn, b=b0.copy(), s=0.37, op=2, bc=mk.BC2)
    return Oracle(p), u0, b0


@pytest.fixture(scope="module")
def d3():
    t = mk.tiny_octree()
    c3 = t3.connectivity(t, t3.STAR3)
    cb = t3.connectivity(t, t3.BOX3)
    v0, w0 = mk.inputs3(t.nblocks_created)
    mk_p = lambda conn, op=0, k2=0.0: gen3.Problem3(tree=t, conn=conn, b=w0.copy(), s=0.37, op=op, k2=k2, bc=mk.BC3)
    return t, c3, cb, v0, w0, mk_p


@pytest.mark.parametrize("l", [1, 2, 3])
def test_order4_fill(o4, l):
    o, u0, _ = o4
    u = u0.copy()
    o.fill_ghost(u, l)
    assert mk.digest(u) == HASHES[f"o4_fill_l{l}"]


@pytest.mark.parametrize("geom", [0, 1, 2])
def test_order4_gs_residual_rhs(o4, geom):
    o, u0, b0 = o4
    o.op.geom = geom
    u = u0.copy()
    olib().orc_gs_iter(_ptr(u), _ptr(b0), 1.0, 0.37, 2, 3, o.ot.ref, ctypes.byref(o.op))
    assert mk.digest(u) == HASHES[f"o4_gs_iter_l3_g{geom}"]
    r = np.zeros_like(u0)
    olib().orc_residual_level(_ptr(r), _ptr(u0), _ptr(b0), 0.37, o.ot.ref, 3, ctypes.byref(o.op))
    assert mk.digest(r) == HASHES[f"o4_residual_l3_g{geom}"]
    q1 = np.zeros_like(u0)
    o.rhs_level(q1, u0, 3)
    assert mk.digest(q1) == HASHES[f"o4_rhs_l3_g{geom}"]


@pytest.mark.parametrize("name", ["star", "box"])
def test_3d_fill(d3, name):
    t, c3, cb, v0, w0, mk_p = d3
    o = Oracle3(mk_p(c3 if name == "star" else cb))
    for l in (1, 2, 3):
        u = v0.copy()
        o.fill_ghost(u, l)
        assert mk.digest(u) == HASHES[f"d3_fill_{name}_l{l}"], l


def test_3d_transfers(d3):
    t, c3, cb, v0, w0, mk_p = d3
    o = Oracle3(mk_p(c3))
    u = v0.copy()
    olib().orc3_restrict_level(_ptr(u), o.ot.ref, 3)
    assert mk.digest(u) == HASHES["d3_restrict_l3"]
    u = v0.copy()
    olib().orc3_interp_add_level(_ptr(u), _ptr(w0), o.ot.ref, 3)
    assert mk.digest(u) == HASHES["d3_interp_add_l3"]


@pytest.mark.parametrize("op,k2", [(0, 0.0), (1, 30.0), (2, 0.0)])
def test_3d_gs_residual(d3, op, k2):
    t, c3, cb, v0, w0, mk_p = d3
    o = Oracle3(mk_p(c3, op, k2))
    if op != 2:
        u = v0.copy()
        olib().orc3_gs_iter(_ptr(u), _ptr(w0), 1.0, 0.37, 1, 3, o.ot.ref, ctypes.byref(o.op))
        assert mk.digest(u) == HASHES[f"d3_gs_iter_l3_op{op}"]
    r = np.zeros_like(v0)
    olib().orc3_residual_level(_ptr(r), _ptr(v0), _ptr(w0), 0.37, o.ot.ref, 3, ctypes.byref(o.op))
    assert mk.digest(r) == HASHES[f"d3_residual_l3_op{op}"]


def test_3d_vcycle(d3):
    t, c3, cb, v0, w0, mk_p = d3
    o = Oracle3(mk_p(c3))
    u, b = v0.copy(), w0.copy()
    o.fill_ghost_all(u)
    o.vcycle(u, b, np.zeros_like(u), np.zeros_like(u), ndown=1, ntop=2, nup=1, s=0.5)
    assert mk.digest(u) == HASHES["d3_vcycle_u"]
    assert mk.digest(b) == HASHES["d3_vcycle_b"]
