"""The C oracle reproduces, bit for bit, an independent pure-Python restatement of
the reference arithmetic (tests/golden/make_golden.py -> mg_tiny.npz).

The reference itself ships no golden vectors and cannot run here (pure Julia, no
Julia toolchain), so parity with the reference stays unpinned; this pins the oracle
against a second restatement written separately from the same reference lines.
"""
import os

import numpy as np
import pytest

from conftest import ROOT
import sys
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_golden as mk  # noqa: E402
from oracle import Oracle  # noqa: E402
from srmg.gen import Problem  # noqa: E402
from srmg.tree import connectivity  # noqa: E402

GOLD = np.load(os.path.join(ROOT, "tests", "golden", "mg_tiny.npz"))


@pytest.fixture(scope="module")
def orc():
    tree = mk.tiny_tree()
    conn = connectivity(tree)
    p = Problem(tree=tree, conn=conn, b=GOLD["b0"].copy(), s=0.5, bc=GOLD["bc"])
    return Oracle(p)


def bits_equal(a, b):
    return np.array_equal(a.view(np.uint64), b.view(np.uint64))


@pytest.mark.parametrize("l", [1, 2, 3])
def test_fill_ghost(orc, l):
    u = GOLD["u0"].copy()
    orc.fill_ghost(u, l)
    assert bits_equal(u, GOLD[f"fill_ghost_l{l}"])


def test_restrict(orc):
    from oracle import lib, _ptr
    u = GOLD["u0"].copy()
    lib().orc_restrict_level(_ptr(u), orc.ot.ref, 3)
    assert bits_equal(u, GOLD["restrict_l3"])


def test_interp_add(orc):
    from oracle import lib, _ptr
    u = GOLD["u0"].copy()
    b = GOLD["b0"].copy()
    lib().orc_interp_add_level(_ptr(u), _ptr(b), orc.ot.ref, 3)
    assert bits_equal(u, GOLD["interp_add_l3"])


def test_gs_iter(orc):
    import ctypes
    from oracle import lib, _ptr
    u = GOLD["u0"].copy()
    b = GOLD["b0"].copy()
    lib().orc_gs_iter(_ptr(u), _ptr(b), 1.0, 0.37, 2, 3, orc.ot.ref, ctypes.byref(orc.op))
    assert bits_equal(u, GOLD["gs_iter_l3"])


def test_residual(orc):
    import ctypes
    from oracle import lib, _ptr
    u = GOLD["u0"].copy()
    b = GOLD["b0"].copy()
    r = np.zeros_like(u)
    lib().orc_residual_level(_ptr(r), _ptr(u), _ptr(b), 0.37, orc.ot.ref, 3, ctypes.byref(orc.op))
    assert bits_equal(r, GOLD["residual_l3"])


def test_vcycle(orc):
    u = GOLD["vcycle_u_in"].copy()
    b = GOLD["b0"].copy()
    r, u1 = np.zeros_like(u), np.zeros_like(u)
    orc.vcycle(u, b, r, u1, ndown=2, ntop=4, nup=2, omega=1.0, s=0.5)
    assert bits_equal(u, GOLD["vcycle_u"])
    assert bits_equal(b, GOLD["vcycle_b"])
