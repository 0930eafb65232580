"""The C-ABI library loads and exports every entry point include/srmg.h declares.

No compute call is made here: these run on the CPU-only container too.
"""
import ctypes
import os

from conftest import ROOT, gpu_available
from srmg import multigrid as mg

HEADER = os.path.join(ROOT, "include", "srmg.h")


def test_library_loads():
    assert os.path.exists(mg.LIB_PATH), "libsrmg.so must be built (build())"
    mg.lib()


def test_every_declared_symbol_is_exported():
    names = mg.exported_symbols_from_header(HEADER)
    assert len(names) >= 20
    L = ctypes.CDLL(mg.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_the_header():
    names = set(mg.exported_symbols_from_header(HEADER))
    assert names == set(mg.SIGNATURES), names ^ set(mg.SIGNATURES)


def test_edge_struct_layouts_match_julia_isbits():
    from srmg import tree as t
    # Pair{CartesianIndex{2},Int}=24, Neighbor=32, Boundary=48, RefBoundary=48, Child=32
    assert t.PAIR_DTYPE.itemsize == 24
    assert t.NEIGHBOR_DTYPE.itemsize == 32
    assert t.BOUNDARY_DTYPE.itemsize == 48
    assert t.REFBND_DTYPE.itemsize == 48
    assert t.CHILD_DTYPE.itemsize == 32


def test_create_without_gpu_fails_cleanly():
    if gpu_available():
        return
    h = ctypes.c_void_p()
    rc = mg.lib().srmg_create(ctypes.byref(h), 2, 16, 2, 0)
    assert rc == -3 and not h.value


def test_unsupported_shapes_rejected():
    h = ctypes.c_void_p()
    assert mg.lib().srmg_create(ctypes.byref(h), 4, 16, 2, 0) == -6
    assert mg.lib().srmg_create(ctypes.byref(h), 1, 16, 2, 0) == -6
    assert mg.lib().srmg_create(ctypes.byref(h), 2, 8, 2, 0) == -6
    assert mg.lib().srmg_create(ctypes.byref(h), 3, 16, 4, 0) == -6


def test_three_dimensional_struct_layouts():
    """The D = 3 edge records the Python builder emits have the isbits sizes of
    Pair{CartesianIndex{3},Int}, Neighbor{3}, Boundary{3}, RefBoundary{3}, Child{3}
    (the srmg_*3 structs of include/srmg.h)."""
    from srmg import tree3
    assert tree3.PAIR3_DTYPE.itemsize == 32
    assert tree3.NEIGHBOR3_DTYPE.itemsize == 40
    assert tree3.BOUNDARY3_DTYPE.itemsize == 64
    assert tree3.REFBND3_DTYPE.itemsize == 64
    assert tree3.CHILD3_DTYPE.itemsize == 40
