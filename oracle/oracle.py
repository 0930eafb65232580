"""ctypes binding to the oracle (CPU FP64 restatement of the reference solve).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / reference legs.  Parity of the oracle with the reference is unpinned
(no reference golden vectors exist and Julia is absent); see srmg_oracle.h.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_P = ctypes.c_void_p
_I64P = ctypes.POINTER(ctypes.c_int64)


class _Tree(ctypes.Structure):
    _fields_ = [("M", ctypes.c_int), ("G", ctypes.c_int), ("nlev", ctypes.c_int),
                ("npairs", _I64P), ("pairs", ctypes.POINTER(_P)),
                ("nnb", _I64P), ("nb", ctypes.POINTER(_P)),
                ("nbd", _I64P), ("bd", ctypes.POINTER(_P)),
                ("nrb", _I64P), ("rb", ctypes.POINTER(_P)),
                ("nch", _I64P), ("ch", ctypes.POINTER(_P)),
                ("nblk_alloc", ctypes.c_int64), ("coord_of", _I64P)]


class _Op(ctypes.Structure):
    _fields_ = [("op", ctypes.c_int), ("k2", ctypes.c_double), ("geom", ctypes.c_int),
                ("bc", ctypes.c_int8 * 9), ("bc27", ctypes.c_int8 * 27)]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        TP, OP, D = ctypes.POINTER(_Tree), ctypes.POINTER(_Op), ctypes.c_double
        PP = _P
        I = ctypes.c_int
        sig = {
            "orc_tree_index": (None, [TP]),
            "orc_fill_ghost_copy": (None, [PP, TP, I]),
            "orc_fill_ghost_bnd": (None, [PP, TP, I, PP]),
            "orc_fill_ghost_interp": (None, [PP, TP, I]),
            "orc_fill_ghost": (None, [PP, TP, I, PP]),
            "orc_restrict_level": (None, [PP, TP, I]),
            "orc_restrict_full": (None, [PP, TP]),
            "orc_interp_add_level": (None, [PP, PP, TP, I]),
            "orc_copyto_level": (None, [PP, PP, TP, I]),
            "orc_diffto_level": (None, [PP, PP, PP, TP, I]),
            "orc_gs_level": (None, [PP, PP, D, D, TP, I, OP, I]),
            "orc_gs4_level": (None, [PP, PP, D, D, TP, I, OP, I, I]),
            "orc_gs_iter": (None, [PP, PP, D, D, I, I, TP, OP]),
            "orc_rhs_level": (None, [PP, PP, TP, I, OP]),
            "orc_residual_level": (None, [PP, PP, PP, D, TP, I, OP]),
            "orc_residual_postrestrict_level": (None, [PP, PP, PP, D, TP, I, OP]),
            "orc_vcycle": (None, [PP, PP, PP, PP, D, TP, OP, I, I, I, I, D]),
            "orc_fmg": (None, [PP, PP, PP, PP, D, TP, OP, I, I, I, D]),
            "orc_resnorm": (D, [PP, PP, PP, D, TP, OP]),
            "orc_leafnorm": (D, [PP, PP, TP]),
            "orc_solve": (I, [PP, PP, PP, PP, D, TP, OP, I, I, I, D, D, I, ctypes.POINTER(D)]),
            "orc_netcharge": (None, [PP, PP, PP, TP]),
            "orc_electric_field": (None, [PP, PP, PP, D, PP, TP]),
            "orc3_tree_index": (None, [TP]),
            "orc3_fill_ghost_copy": (None, [PP, TP, I]),
            "orc3_fill_ghost_bnd": (None, [PP, TP, I, PP]),
            "orc3_fill_ghost_interp": (None, [PP, TP, I]),
            "orc3_fill_ghost": (None, [PP, TP, I, PP]),
            "orc3_restrict_level": (None, [PP, TP, I]),
            "orc3_interp_add_level": (None, [PP, PP, TP, I]),
            "orc3_gs_level": (None, [PP, PP, D, D, TP, I, OP, I]),
            "orc3_gs4_level": (None, [PP, PP, D, D, TP, I, OP, I, I]),
            "orc3_gs_iter": (None, [PP, PP, D, D, I, I, TP, OP]),
            "orc3_residual_level": (None, [PP, PP, PP, D, TP, I, OP]),
            "orc3_residual_postrestrict_level": (None, [PP, PP, PP, D, TP, I, OP]),
            "orc3_rhs_level": (None, [PP, PP, TP, I, OP]),
            "orc3_vcycle": (None, [PP, PP, PP, PP, D, TP, OP, I, I, I, I, D]),
            "orc3_fmg": (None, [PP, PP, PP, PP, D, TP, OP, I, I, I, D]),
            "orc3_resnorm": (D, [PP, PP, PP, D, TP, OP]),
            "orc3_leafnorm": (D, [PP, PP, TP]),
            "orc3_solve": (I, [PP, PP, PP, PP, D, TP, OP, I, I, I, D, D, I, ctypes.POINTER(D)]),
            "orc_set_threads": (None, [I]),
            "orc_get_threads": (I, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.c_void_p)


class OracleTree:
    """Holds ctypes views of a tree + connectivity for the oracle."""

    def __init__(self, tree, conn, nblk_alloc, M=16, G=2):
        nlev = len(tree)
        D = getattr(tree, "D", 2)
        self._keep = []
        pairs = [np.ascontiguousarray(layer.pairs_array()) for layer in tree]

        def arrs(lists):
            lists = [np.ascontiguousarray(x) for x in lists]
            self._keep.extend(lists)
            n = (ctypes.c_int64 * nlev)(*[len(x) for x in lists])
            p = (_P * nlev)(*[x.ctypes.data for x in lists])
            self._keep.extend([n, p])
            return n, p

        t = _Tree()
        t.M, t.G, t.nlev = M, G, nlev
        n, p = arrs(pairs)
        t.npairs, t.pairs = ctypes.cast(n, _I64P), ctypes.cast(p, ctypes.POINTER(_P))
        for field, lists in (("nb", conn.neighbor), ("bd", conn.boundary),
                             ("rb", conn.refboundary), ("ch", conn.child)):
            n, p = arrs(lists)
            setattr(t, "n" + field, ctypes.cast(n, _I64P))
            setattr(t, field, ctypes.cast(p, ctypes.POINTER(_P)))
        # orc3_tree has orc_tree's layout; only the edge records and coord_of differ
        self.coord_of = np.zeros(D * nblk_alloc, dtype=np.int64)
        t.nblk_alloc = nblk_alloc
        t.coord_of = self.coord_of.ctypes.data_as(_I64P)
        self.t = t
        self.nlev = nlev
        (lib().orc3_tree_index if D == 3 else lib().orc_tree_index)(ctypes.byref(t))

    @property
    def ref(self):
        return ctypes.byref(self.t)


def make_op(op, k2, geom, bc):
    o = _Op()
    o.op, o.k2, o.geom = op, k2, geom
    if len(bc) == 27:
        for i in range(27):
            o.bc27[i] = int(bc[i])
    else:
        for i in range(9):
            o.bc[i] = int(bc[i])
    return o


def bc_ptr(bc):
    a = np.ascontiguousarray(np.asarray(bc, dtype=np.int8))
    return a, _ptr(a)


class Oracle:
    """Convenience wrapper mirroring the reference's Julia entry points."""

    def __init__(self, problem, threads=None):
        self.p = problem
        self.ot = OracleTree(problem.tree, problem.conn, problem.nblk)
        self.op = make_op(problem.op, problem.k2, problem.geom, problem.bc)
        self._bc, self._bcp = bc_ptr(problem.bc)
        if threads:
            lib().orc_set_threads(threads)

    def fill_ghost(self, u, l):
        lib().orc_fill_ghost(_ptr(u), self.ot.ref, l, self._bcp)

    def fill_ghost_all(self, u):
        for l in range(1, self.ot.nlev + 1):
            self.fill_ghost(u, l)

    def rhs_level(self, q1, q, l):
        lib().orc_rhs_level(_ptr(q1), _ptr(q), self.ot.ref, l, ctypes.byref(self.op))

    def vcycle(self, u, b, r, u1, lmax=0, ndown=2, ntop=4, nup=2, omega=1.0, s=None):
        lib().orc_vcycle(_ptr(u), _ptr(b), _ptr(r), _ptr(u1), self.p.s if s is None else s,
                         self.ot.ref, ctypes.byref(self.op), lmax, ndown, ntop, nup, omega)

    def fmg(self, u, b, r, u1, ndown=2, ntop=4, nup=2, omega=1.25):
        lib().orc_fmg(_ptr(u), _ptr(b), _ptr(r), _ptr(u1), self.p.s, self.ot.ref,
                      ctypes.byref(self.op), ndown, ntop, nup, omega)

    def resnorm(self, r, b, u):
        return lib().orc_resnorm(_ptr(r), _ptr(b), _ptr(u), self.p.s, self.ot.ref,
                                 ctypes.byref(self.op))

    def leafnorm(self, f):
        scratch = np.empty_like(f)
        return lib().orc_leafnorm(_ptr(scratch), _ptr(f), self.ot.ref)

    def solve(self, u, b, tol, max_cycles=500, ndown=2, ntop=4, nup=2, omega=1.0):
        r, u1 = np.zeros_like(u), np.zeros_like(u)
        rel = ctypes.c_double()
        c = lib().orc_solve(_ptr(u), _ptr(b), _ptr(r), _ptr(u1), self.p.s, self.ot.ref,
                            ctypes.byref(self.op), ndown, ntop, nup, omega, tol, max_cycles,
                            ctypes.byref(rel))
        return c, rel.value


class Oracle3:
    """The D = 3 oracle (srmg_oracle3.c) for a Problem3-like object with tree, conn, b
    ([nblk, 20, 20, 20]), s, op, k2 and a 27-entry bc."""

    def __init__(self, problem, threads=None):
        self.p = problem
        self.ot = OracleTree(problem.tree, problem.conn, problem.nblk)
        self.op = make_op(problem.op, problem.k2, 0, problem.bc)
        self._bc, self._bcp = bc_ptr(problem.bc)
        if threads:
            lib().orc_set_threads(threads)

    def fill_ghost(self, u, l):
        lib().orc3_fill_ghost(_ptr(u), self.ot.ref, l, self._bcp)

    def fill_ghost_all(self, u):
        for l in range(1, self.ot.nlev + 1):
            self.fill_ghost(u, l)

    def rhs_level(self, q1, q, l):
        lib().orc3_rhs_level(_ptr(q1), _ptr(q), self.ot.ref, l, ctypes.byref(self.op))

    def vcycle(self, u, b, r, u1, lmax=0, ndown=2, ntop=4, nup=2, omega=1.0, s=None):
        lib().orc3_vcycle(_ptr(u), _ptr(b), _ptr(r), _ptr(u1), self.p.s if s is None else s, self.ot.ref,
                          ctypes.byref(self.op), lmax, ndown, ntop, nup, omega)

    def fmg(self, u, b, r, u1, ndown=2, ntop=4, nup=2, omega=1.25):
        lib().orc3_fmg(_ptr(u), _ptr(b), _ptr(r), _ptr(u1), self.p.s, self.ot.ref, ctypes.byref(self.op),
                       ndown, ntop, nup, omega)

    def resnorm(self, r, b, u):
        return lib().orc3_resnorm(_ptr(r), _ptr(b), _ptr(u), self.p.s, self.ot.ref, ctypes.byref(self.op))

    def leafnorm(self, f):
        scratch = np.empty_like(f)
        return lib().orc3_leafnorm(_ptr(scratch), _ptr(f), self.ot.ref)

    def solve(self, u, b, tol, max_cycles=500, ndown=2, ntop=4, nup=2, omega=1.0):
        r, u1 = np.zeros_like(u), np.zeros_like(u)
        rel = ctypes.c_double()
        c = lib().orc3_solve(_ptr(u), _ptr(b), _ptr(r), _ptr(u1), self.p.s, self.ot.ref, ctypes.byref(self.op),
                             ndown, ntop, nup, omega, tol, max_cycles, ctypes.byref(rel))
        return c, rel.value
