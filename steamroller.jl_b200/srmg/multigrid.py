"""ctypes binding of libsrmg with the reference's entry-point names.

``vcycle_`` / ``fmg_`` / ``resnorm`` / ``fill_ghost_`` take the same arguments, in the
same order and with the same meaning, as the Julia functions they replace
(src/multigrid.jl:17-106, 391-417; src/connectivity.jl:155-159); fields are numpy
arrays of shape (nblk, 20, 20) in C order, i.e. Julia's column-major (i, j, blk)
layout.  Errors raise ``SrmgError`` the way the reference raises Julia exceptions.

There is no CPU fallback: if ``libsrmg.so`` is missing this module raises on import
of the library (``lib()``), and every call runs on the GPU.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .tree import Tree, Connectivity

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsrmg.so")

SRMG_OK = 0
# error codes of include/srmg.h
SRMG_ERR_BADARG, SRMG_ERR_BADTREE, SRMG_ERR_CUDA, SRMG_ERR_TIMEOUT = -1, -2, -3, -4
SRMG_ERR_DIVERGED, SRMG_ERR_UNSUPPORTED, SRMG_ERR_NOMEM, SRMG_ERR_NOTREE = -5, -6, -7, -8
ERRORS = {-1: "BADARG", -2: "BADTREE", -3: "CUDA", -4: "TIMEOUT", -5: "DIVERGED",
          -6: "UNSUPPORTED", -7: "NOMEM", -8: "NOTREE"}
MODE_FP64, MODE_MIXED, MODE_FP64_DIRECT = 0, 1, 2
# Smoother of the mixed-precision (and FP64-direct) solves as the autotuner picks it on
# the refined 1.5M- and 10M-leaf-cell trees: one red-black sweep down and one up per
# level, relaxation factor 1.1 (the reference's own cycle, V(2,2) with omega 1, stays the
# default of every entry point).
TUNED = dict(ndown=1, nup=1, ntop=4, omega=1.1)


class SrmgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"srmg error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class SolveOpts(ctypes.Structure):
    _fields_ = [("tol", ctypes.c_double), ("max_cycles", ctypes.c_int), ("mode", ctypes.c_int),
                ("ndown", ctypes.c_int), ("ntop", ctypes.c_int), ("nup", ctypes.c_int),
                ("omega", ctypes.c_double), ("inner_cycles", ctypes.c_int),
                ("warm_start", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("cycles", ctypes.c_int), ("outer", ctypes.c_int),
                ("rel_residual", ctypes.c_double), ("initial_rel", ctypes.c_double),
                ("bnorm", ctypes.c_double), ("device_ms", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneTrial(ctypes.Structure):
    _fields_ = [("engine_ctas", ctypes.c_int), ("local_max_blocks", ctypes.c_int), ("ndown", ctypes.c_int),
                ("nup", ctypes.c_int), ("ntop", ctypes.c_int), ("cycles", ctypes.c_int), ("ms", ctypes.c_double),
                ("omega", ctypes.c_double), ("inner_cycles", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Item(ctypes.Structure):
    """srmg_item: one problem of a batch (its tree's context and its operator)."""
    _fields_ = [("tree", ctypes.c_void_p), ("s", ctypes.c_double), ("op", ctypes.c_int),
                ("k2", ctypes.c_double), ("bc", ctypes.c_int8 * 9)]


_lib = None
_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_D = ctypes.c_double

# name -> (restype, argtypes); the complete exported surface of include/srmg.h
class Transport(ctypes.Structure):
    """srmg_transport: the MinimalTransportModel (src/transport.jl:9-35)."""
    _fields_ = [("mu", _D), ("D", _D), ("ai", _D), ("Ei", _D), ("aa", _D), ("Ea", _D)]


SIGNATURES = {
    "srmg_create": (_I, [ctypes.POINTER(_P), _I, _I, _I, _I]),
    "srmg_destroy": (None, [_P]),
    "srmg_last_error": (ctypes.c_char_p, [_P]),
    "srmg_set_stream": (_I, [_P, _P]),
    "srmg_synchronize": (_I, [_P]),
    "srmg_set_tree": (_I, [_P, _I] + [_P] * 10 + [ctypes.c_uint64]),
    "srmg_set_tree3": (_I, [_P, _I] + [_P] * 10 + [ctypes.c_uint64]),
    "srmg_tree_generation": (ctypes.c_uint64, [_P]),
    "srmg_vcycle": (_I, [_P, _P, _P, _P, _P, _I64, _D, _I, _D, _I, _P, _I, _I, _I, _I, _D, _I]),
    "srmg_fmg": (_I, [_P, _P, _P, _P, _P, _I64, _D, _I, _D, _I, _P, _I, _I, _I, _D]),
    "srmg_resnorm": (_I, [_P, _P, _P, _P, _I64, _D, _I, _D, _I, _P, ctypes.POINTER(_D)]),
    "srmg_fill_ghost": (_I, [_P, _P, _I64, _I, _P]),
    "srmg_solve_opts_default": (None, [ctypes.POINTER(SolveOpts)]),
    "srmg_solve": (_I, [_P, _P, _P, _I64, _D, _I, _D, _I, _P, ctypes.POINTER(SolveOpts),
                        ctypes.POINTER(Stats)]),
    "srmg_vcycle_dev": (_I, [_P, _P, _P, _P, _P, _I64, _D, _I, _D, _I, _P, _I, _I, _I, _I, _D, _I]),
    "srmg_fmg_dev": (_I, [_P, _P, _P, _P, _P, _I64, _D, _I, _D, _I, _P, _I, _I, _I, _D]),
    "srmg_resnorm_dev": (_I, [_P, _P, _P, _P, _I64, _D, _I, _D, _I, _P, ctypes.POINTER(_D)]),
    "srmg_solve_dev": (_I, [_P, _P, _P, _I64, _D, _I, _D, _I, _P, ctypes.POINTER(SolveOpts),
                            ctypes.POINTER(Stats)]),
    "srmg_solve_async": (_I, [_P, _P, _P, _I64, _D, _I, _D, _I, _P, ctypes.POINTER(SolveOpts)]),
    "srmg_solve_wait": (_I, [_P, ctypes.POINTER(Stats)]),
    "srmg_fill_ghost_dev": (_I, [_P, _P, _I64, _I, _P, _I]),
    "srmg_gs_level_dev": (_I, [_P, _P, _P, _I64, _I, _D, _D, _I, _D, _I, _I]),
    "srmg_gs_iter_dev": (_I, [_P, _P, _P, _I64, _I, _D, _D, _I, _I, _D, _I, _P]),
    "srmg_residual_level_dev": (_I, [_P, _P, _P, _P, _I64, _I, _D, _I, _D, _I]),
    "srmg_restrict_level_dev": (_I, [_P, _P, _I64, _I]),
    "srmg_restrict_full_dev": (_I, [_P, _P, _I64]),
    "srmg_rhs_level": (_I, [_P, _P, _P, _I64, _I, _I, _I]),
    "srmg_freebc_set": (_I, [_P, _I, _I, _P, _P, _I64]),
    "srmg_freebc": (_I, [_P, _P, _P, _I64, _D, _D, _P]),
    "srmg_freebc_dev": (_I, [_P, _P, _P, _I64, _D, _D, _P]),
    "srmg_fill_ghost_free": (_I, [_P, _P, _I64, _I]),
    "srmg_fill_ghost_free_dev": (_I, [_P, _P, _I64, _I]),
    "srmg_rhs_level_dev": (_I, [_P, _P, _P, _I64, _I, _I, _I]),
    "srmg_netcharge": (_I, [_P, _P, _P, _P, _I64]),
    "srmg_netcharge_dev": (_I, [_P, _P, _P, _P, _I64]),
    "srmg_electric_field": (_I, [_P, _P, _P, _P, _I64, ctypes.c_double, _P]),
    "srmg_electric_field_dev": (_I, [_P, _P, _P, _P, _I64, ctypes.c_double, _P]),
    "srmg_interp_add_level_dev": (_I, [_P, _P, _P, _I64, _I]),
    "srmg_residual_postrestrict_level_dev": (_I, [_P, _P, _P, _P, _I64, _I, _D, _I, _D, _I]),
    "srmg_resnorm_noalloc": (_I, [_P, _P, _P, _I64, _D, _I, _D, _I, _P]),
    "srmg_selftest_barrier_timeout": (_I, [_P, _I]),
    "srmg_set_option": (_I, [_P, ctypes.c_char_p, _I64]),
    "srmg_host_register": (_I, [_P, _P, _I64]),
    "srmg_host_unregister": (_I, [_P, _P]),
    "srmg_get_trace": (_I, [_P, _P, _I]),
    "srmg_launch_count": (_I64, [_P]),
    "srmg_batch_set": (_I, [_P, _I, ctypes.POINTER(Item), _I]),
    "srmg_batch_items": (_I, [_P]),
    "srmg_batch_offset": (_I64, [_P, _I]),
    "srmg_batch_nblk": (_I64, [_P, _I]),
    "srmg_batch_solve_dev": (_I, [_P, _P, _P, ctypes.POINTER(SolveOpts), ctypes.POINTER(Stats)]),
    "srmg_batch_solve": (_I, [_P, _P, _P, ctypes.POINTER(SolveOpts), ctypes.POINTER(Stats)]),
    "srmg_batch_solve_forest_dev": (_I, [_P, _P, _P, ctypes.POINTER(SolveOpts), ctypes.POINTER(Stats)]),
    "srmg_autotune": (_I, [_P, _P, _P, _I64, _D, _I, _D, _I, _P, ctypes.POINTER(SolveOpts),
                           ctypes.POINTER(TuneTrial), _I]),
    "srmg_batch_autotune": (_I, [_P, _P, _P, ctypes.POINTER(SolveOpts), ctypes.POINTER(TuneTrial), _I]),
    "srmg_cnn_create": (_I, [ctypes.POINTER(_P), _I, ctypes.c_uint64]),
    "srmg_cnn_destroy": (None, [_P]),
    "srmg_cnn_last_error": (ctypes.c_char_p, [_P]),
    "srmg_cnn_nparams": (_I, []),
    "srmg_cnn_get_params": (_I, [_P, _P, _I]),
    "srmg_cnn_set_params": (_I, [_P, _P, _I]),
    "srmg_cnn_synchronize": (_I, [_P]),
    "srmg_cnn_forward": (_I, [_P, _P, _P, _I]),
    "srmg_cnn_gradients": (_I, [_P, _P, _P, _P, ctypes.c_float, _I, _I, _P, ctypes.POINTER(_D)]),
    "srmg_cnn_train_step": (_I, [_P, _P, _P, _P, ctypes.c_float, _I, _I, ctypes.c_float, ctypes.POINTER(_D)]),
    "srmg_cnn_forward_train": (_I, [_P, _P, _I, _P]),
    "srmg_cnn_forward_tc": (_I, [_P, _P, _P, _I]),
    "srmg_cnn_tc_status": (_I, [_P]),
    "srmg_cnn_use_tcgen05": (_I, [_P, _I]),
    "srmg_cnn_backward_step": (_I, [_P, _P, _I, ctypes.c_float, _P]),
    "srmg_cnn_leaf_blocks": (_I, [_P]),
    "srmg_cnn_last_active": (_I, [_P]),
    "srmg_cnn_pack_dev": (_I, [_P, _P, _P, _I64, _D, _I, _D, _I, _P, _P, _P, _P, _I]),
    "srmg_cnn_predict_dev": (_I, [_P, _P, _P, _P, _P, _P, _P, _I64, _D, _I, _D, _I, _P, ctypes.POINTER(_I),
                                  ctypes.POINTER(_D)]),
    "srmg_streamer_flux_dev": (_I, [_P, _P, _P, _P, _P, _P, _P, _I64, _D, ctypes.POINTER(Transport)]),
    "srmg_streamer_rates_dev": (_I, [_P, _P, _P, _P, _P, _P, _I64, _D, _I, ctypes.POINTER(Transport)]),
    "srmg_ssprk3_stage_dev": (_I, [_P, _P, _P, _P, _P, _P, _I64, _D, _I]),
}


def lib():
    """Load libsrmg.so; raises if it has not been built (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libsrmg.so not built at {LIB_PATH}; run __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _order_after_torch(ctx, *arrays):
    """Device arrays written by torch on another stream must be complete before the
    context's stream reads them: synchronise torch's current stream unless the
    context launches on it."""
    if any(a is not None and not isinstance(a, np.ndarray) for a in arrays):
        import torch
        cur = torch.cuda.current_stream()
        if cur.cuda_stream != ctx.stream_ptr:
            cur.synchronize()


def _ptr(a):
    """Address of a numpy array (host) or a torch tensor (device)."""
    if isinstance(a, np.ndarray):
        assert a.flags.c_contiguous
        return a.ctypes.data
    return a.data_ptr()


class Context:
    """An srmg context bound to one device with a tree uploaded."""

    def __init__(self, device: int = 0, D: int = 2):
        self._h = _P()
        self.D = D
        rc = lib().srmg_create(ctypes.byref(self._h), D, 16, 2, device)
        if rc != SRMG_OK:
            raise SrmgError(rc, "srmg_create failed")
        self._tree_keep = None
        self.generation = 0
        self.stream_ptr = -1  # the context's own stream

    def close(self):
        if self._h:
            lib().srmg_destroy(self._h)
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def check(self, rc):
        if rc != SRMG_OK:
            msg = lib().srmg_last_error(self._h)
            raise SrmgError(rc, msg.decode() if msg else "")

    def set_tree(self, tree: Tree, conn: Connectivity, generation: int | None = None):
        nlev = len(tree)
        keep = []

        def arrs(lists):
            lists = [np.ascontiguousarray(x) for x in lists]
            keep.extend(lists)
            n = (ctypes.c_int64 * nlev)(*[len(x) for x in lists])
            p = (_P * nlev)(*[x.ctypes.data if len(x) else 0 for x in lists])
            keep.extend([n, p])
            return ctypes.cast(n, _P), ctypes.cast(p, _P)

        pairs = arrs([layer.pairs_array() for layer in tree])
        nb = arrs(conn.neighbor)
        bd = arrs(conn.boundary)
        rb = arrs(conn.refboundary)
        ch = arrs(conn.child)
        self.generation = (self.generation + 1) if generation is None else generation
        f = lib().srmg_set_tree3 if getattr(tree, "D", 2) == 3 else lib().srmg_set_tree
        self.check(f(self._h, nlev, *pairs, *nb, *bd, *rb, *ch, self.generation))
        self._tree_keep = keep
        return self

    def set_option(self, key: str, value: int):
        self.check(lib().srmg_set_option(self._h, key.encode(), int(value)))
        return self

    def trace(self):
        """Phase timestamps (ns) of the last persistent-kernel launch."""
        out = np.zeros(1024, dtype=np.int64)
        n = lib().srmg_get_trace(self._h, out.ctypes.data, len(out))
        if n < 0:
            self.check(n)
        return out[:n].copy()

    def launches(self) -> int:
        return lib().srmg_launch_count(self._h)

    def synchronize(self):
        self.check(lib().srmg_synchronize(self._h))

    def set_stream(self, stream_ptr: int | None):
        self.check(lib().srmg_set_stream(self._h, stream_ptr or None))
        self.stream_ptr = stream_ptr if stream_ptr else -1


def _bc(bc):
    """The boundary table: 9 entries (D = 2) or 27 (D = 3), column-major."""
    a = np.ascontiguousarray(np.asarray(bc, dtype=np.int8).reshape(-1))
    if a.size not in (9, 27):
        raise ValueError("a boundary table has 9 (D = 2) or 27 (D = 3) entries")
    return a


def _disc(lpldisc):
    """(op, k2) from a discretisation descriptor: None/'laplacian' (LaplacianDiscretization
    {2,2}), ('helmholtz', k2) (HelmholtzDiscretization{2,2}(k2)) or 'laplacian4'
    (LaplacianDiscretization{2,4}, the compact order-4 scheme)."""
    if lpldisc is None or lpldisc == "laplacian" or lpldisc == 0:
        return 0, 0.0
    if lpldisc == "laplacian4" or lpldisc == 2:
        return 2, 0.0
    if isinstance(lpldisc, tuple) and lpldisc[0] in ("helmholtz", 1):
        return 1, float(lpldisc[1])
    raise ValueError(f"unsupported discretisation {lpldisc!r}")


def vcycle_(ctx: Context, u, b, r, u1, s, geometry, bc, lpldisc=None, lmax=0, ndown=3, ntop=5,
            nup=3, omega=1.0, ncycles=1):
    """vcycle!(u, b, r, u1, s, tree, conn, geometry, bc, lpldisc; ...) (src/multigrid.jl:60)."""
    op, k2 = _disc(lpldisc)
    bca = _bc(bc)
    dev = not isinstance(u, np.ndarray)
    _order_after_torch(ctx, u, b, r, u1)
    f = lib().srmg_vcycle_dev if dev else lib().srmg_vcycle
    ctx.check(f(ctx.handle, _ptr(u), _ptr(b), _ptr(r), _ptr(u1), u.shape[0], s, op, k2, geometry,
                bca.ctypes.data, lmax, ndown, ntop, nup, omega, ncycles))


def fmg_(ctx: Context, u, b, r, u1, s, geometry, bc, lpldisc=None, ndown=3, ntop=5, nup=3,
         omega=1.25):
    """fmg!(u, b, r, u1, s, tree, conn, geometry, bc, lpldisc; ...) (src/multigrid.jl:17)."""
    op, k2 = _disc(lpldisc)
    bca = _bc(bc)
    dev = not isinstance(u, np.ndarray)
    _order_after_torch(ctx, u, b, r, u1)
    f = lib().srmg_fmg_dev if dev else lib().srmg_fmg
    ctx.check(f(ctx.handle, _ptr(u), _ptr(b), _ptr(r), _ptr(u1), u.shape[0], s, op, k2, geometry,
                bca.ctypes.data, ndown, ntop, nup, omega))


def resnorm(ctx: Context, r, b, u, s, geometry, bc, lpldisc=None) -> float:
    """resnorm!(r, b, u, s, tree, conn, geometry, bc, lpldisc) (src/multigrid.jl:391)."""
    op, k2 = _disc(lpldisc)
    bca = _bc(bc)
    out = ctypes.c_double()
    dev = not isinstance(u, np.ndarray)
    _order_after_torch(ctx, r, b, u)
    f = lib().srmg_resnorm_dev if dev else lib().srmg_resnorm
    ctx.check(f(ctx.handle, _ptr(r) if r is not None else None, _ptr(b), _ptr(u), u.shape[0], s,
                op, k2, geometry, bca.ctypes.data, ctypes.byref(out)))
    return out.value


def fill_ghost_(ctx: Context, u, l, bc, mask=7):
    """fill_ghost!(u, l, conn, bc) (src/connectivity.jl:155-159)."""
    bca = _bc(bc)
    if isinstance(u, np.ndarray):
        ctx.check(lib().srmg_fill_ghost(ctx.handle, _ptr(u), u.shape[0], l, bca.ctypes.data))
    else:
        _order_after_torch(ctx, u)
        ctx.check(lib().srmg_fill_ghost_dev(ctx.handle, _ptr(u), u.shape[0], l, bca.ctypes.data, mask))


def netcharge(ctx: Context, q, ne, nion):
    """netcharge!(tree, q, n, chem) for NetIonization (src/streamer.jl:369-373): q = -ne + nion
    on every valid cell.  numpy (host) or torch (device) fields of one kind."""
    if isinstance(q, np.ndarray):
        ctx.check(lib().srmg_netcharge(ctx.handle, _ptr(q), _ptr(ne), _ptr(nion), q.shape[0]))
    else:
        _order_after_torch(ctx, q, ne, nion)
        ctx.check(lib().srmg_netcharge_dev(ctx.handle, _ptr(q), _ptr(ne), _ptr(nion), q.shape[0]))


def rhs_level_(ctx: Context, q1, q, l, geometry, lpldisc=None):
    """rhs_level!(q1, q, tree[l], lpldisc, geometry) (src/multigrid.jl:363-388): q1 = R q
    on level l (identity at order 2, the compact right-hand side at order 4)."""
    op, _ = _disc(lpldisc)
    if isinstance(q1, np.ndarray):
        ctx.check(lib().srmg_rhs_level(ctx.handle, _ptr(q1), _ptr(q), q1.shape[0], l, op, geometry))
    else:
        _order_after_torch(ctx, q1, q)
        ctx.check(lib().srmg_rhs_level_dev(ctx.handle, _ptr(q1), _ptr(q), q1.shape[0], l, op, geometry))


def freebc_set(ctx: Context, dim, level, rootsize, f):
    """FreeBC(CylindricalGeometry{dim}, u, level, rootsize, h) (src/freebc.jl:29-53): hand
    the library the transform kernel f (computed as FreeBC does)."""
    fa = np.ascontiguousarray(f, dtype=np.float64)
    ra = np.ascontiguousarray(rootsize, dtype=np.int64)
    ctx.check(lib().srmg_freebc_set(ctx.handle, dim, level, ra.ctypes.data, fa.ctypes.data, len(fa)))


def freebc_(ctx: Context, q, u, h, s, b_out=None):
    """freebc!(q, u, h, s, tree, conn, conf) (src/freebc.jl:83-105): q += boundary sources
    from the homogeneous potential u.  numpy (host) or torch (device) fields; b_out
    receives conf.b (numpy for host fields, a torch tensor for device fields)."""
    if isinstance(q, np.ndarray):
        bp = b_out.ctypes.data if b_out is not None else None
        ctx.check(lib().srmg_freebc(ctx.handle, _ptr(q), _ptr(u), q.shape[0], h, s, bp))
    else:
        _order_after_torch(ctx, q, u)
        bp = b_out.data_ptr() if b_out is not None else None
        ctx.check(lib().srmg_freebc_dev(ctx.handle, _ptr(q), _ptr(u), q.shape[0], h, s, bp))


def fill_ghost_free_(ctx: Context, u, l):
    """fill_ghost_free!(u, conf, tree, l) (src/freebc.jl:224-243)."""
    if isinstance(u, np.ndarray):
        ctx.check(lib().srmg_fill_ghost_free(ctx.handle, _ptr(u), u.shape[0], l))
    else:
        _order_after_torch(ctx, u)
        ctx.check(lib().srmg_fill_ghost_free_dev(ctx.handle, _ptr(u), u.shape[0], l))


def restrict_full_(ctx: Context, u):
    """restrict_full!(u, conn) (src/restrict.jl:43-47) on a device field."""
    _order_after_torch(ctx, u)
    ctx.check(lib().srmg_restrict_full_dev(ctx.handle, _ptr(u), u.shape[0]))


def electric_field(ctx: Context, e, eabs, u, h, e0):
    """electric_field!(tree, e, eabs, u, h, t, e0) with a constant background field e0 =
    (e0_r, e0_z) (src/multigrid.jl:421-451).  e: [nblk, 2, 21, 21] (VectorBlockField
    storage), eabs and u: [nblk, 20, 20]; numpy (host) or torch (device)."""
    e0a = np.ascontiguousarray(e0, dtype=np.float64)
    if isinstance(u, np.ndarray):
        ctx.check(lib().srmg_electric_field(ctx.handle, _ptr(e), _ptr(eabs), _ptr(u), u.shape[0], float(h),
                                            e0a.ctypes.data))
    else:
        _order_after_torch(ctx, e, eabs, u)
        ctx.check(lib().srmg_electric_field_dev(ctx.handle, _ptr(e), _ptr(eabs), _ptr(u), u.shape[0], float(h),
                                                e0a.ctypes.data))


def solve(ctx: Context, u, b, s, geometry, bc, lpldisc=None, tol=1e-8, mode=MODE_FP64,
          max_cycles=1000, ndown=2, ntop=4, nup=2, omega=1.0, inner_cycles=2, warm_start=0):
    """Solve L u + s b = 0 to resnorm(u)/leafnorm(b) <= tol; returns the stats dict."""
    op, k2 = _disc(lpldisc)
    bca = _bc(bc)
    o = SolveOpts(tol, max_cycles, mode, ndown, ntop, nup, omega, inner_cycles, warm_start)
    st = Stats()
    dev = not isinstance(u, np.ndarray)
    _order_after_torch(ctx, u, b)
    f = lib().srmg_solve_dev if dev else lib().srmg_solve
    rc = f(ctx.handle, _ptr(u), _ptr(b), u.shape[0], s, op, k2, geometry, bca.ctypes.data,
           ctypes.byref(o), ctypes.byref(st))
    ctx.check(rc)
    return st.as_dict()


def solve_async(ctx: Context, u, b, s, geometry, bc, lpldisc=None, tol=1e-8, mode=MODE_FP64,
                max_cycles=1000, ndown=2, ntop=4, nup=2, omega=1.0, inner_cycles=2):
    """srmg_solve_async on host arrays (numpy, page-locked for overlap): enqueues the
    copies in, the solve and the copy out on the context's stream and returns at once.
    u and b must stay alive and untouched until solve_wait(ctx)."""
    assert isinstance(u, np.ndarray) and isinstance(b, np.ndarray)
    op, k2 = _disc(lpldisc)
    bca = _bc(bc)
    o = SolveOpts(tol, max_cycles, mode, ndown, ntop, nup, omega, inner_cycles, 0)
    ctx.check(lib().srmg_solve_async(ctx.handle, _ptr(u), _ptr(b), u.shape[0], s, op, k2, geometry,
                                     bca.ctypes.data, ctypes.byref(o)))


def solve_wait(ctx: Context):
    """Waits for the context's srmg_solve_async; returns its stats dict."""
    st = Stats()
    ctx.check(lib().srmg_solve_wait(ctx.handle, ctypes.byref(st)))
    return st.as_dict()


class Batch(Context):
    """A batch context: a forest of independent problems solved by one persistent launch.

    ``problems`` is a list of ``(tree_context, s, lpldisc, bc)``; the same tree context
    may appear several times (e.g. the Poisson potential and the three photoionization
    Helmholtz terms of one tree).  No single counterpart in the reference, which calls
    vcycle!/fmg! once per field (src/streamer.jl:322-334, src/photo.jl)."""

    def __init__(self, problems, geometry, device: int = 0):
        super().__init__(device)
        items = (Item * len(problems))()
        for i, (tctx, s, lpldisc, bc) in enumerate(problems):
            op, k2 = _disc(lpldisc)
            items[i].tree = tctx.handle.value
            items[i].s = float(s)
            items[i].op = op
            items[i].k2 = k2
            items[i].bc[:] = [int(v) for v in _bc(bc)]
        self.check(lib().srmg_batch_set(self._h, len(problems), items, int(geometry)))
        self.nitems = len(problems)
        self.offsets = [lib().srmg_batch_offset(self._h, i) for i in range(self.nitems)]
        self.nblks = [lib().srmg_batch_nblk(self._h, i) for i in range(self.nitems)]
        self.total_blocks = sum(self.nblks)

    def solve(self, us, bs, tol=1e-8, mode=MODE_FP64, max_cycles=1000, ndown=2, ntop=4, nup=2,
              omega=1.0, inner_cycles=2, warm_start=0):
        """Solve every item; ``us``/``bs`` are per-item fields (numpy arrays: host entry
        point; torch tensors: device entry point).  Returns one stats dict per item."""
        assert len(us) == self.nitems and len(bs) == self.nitems
        o = SolveOpts(tol, max_cycles, mode, ndown, ntop, nup, omega, inner_cycles, warm_start)
        st = (Stats * self.nitems)()
        up = (_P * self.nitems)(*[_ptr(x) for x in us])
        bp = (_P * self.nitems)(*[_ptr(x) for x in bs])
        dev = not isinstance(us[0], np.ndarray)
        _order_after_torch(self, *us, *bs)
        f = lib().srmg_batch_solve_dev if dev else lib().srmg_batch_solve
        self.check(f(self._h, ctypes.cast(up, _P), ctypes.cast(bp, _P), ctypes.byref(o), st))
        return [x.as_dict() for x in st]

    def solve_forest(self, u, b, tol=1e-8, mode=MODE_FP64, max_cycles=1000, ndown=2, ntop=4, nup=2,
                     omega=1.0, inner_cycles=2, warm_start=0):
        """Solve every item on device fields in the forest layout (no copies)."""
        o = SolveOpts(tol, max_cycles, mode, ndown, ntop, nup, omega, inner_cycles, warm_start)
        st = (Stats * self.nitems)()
        _order_after_torch(self, u, b)
        self.check(lib().srmg_batch_solve_forest_dev(self._h, _ptr(u), _ptr(b), ctypes.byref(o), st))
        return [x.as_dict() for x in st]


def autotune(ctx: Context, u, b, s, geometry, bc, lpldisc=None, tol=1e-8, mode=MODE_MIXED,
             max_cycles=1000, ndown=2, ntop=4, nup=2, omega=1.0, inner_cycles=2):
    """Autotune launch shape and sweep counts on this problem (device fields); returns
    (chosen options dict, list of trial dicts).  The chosen launch options stay set on
    the context."""
    op, k2 = _disc(lpldisc)
    bca = _bc(bc)
    o = SolveOpts(tol, max_cycles, mode, ndown, ntop, nup, omega, inner_cycles, 0)
    tr = (TuneTrial * 64)()
    _order_after_torch(ctx, u, b)
    n = lib().srmg_autotune(ctx.handle, _ptr(u), _ptr(b), u.shape[0], s, op, k2, geometry, bca.ctypes.data,
                            ctypes.byref(o), tr, 64)
    if n < 0:
        ctx.check(n)
    chosen = {k: getattr(o, k) for k, _ in SolveOpts._fields_}
    return chosen, [tr[i].as_dict() for i in range(min(n, 64))]


def batch_autotune(batch: "Batch", us, bs, tol=1e-8, mode=MODE_MIXED, max_cycles=1000, ndown=2, ntop=4,
                   nup=2, omega=1.0, inner_cycles=2):
    """Autotune a batch on its items' device fields; returns (options, trials)."""
    o = SolveOpts(tol, max_cycles, mode, ndown, ntop, nup, omega, inner_cycles, 0)
    tr = (TuneTrial * 64)()
    up = (_P * batch.nitems)(*[_ptr(x) for x in us])
    bp = (_P * batch.nitems)(*[_ptr(x) for x in bs])
    _order_after_torch(batch, *us, *bs)
    n = lib().srmg_batch_autotune(batch.handle, ctypes.cast(up, _P), ctypes.cast(bp, _P), ctypes.byref(o), tr, 64)
    if n < 0:
        batch.check(n)
    chosen = {k: getattr(o, k) for k, _ in SolveOpts._fields_}
    return chosen, [tr[i].as_dict() for i in range(min(n, 64))]


class Cnn:
    """The learned warm-start network (BF16, tensor-core kernels of libsrmg)."""

    def __init__(self, device: int = 0, seed: int = 0):
        self._h = _P()
        rc = lib().srmg_cnn_create(ctypes.byref(self._h), device, seed)
        if rc != SRMG_OK:
            raise SrmgError(rc, "srmg_cnn_create failed")
        self.device = device
        self.nparams = lib().srmg_cnn_nparams()

    def close(self):
        if self._h:
            lib().srmg_cnn_destroy(self._h)
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def check(self, rc):
        if rc != SRMG_OK:
            msg = lib().srmg_cnn_last_error(self._h)
            raise SrmgError(rc, msg.decode() if msg else "")

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.nparams, dtype=np.float32)
        self.check(lib().srmg_cnn_get_params(self._h, out.ctypes.data, self.nparams))
        return out

    def set_params(self, theta):
        a = np.ascontiguousarray(theta, dtype=np.float32)
        assert a.size == self.nparams
        self.check(lib().srmg_cnn_set_params(self._h, a.ctypes.data, self.nparams))

    def synchronize(self):
        self.check(lib().srmg_cnn_synchronize(self._h))

    def forward(self, x):
        """x: torch bf16 [n, 400, 2] on the device -> torch float32 [n, 256]."""
        import torch
        n = x.shape[0]
        y = torch.empty((n, 256), dtype=torch.float32, device=x.device)
        torch.cuda.synchronize()
        self.check(lib().srmg_cnn_forward(self._h, x.data_ptr(), y.data_ptr(), n))
        self.synchronize()
        return y

    def gradients(self, x, t, ir0=None, lam=0.0, geom=1):
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = ctypes.c_double()
        import torch
        torch.cuda.synchronize()
        self.check(lib().srmg_cnn_gradients(self._h, x.data_ptr(), t.data_ptr(),
                                            ir0.data_ptr() if ir0 is not None else None, float(lam), int(geom),
                                            x.shape[0], g.ctypes.data, ctypes.byref(loss)))
        return loss.value, g

    def train_step(self, x, t, lr, ir0=None, lam=0.0, geom=1):
        """One Adam step; returns the loss of the batch before the step."""
        loss = ctypes.c_double()
        self.check(lib().srmg_cnn_train_step(self._h, x.data_ptr(), t.data_ptr(),
                                             ir0.data_ptr() if ir0 is not None else None, float(lam), int(geom),
                                             x.shape[0], float(lr), ctypes.byref(loss)))
        return loss.value


def _cnn_forward_train(self, x):
    """Forward keeping activations; returns y (torch float32 [n, 256])."""
    import torch
    y = torch.empty((x.shape[0], 256), dtype=torch.float32, device=x.device)
    torch.cuda.synchronize()
    self.check(lib().srmg_cnn_forward_train(self._h, x.data_ptr(), x.shape[0], y.data_ptr()))
    return y


def _cnn_backward_step(self, dy, lr, want_grad=False):
    """Backward from dLoss/dy of the last forward_train; Adam step when lr > 0."""
    import torch
    g = np.zeros(self.nparams, dtype=np.float32) if want_grad else None
    dy = dy.contiguous()
    torch.cuda.synchronize()
    self.check(lib().srmg_cnn_backward_step(self._h, dy.data_ptr(), dy.shape[0], float(lr),
                                            g.ctypes.data if want_grad else None))
    return g


def _cnn_forward_tc(self, x):
    """Inference forward on the tcgen05 tensor cores: x torch bf16 [n, 400, 2] -> float32 [n, 256]."""
    import torch
    n = x.shape[0]
    y = torch.empty((n, 256), dtype=torch.float32, device=x.device)
    torch.cuda.synchronize()
    self.check(lib().srmg_cnn_forward_tc(self._h, x.data_ptr(), y.data_ptr(), n))
    self.check(lib().srmg_cnn_tc_status(self._h))
    return y


def _cnn_use_tcgen05(self, enable=True):
    self.check(lib().srmg_cnn_use_tcgen05(self._h, int(enable)))
    return self


Cnn.forward_tc = _cnn_forward_tc
Cnn.use_tcgen05 = _cnn_use_tcgen05
Cnn.forward_train = _cnn_forward_train
Cnn.backward_step = _cnn_backward_step


def cnn_pack(ctx: Context, f, g, s, geometry, bc, lpldisc=None):
    """Samples of a tree for the network from input fields f and g:
    (x bf16 [n,400,2], scale float64 [n], blk int32 [n])."""
    import torch
    op, k2 = _disc(lpldisc)
    bca = _bc(bc)
    n = lib().srmg_cnn_leaf_blocks(ctx.handle)
    dev = f.device
    x = torch.empty((n, 400, 2), dtype=torch.bfloat16, device=dev)
    scale = torch.empty(n, dtype=torch.float64, device=dev)
    blk = torch.empty(n, dtype=torch.int32, device=dev)
    _order_after_torch(ctx, f, g)
    rc = lib().srmg_cnn_pack_dev(ctx.handle, f.data_ptr(), g.data_ptr(), f.shape[0], s, op, k2, geometry,
                                 bca.ctypes.data, x.data_ptr(), scale.data_ptr(), blk.data_ptr(), n)
    if rc < 0:
        ctx.check(rc)
    ctx.synchronize()
    return x, scale, blk


def cnn_predict(ctx: Context, net: Cnn, u, b, b1, phi2, b2, s, geometry, bc, lpldisc=None, resid=False):
    """Warm start in place on u (phi_{n-1} on entry); returns which guess was kept:
    0 the previous potential, 1 the extrapolation, 2 the learned guess (and, with
    resid=True, the three candidates' residual norms)."""
    op, k2 = _disc(lpldisc)
    bca = _bc(bc)
    which = ctypes.c_int()
    r3 = (_D * 3)()
    _order_after_torch(ctx, u, b, b1, phi2, b2)
    ctx.check(lib().srmg_cnn_predict_dev(ctx.handle, net.handle, u.data_ptr(), b.data_ptr(), b1.data_ptr(),
                                         phi2.data_ptr(), b2.data_ptr(), u.shape[0], s, op, k2, geometry,
                                         bca.ctypes.data, ctypes.byref(which), r3))
    return (which.value, list(r3)) if resid else which.value


def exported_symbols_from_header(header_path: str) -> list[str]:
    """Names of the functions declared in include/srmg.h."""
    import re
    text = open(header_path).read()
    return sorted(set(re.findall(r"\b(srmg_[a-z0-9_]+)\s*\(", text)))
