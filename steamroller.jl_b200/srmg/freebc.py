"""The free-boundary transform kernel, computed on the host as FreeBC does
(src/freebc.jl:29-53): the caller hands f to the library once (srmg_freebc_set /
multigrid.freebc_set).

For the outer column along `dim` of a tree with root grid `rootsize` at level `level`
(finest-level cell size h / 2^(level-1)): n = rootsize[other] 16 2^(level-1) transform
points, H = rootsize[other] 16 h the domain length along the other dimension,
R = rootsize[dim] 16 h the radius, k_j = (pi / H) j (j = 1..n), and
f_j = (2 / H) / (k_j (I1(k_j R) / I0(k_j R) + K1(k_j R) / K0(k_j R))), the modified
Bessel ratios taken from the exponentially scaled functions (their scale factors
cancel within each ratio).
"""
from __future__ import annotations

import numpy as np
import scipy.special

M = 16  # valid cells per block side


def kernel(dim: int, level: int, rootsize, h: float):
    """(n, H, R, f) of FreeBC(geometry along `dim`, level, rootsize, h)."""
    other = 2 if dim == 1 else 1
    n = int(rootsize[other - 1]) * 2 ** (level - 1) * M
    H = rootsize[other - 1] * h * M
    R = rootsize[dim - 1] * h * M
    k = (np.pi / H) * np.arange(1, n + 1)
    x = k * R
    ratio = scipy.special.i1e(x) / scipy.special.i0e(x) + scipy.special.k1e(x) / scipy.special.k0e(x)
    return n, H, R, (2 / H) / (k * ratio)
