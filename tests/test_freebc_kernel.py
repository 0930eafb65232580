"""The host-side free-boundary kernel of the Python API (srmg.freebc.kernel, FreeBC's
f, src/freebc.jl:29-53) equals the oracle's restatement bit for bit, for both boundary
dimensions and oblong root grids."""
import numpy as np
import pytest

import freebc_oracle as fo
from srmg import freebc


@pytest.mark.parametrize("dim,level,rootsize,h", [(1, 9, (1, 1), 1e-4), (2, 6, (1, 2), 3e-5), (1, 7, (2, 1), 1e-3),
                                                  (2, 11, (3, 1), 2e-6)])
def test_kernel_matches_oracle(dim, level, rootsize, h):
    got = freebc.kernel(dim, level, rootsize, h)
    want = fo.kernel(dim, level, rootsize, h)
    assert got[:3] == want[:3]
    assert np.array_equal(got[3].view(np.uint64), want[3].view(np.uint64))
    assert np.all(got[3] > 0)
