"""Algorithmic-bytes model of one FAS V-cycle, used for roofline fractions.

With n_l the valid cells of level l (all blocks of the level, leaves and parents),
w the bytes per value and (nd, nu, ntop) the sweep counts:

  B = sum_{l=2..L} [ w n_l (3(nd+nu) + 8.5) + 5 w n_{l-1} ] + 3 w ntop n_1

Terms: each Gauss-Seidel iteration reads u and b and writes u (3w per cell); the
residual reads u, b and writes r (3w); restricting u and r reads 2w per fine cell and
writes 2 w/4; the FAS right-hand side writes 3w/4; prolongation-add reads the fine u
and writes it (2w) and reads w/4 of the coarse correction; the coarse copy u1 = u costs
2w and the difference u1 = u - u1 costs 3w per coarse cell.  Ghost fills are not
counted.  For (2,2,4) in FP64: 164 B per level-l cell + 40 B per level-(l-1) cell.
"""
from __future__ import annotations


def level_cells(tree, M=16):
    """Valid cells per level: M^D per block (D from the tree, 2 by default)."""
    D = getattr(tree, "D", 2)
    return [len(layer.index) * M ** D for layer in tree]


def vcycle_bytes(tree, w=8, ndown=2, nup=2, ntop=4, M=16):
    n = level_cells(tree, M)
    L = max((i + 1 for i, x in enumerate(n) if x), default=0)
    total = 0.0
    for l in range(2, L + 1):
        total += w * n[l - 1] * (3 * (ndown + nup) + 8.5) + 5 * w * n[l - 2]
    total += 3 * w * ntop * (n[0] if n else 0)
    return total


def mixed_solve_bytes(tree, cycles, steps, ndown=2, nup=2, ntop=4, M=16):
    """Algorithmic bytes of one mixed-precision solve (one persistent launch).

    `cycles` FP32 V-cycles (w = 4) plus the FP64 side of the defect correction, with N
    the valid cells of all levels and N2 those of levels >= 2:
      * steps + 1 defect passes: read u64 and b64, write the FP32 right-hand side and
        zero the FP32 correction (24 B per cell);
      * steps + 1 restrictions of u64 onto the covered subblocks (8 B read per fine
        cell + 8/4 B written: 10 B per cell of levels >= 2);
      * steps updates u64 += e: read u64 and e, write u64 (20 B per cell).
    The coarsest level's direct solve (one 256 x 256 FP64 matrix-vector product per
    item) replaces the ntop sweeps; both are negligible next to the finer levels.
    """
    n = level_cells(tree, M)
    N = float(sum(n))
    N2 = float(sum(n[1:]))
    fp64 = (steps + 1) * (24.0 * N + 10.0 * N2) + steps * 20.0 * N
    return cycles * vcycle_bytes(tree, 4, ndown, nup, ntop, M) + fp64
