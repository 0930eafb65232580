"""Seeded streamer runs on config-1-sized trees that generate (phi_prev, b_prev, b,
phi_new) solve pairs for the learned warm start.

A run: the uniform level-5 tree (256 x 256 cells on 16 x 16 leaf blocks, L = 1.25 cm,
cylindrical r-z), an elongated neutral electron/ion seed column on the axis near the
top electrode over a uniform background, and a uniform applied field of 1.5 MV/m.  Every step moves the
densities with libsrmg's stepper kernel (Koren-limited electron drift-diffusion,
ionisation and attachment into two immobile ion species), forms the net charge
b = n+ - ne - n- (restricted onto the coarse levels, restrict_full!,
src/streamer.jl:313), and solves the Poisson equation with libsrmg's mixed-precision
solve from the previous potential -- one solve pair per step.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import gen
from . import multigrid as mg

MU_E = 0.0372          # electron mobility in air, m^2/(V s)
D_E = 0.18             # electron diffusion, m^2/s
ALPHA_A, ALPHA_B = 4.332e5, 1.41e7   # alpha(E) = A exp(-B/E), 1/m (gen.townsend_alpha)
ETA = 500.0            # attachment, 1/m
E_APPLIED = 1.5e6      # V/m
BC_DENSITY = np.ones(9, dtype=np.int8)  # zero-gradient ghosts for the densities


class Streamer:
    def __init__(self, seed: int, device: int = 0, level: int = 5, E0: float = E_APPLIED,
                 background: float = 1e13, cfl: float = 0.4, problem=None, stream=None):
        """A seeded run on the uniform tree of `level`, or on `problem`'s tree: then the
        densities start as a neutral conducting plasma where the problem's charge is
        (n_e = background + 10 |b|, n+ = n_e + b, so the initial net charge is b)."""
        import torch
        self.rng = np.random.default_rng(seed)
        given = problem is not None
        if not given:
            self.tree = gen._uniform(level)
            problem = gen.make_problem(self.tree, lambda r, z, l, gi, gj: np.zeros_like(r), gen.poisson_scale())
        self.tree = problem.tree
        self.problem = problem
        p = self.problem
        self.s, self.geom, self.bc = p.s, p.geom, p.bc
        self.h1 = p.h1
        self.E0 = E0
        self.cfl = cfl
        self.ctx = mg.Context(device).set_tree(p.tree, p.conn)
        if stream is not None:
            self.ctx.set_stream(stream.cuda_stream)
        self.nblk = p.nblk
        dev = torch.device("cuda", device)
        z = lambda: torch.zeros((self.nblk, 20, 20), dtype=torch.float64, device=dev)
        self.ne, self.npos, self.nneg, self.phi, self.b = z(), z(), z(), z(), z()
        self.work = torch.zeros(3 * self.nblk * 400 + 2, dtype=torch.float64, device=dev)
        if given:
            bh = p.b.copy()
            leaf = np.zeros(bh.shape, dtype=bool)
            for layer in self.tree:
                for cc, blk in layer.index.items():
                    if self.tree.isleaf(layer.level, cc):
                        leaf[blk - 1, 2:18, 2:18] = True
            ne = np.where(leaf, background + 10.0 * np.abs(bh), 0.0)
            npos = np.where(leaf, ne + bh, 0.0)
            self.ne.copy_(torch.from_numpy(ne))
            self.npos.copy_(torch.from_numpy(npos))
            self.t = 0.0
            self._charge()
            torch.cuda.synchronize()
            mg.solve(self.ctx, self.phi, self.b, self.s, self.geom, self.bc, tol=1e-8, mode=mg.MODE_MIXED)
            return
        # seed: an elongated neutral plasma column on the axis hanging from near the top
        # electrode (Gaussian radial profile and ends), length, radius, density and
        # position jittered
        L = gen.L_DOMAIN
        z0 = L - self.rng.uniform(0.3e-3, 1.0e-3)
        length = self.rng.uniform(1.5e-3, 3.0e-3)
        w = self.rng.uniform(0.2e-3, 0.4e-3)
        amp = 10 ** self.rng.uniform(19.5, 20.5)
        lev = len(self.tree)
        blks, r, zz, _, _ = gen.block_cell_centres(self.tree, lev, self.h1)
        dz = np.maximum(0.0, np.maximum(zz - z0, (z0 - length) - zz))
        n0 = background + amp * np.exp(-(r * r + dz * dz) / (w * w))
        ne = np.zeros((self.nblk, 20, 20))
        ne[blks - 1, 2:18, 2:18] = n0
        self.ne.copy_(torch.from_numpy(ne))
        self.npos.copy_(torch.from_numpy(ne))
        self.t = 0.0
        self._charge()
        torch.cuda.synchronize()
        mg.solve(self.ctx, self.phi, self.b, self.s, self.geom, self.bc, tol=1e-10, mode=mg.MODE_FP64)

    def _charge(self):
        """b = n+ - ne - n- on the leaves, restricted onto every coarser level."""
        import torch
        self.b.copy_(self.npos - self.ne - self.nneg)
        torch.cuda.synchronize()
        for l in range(len(self.tree), 1, -1):
            self.ctx.check(mg.lib().srmg_restrict_level_dev(self.ctx.handle, self.b.data_ptr(), self.nblk, l))
        self.ctx.synchronize()

    def step(self, dt_max: float = 1e-10, mode=mg.MODE_MIXED, tol=1e-8):
        """Advance one step; returns (phi_prev, b_prev, stats of the new solve)."""
        phi_prev, b_prev = self.advance(dt_max)
        st = mg.solve(self.ctx, self.phi, self.b, self.s, self.geom, self.bc, tol=tol, mode=mode)
        return phi_prev, b_prev, st

    def advance(self, dt_max: float = 1e-10):
        """Move the densities one step and form the new charge; the potential is left at
        its previous value for the caller to solve.  Returns (phi_prev, b_prev)."""
        import torch
        torch.cuda.synchronize()
        for l in range(1, len(self.tree) + 1):
            mg.fill_ghost_(self.ctx, self.ne, l, BC_DENSITY)
        dt = ctypes.c_double()
        self.ctx.check(mg.lib().srmg_streamer_step_dev(
            self.ctx.handle, self.ne.data_ptr(), self.npos.data_ptr(), self.nneg.data_ptr(), self.phi.data_ptr(),
            self.nblk, self.h1, self.E0, MU_E, D_E, ALPHA_A, ALPHA_B, ETA, self.cfl, dt_max, self.work.data_ptr(),
            ctypes.byref(dt)))
        self.ctx.synchronize()
        self.t += dt.value
        phi_prev, b_prev = self.phi.clone(), self.b.clone()
        self._charge()
        return phi_prev, b_prev

    def ir0_of_blocks(self):
        """Global r index before the first cell of every block, by 0-based block id."""
        import torch
        t = np.zeros(self.nblk, dtype=np.int32)
        for layer in self.tree:
            for (cr, cz), blk in layer.index.items():
                t[blk - 1] = 16 * (cr - 1)
        return torch.from_numpy(t).to(self.phi.device)

    def front_z(self) -> float:
        """Lowest z where ne exceeds 1e18 m^-3 on the axis column (the streamer tip)."""
        ne = self.ne.cpu().numpy()
        lev = len(self.tree)
        blks, r, zz, _, _ = gen.block_cell_centres(self.tree, lev, self.h1)
        v = ne[blks - 1, 2:18, 2:18]
        m = (v > 1e18) & (r < 2 * self.h1 / 16)
        return float(zz[m].min()) if m.any() else math.nan
