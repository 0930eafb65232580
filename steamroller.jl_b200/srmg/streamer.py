"""Seeded streamer runs that generate (phi_prev, b_prev, b, phi_new) solve pairs for the
learned warm start, stepped the way the reference's step! does it (src/streamer.jl:
386-425): SSPRK3, each of its three stages one derivs! (src/streamer.jl:292-366).

A stage, all on the device through libsrmg (`_charge`, the solve, `_rates`):
  netcharge! (NetIonization: q = n_ion - n_e), restrict_full!(q), the Poisson solve
  (mixed precision to a tolerance, or the reference's fixed V-cycle count), restrict_full!
  (n_e), ghost fills of n_e (copy, Neumann fluid table, InterpCopy refinement ghosts),
  electric_field! with the applied background field, fill_ghost!(eabs,
  ExtrapolateConst), flux! (Koren) + restrict_flux!, chemderivs! + fluxderivs!.
The species are the NetIonization pair (electrons, net positive ions) with the
reference's MinimalTransportModel and no photoionization (the reference's defaults,
src/simulate.jl:5-11, 86-94).  The time step is min(tmax - t, 0.8 x the smallest
stable step of the first stage's flux!) as in step!.

A run: the uniform level-5 tree (256 x 256 cells on 16 x 16 leaf blocks, L = 1.25 cm,
cylindrical r-z), an elongated neutral plasma seed column on the axis near the lower
electrode over a uniform background, and the reference's default background field
eb = (0, -18.75 kV / 1.25 cm) = (0, -1.5 MV/m), so that electrons drift upwards.  Or, with
`problem`, that problem's (refined) tree with the densities of a neutral conducting
plasma where the problem's charge is.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import gen
from . import multigrid as mg

# MINIMAL_TRANSPORT_MODEL (src/simulate.jl:5-10)
MINIMAL = dict(mu=0.0372193, D=0.18, ai=433200.0, Ei=2e7, aa=2000.0, Ea=3e6)
E_BACKGROUND = (0.0, -18.75e3 / 1.25e-2)  # eb (src/simulate.jl:84), V/m
BC_DENSITY = np.ones(9, dtype=np.int8)    # fbc = boundaryconditions(((1, 1), (1, 1))) (src/simulate.jl:251-253)
BC_EXTRAPOLATE = np.ones(9, dtype=np.int8)  # ExtrapolateConst: ghost = closest valid cell
DT_SAFETY = 0.8                           # dt_safety_factor (src/simulate.jl:151)


class Streamer:
    def __init__(self, seed: int, device: int = 0, level: int = 5, eb=E_BACKGROUND,
                 background: float = 1e13, problem=None, stream=None, tol: float = 1e-8,
                 poisson_iter: int = 0, transport=None):
        """A seeded run on the uniform tree of `level`, or on `problem`'s tree: then the
        densities start as a neutral conducting plasma where the problem's charge is
        (n_e = background + 10 |b|, n_ion = n_e + b, so the initial net charge is b).
        poisson_iter > 0 runs that many V-cycles per stage (derivs!'s fixed count,
        src/streamer.jl:322-334) instead of a mixed-precision solve to `tol`."""
        import torch
        self.rng = np.random.default_rng(seed)
        given = problem is not None
        if not given:
            tree = gen._uniform(level)
            problem = gen.make_problem(tree, lambda r, z, l, gi, gj: np.zeros_like(r), gen.poisson_scale())
        self.tree = problem.tree
        self.problem = p = problem
        self.s, self.geom, self.bc = p.s, p.geom, p.bc
        self.h1 = p.h1
        self.eb = np.ascontiguousarray(eb, dtype=np.float64)
        self.tol = tol
        self.poisson_iter = poisson_iter
        self.tr = mg.Transport(**(transport or MINIMAL))
        self.ctx = mg.Context(device).set_tree(p.tree, p.conn)
        if stream is not None:
            self.ctx.set_stream(stream.cuda_stream)
        self.nblk = n = p.nblk
        dev = torch.device("cuda", device)
        z = lambda *shape: torch.zeros(shape or (n, 20, 20), dtype=torch.float64, device=dev)
        self.ne, self.nion, self.phi, self.b = z(), z(), z(), z()
        self.n1 = [z(), z()]
        self.dn = [[z(), z()] for _ in range(3)]
        self.e, self.flux = z(n, 2, 21, 21), z(n, 2, 21, 21)
        self.eabs = z()
        self.maxdt = z(1)
        self.r, self.u1 = z(), z()  # V-cycle work fields (poisson_iter mode)
        self.t = 0.0
        self.last_dt = 0.0
        self.stage_stats = []
        if given:
            bh = p.b.copy()
            leaf = np.zeros(bh.shape, dtype=bool)
            for layer in self.tree:
                for cc, blk in layer.index.items():
                    if self.tree.isleaf(layer.level, cc):
                        leaf[blk - 1, 2:18, 2:18] = True
            ne = np.where(leaf, background + 10.0 * np.abs(bh), 0.0)
            self.ne.copy_(torch.from_numpy(ne))
            self.nion.copy_(torch.from_numpy(np.where(leaf, ne + bh, 0.0)))
        else:
            # seed: an elongated neutral plasma column on the axis standing on the lower
            # electrode region (Gaussian radial profile and ends), length, radius, density
            # and position jittered
            z0 = self.rng.uniform(0.3e-3, 1.0e-3)
            length = self.rng.uniform(1.5e-3, 3.0e-3)
            w = self.rng.uniform(0.2e-3, 0.4e-3)
            amp = 10 ** self.rng.uniform(19.5, 20.5)
            lev = len(self.tree)
            blks, r, zz, _, _ = gen.block_cell_centres(self.tree, lev, self.h1)
            dz = np.maximum(0.0, np.maximum(z0 - zz, zz - (z0 + length)))
            n0 = background + amp * np.exp(-(r * r + dz * dz) / (w * w))
            ne = np.zeros((n, 20, 20))
            ne[blks - 1, 2:18, 2:18] = n0
            self.ne.copy_(torch.from_numpy(ne))
            self.nion.copy_(torch.from_numpy(ne))
        torch.cuda.synchronize()
        mg.restrict_full_(self.ctx, self.ne)
        mg.restrict_full_(self.ctx, self.nion)
        self._charge(self.ne, self.nion)
        self.ctx.synchronize()
        mg.solve(self.ctx, self.phi, self.b, self.s, self.geom, self.bc, tol=1e-10, mode=mg.MODE_FP64)

    # ---- pieces of derivs! ------------------------------------------------------------

    def _charge(self, ne, nion):
        """netcharge! + restrict_full!(q) (src/streamer.jl:309-313) into self.b."""
        mg.netcharge(self.ctx, self.b, ne, nion)
        mg.restrict_full_(self.ctx, self.b)

    def _solve(self):
        """The stage's Poisson solve, from the current potential."""
        if self.poisson_iter > 0:
            mg.vcycle_(self.ctx, self.phi, self.b.clone(), self.r, self.u1, self.s, self.geom, self.bc,
                       ndown=2, ntop=4, nup=2, ncycles=self.poisson_iter)
            for l in range(1, len(self.tree) + 1):
                mg.fill_ghost_(self.ctx, self.phi, l, self.bc)
            return {"cycles": self.poisson_iter}
        return mg.solve(self.ctx, self.phi, self.b, self.s, self.geom, self.bc, tol=self.tol, mode=mg.MODE_MIXED,
                        **mg.TUNED)

    def _rates(self, dn, ne, nion, maxdt=False):
        """The rest of derivs! after the solve (src/streamer.jl:337-366): dn[0] = dne,
        dn[1] = dnion; with maxdt the smallest stable step goes to self.maxdt."""
        c = self.ctx
        mg.restrict_full_(c, ne)
        for l in range(1, len(self.tree) + 1):
            mg.fill_ghost_(c, ne, l, BC_DENSITY, mask=15)  # copy, bnd, InterpCopy
            mg.fill_ghost_(c, self.phi, l, self.bc)
        mg.electric_field(c, self.e, self.eabs, self.phi, self.h1, self.eb)
        for l in range(1, len(self.tree) + 1):
            mg.fill_ghost_(c, self.eabs, l, BC_EXTRAPOLATE)
        c.check(mg.lib().srmg_streamer_flux_dev(c.handle, self.flux.data_ptr(), None,
                                                self.maxdt.data_ptr() if maxdt else None, ne.data_ptr(),
                                                self.e.data_ptr(), self.eabs.data_ptr(), self.nblk, self.h1,
                                                ctypes.byref(self.tr)))
        c.check(mg.lib().srmg_streamer_rates_dev(c.handle, dn[0].data_ptr(), dn[1].data_ptr(), ne.data_ptr(),
                                                 self.eabs.data_ptr(), self.flux.data_ptr(), self.nblk, self.h1,
                                                 self.geom, ctypes.byref(self.tr)))

    def _combine(self, stage, dt, out):
        c = self.ctx
        for k, nk in enumerate((self.ne, self.nion)):
            c.check(mg.lib().srmg_ssprk3_stage_dev(c.handle, out[k].data_ptr(), nk.data_ptr(),
                                                   self.dn[0][k].data_ptr(), self.dn[1][k].data_ptr(),
                                                   self.dn[2][k].data_ptr(), nk.numel(), dt, stage))

    # ---- step! --------------------------------------------------------------------------

    def advance(self, tmax: float = math.inf, on_stage=None, poisson=None):
        """One SSPRK3 step of step! (src/streamer.jl:386-425).  self.phi must hold the
        solution for the current charge self.b (the first stage's solve); the second
        and third stages solve from the previous stage's potential (poisson(k) for
        stage k if given, else the run's own solve).  Afterwards the densities and
        self.b are those of t + dt, and self.phi is back at the first stage's
        potential, which is returned with the first stage's charge as (phi_prev,
        b_prev).  on_stage(k) runs after stage k's rates (k = 1, 2, 3)."""
        solve = poisson or (lambda k: self._solve())
        c = self.ctx
        phi_prev, b_prev = self.phi.clone(), self.b.clone()
        self.stage_stats = []
        self._rates(self.dn[0], self.ne, self.nion, maxdt=True)
        if on_stage:
            on_stage(1)
        md = float(self.maxdt.cpu()[0])
        dt = min(tmax - self.t, DT_SAFETY * md)
        self._combine(1, dt, self.n1)
        self._charge(*self.n1)
        self.stage_stats.append(solve(2))
        self._rates(self.dn[1], *self.n1)
        if on_stage:
            on_stage(2)
        self._combine(2, dt, self.n1)
        self._charge(*self.n1)
        self.stage_stats.append(solve(3))
        self._rates(self.dn[2], *self.n1)
        if on_stage:
            on_stage(3)
        self._combine(3, dt, (self.ne, self.nion))
        mg.restrict_full_(c, self.ne)
        mg.restrict_full_(c, self.nion)
        self._charge(self.ne, self.nion)
        self.phi.copy_(phi_prev)
        c.synchronize()
        self.t += dt
        self.last_dt = dt
        return phi_prev, b_prev

    def step(self, tmax: float = math.inf, mode=mg.MODE_MIXED, tol=1e-8):
        """Advance one step and solve the new charge from the previous potential;
        returns (phi_prev, b_prev, stats of the new solve)."""
        phi_prev, b_prev = self.advance(tmax)
        kw = mg.TUNED if mode != mg.MODE_FP64 else {}
        st = mg.solve(self.ctx, self.phi, self.b, self.s, self.geom, self.bc, tol=tol, mode=mode, **kw)
        return phi_prev, b_prev, st

    def ionisation_rate(self, stage):
        """The net positive-ion rate of stage k's chemderivs! (valid leaf cells)."""
        return self.dn[stage - 1][1]

    def ir0_of_blocks(self):
        """Global r index before the first cell of every block, by 0-based block id."""
        import torch
        t = np.zeros(self.nblk, dtype=np.int32)
        for layer in self.tree:
            for (cr, cz), blk in layer.index.items():
                t[blk - 1] = 16 * (cr - 1)
        return torch.from_numpy(t).to(self.phi.device)

    def front_z(self) -> float:
        """Highest z where ne exceeds 1e18 m^-3 on the axis column (the streamer tip)."""
        ne = self.ne.cpu().numpy()
        lev = len(self.tree)
        blks, r, zz, _, _ = gen.block_cell_centres(self.tree, lev, self.h1)
        v = ne[blks - 1, 2:18, 2:18]
        m = (v > 1e18) & (r < 2 * self.h1 / 16)
        return float(zz[m].max()) if m.any() else math.nan
