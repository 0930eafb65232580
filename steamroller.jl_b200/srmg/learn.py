"""Training data, training loop and evaluation of the learned warm start.

Data: seeded streamer runs (srmg.streamer) on config-1-sized trees; every step gives a
solve pair (phi_prev, b_prev, b, phi_new) from the library's own solver.  The library
cuts each pair into per-block network inputs (srmg_cnn_pack_dev: the 20 x 20 tile of
(phi_prev a, (b - b_prev) c)); the true correction (phi_new - phi_prev) / (s_l |db|)
and the normalised db are kept on the leaf grid.  All stored on the device.

Training: the library's forward and backward kernels, with the loss computed on the
assembled guess over the whole leaf grid -- mean rho^2, rho = L(y) + db the residual
the guess leaves (the quantity the multigrid tolerance is measured on, so block-edge
mismatches count) -- plus a small squared-error anchor to the true correction.

Evaluation: on held-out runs, every k-th step is solved to the tolerance three times
-- from zero, from the previous potential and from the learned guess (which the
library keeps only if it lowers the residual) -- and the V-cycles and times compared.
"""
from __future__ import annotations

import time

import numpy as np

from . import multigrid as mg
from .streamer import Streamer


class Pairs:
    """Device-resident solve pairs of one tree shape: the network inputs of every leaf
    block (x), the normalised right-hand-side change on the leaf grid (db) and the
    normalised true correction (t) per block."""

    def __init__(self, capacity: int, nleaf: int, device: int = 0):
        import torch
        dev = torch.device("cuda", device)
        self.x = torch.empty((capacity, nleaf, 400, 2), dtype=torch.bfloat16, device=dev)
        self.t = torch.empty((capacity, nleaf, 256), dtype=torch.float32, device=dev)
        self.db = torch.empty((capacity, nleaf, 256), dtype=torch.float32, device=dev)
        self.n = 0
        self.capacity = capacity
        self.nleaf = nleaf


class LeafGrid:
    """Leaf blocks of a uniform tree as one (ny, nx) grid with the solver's stencil and
    boundary conditions, for the residual of an assembled guess (training loss)."""

    def __init__(self, s: Streamer, blk):
        import torch
        tree = s.tree
        lev = len(tree)
        coord = {b: c for c, b in tree[lev - 1].index.items()}
        nb = int(blk.shape[0])
        side = int(round(nb ** 0.5)) * 16
        self.ny = self.nx = side
        perm = np.zeros(side * side, dtype=np.int64)
        bl = blk.cpu().numpy()
        for k in range(nb):
            cr, cz = coord[int(bl[k]) + 1]
            yy, xx = np.meshgrid(np.arange(16), np.arange(16), indexing="ij")
            g = (16 * (cz - 1) + yy) * side + 16 * (cr - 1) + xx
            perm[g.ravel()] = k * 256 + (yy * 16 + xx).ravel()
        self.perm = torch.from_numpy(perm).to(blk.device)
        i = np.arange(1, side + 1, dtype=np.float64)
        self.wm = torch.from_numpy((2 * i - 2) / (2 * i - 1)).float().to(blk.device)
        self.wp = torch.from_numpy((2 * i) / (2 * i - 1)).float().to(blk.device)

    def grid(self, f):
        """[P, nleaf, 256] block order -> [P, ny, nx]."""
        return f.reshape(f.shape[0], -1)[:, self.perm].reshape(f.shape[0], self.ny, self.nx)

    def lap(self, Y):
        """Cylindrical 5-point operator with Neumann r and Dirichlet z boundaries."""
        import torch
        left = torch.cat([Y[:, :, :1], Y[:, :, :-1]], 2)     # axis mirror (weight 0 there)
        right = torch.cat([Y[:, :, 1:], Y[:, :, -1:]], 2)    # Neumann at the outer radius
        down = torch.cat([-Y[:, :1, :], Y[:, :-1, :]], 1)    # Dirichlet electrodes
        up = torch.cat([Y[:, 1:, :], -Y[:, -1:, :]], 1)
        return self.wm * left + self.wp * right + down + up - 4 * Y


def generate(runs, steps, seed=0, device=0, log=None):
    """Solve pairs from `runs` seeded streamer runs of `steps` steps each (the first two
    steps of a run only build the history)."""
    import torch
    pairs = None
    t0 = time.time()
    for r in range(runs):
        s = Streamer(seed=1000 * seed + r, device=device)
        hist = None  # (phi_{n-2}, b_{n-2})
        for k in range(steps):
            phi_prev, b_prev, st = s.step()
            if hist is not None:
                phi2, b2 = hist
                f = phi_prev - phi2
                g = s.b - 2 * b_prev + b2
                x, scale, blk = mg.cnn_pack(s.ctx, f, g, s.s, s.geom, s.bc)
                if pairs is None:
                    pairs = Pairs(runs * steps, x.shape[0], device)
                    pairs.grid = LeafGrid(s, blk)
                bi = blk.long()
                d = (s.phi - phi_prev - f)[bi, 2:18, 2:18].reshape(-1, 256)
                gv = g[bi, 2:18, 2:18].reshape(-1, 256)
                sl = s.s / 4 ** (len(s.tree) - 1)
                gn = scale[0] / sl  # the leaf norm of g (scale = s_l |g|)
                k_ = pairs.n
                pairs.x[k_] = x
                pairs.t[k_] = (d / scale[:, None]).float()
                pairs.db[k_] = (gv / gn).float()
                pairs.n += 1
            hist = (phi_prev, b_prev)
        if log:
            log(f"run {r}: {steps} steps, t = {s.t:.3e} s, front z = {s.front_z():.4f} m, "
                f"{pairs.n} pairs, {time.time() - t0:.1f} s")
        s.ctx.close()
    torch.cuda.synchronize()
    return pairs


def train(net: mg.Cnn, pairs: Pairs, steps: int, batch: int = 4, lr: float = 1e-3, mu: float = 0.01,
          seed: int = 0, log=None):
    """Adam on the residual the assembled guess leaves on the leaf grid, plus mu times
    the squared error against the true correction; cosine learning-rate decay.
    Returns the losses."""
    import torch
    g = torch.Generator(device=pairs.x.device)
    g.manual_seed(seed)
    G = pairs.grid
    losses = []
    for k in range(steps):
        idx = torch.randint(0, pairs.n, (batch,), generator=g, device=pairs.x.device)
        x = pairs.x[idx].reshape(-1, 400, 2).contiguous()
        y = net.forward_train(x).reshape(batch, pairs.nleaf, 256).detach().requires_grad_(True)
        Y = G.grid(y)
        rho = G.lap(Y) + G.grid(pairs.db[idx])
        loss = (rho * rho).mean() + mu * ((y - pairs.t[idx]) ** 2).mean()
        loss.backward()
        lr_k = max(lr * 0.5 * (1 + np.cos(np.pi * k / steps)), 1e-6)
        net.backward_step(y.grad.reshape(-1, 256), lr_k)
        losses.append(float(loss.detach()))
        if log and (k % max(1, steps // 10) == 0 or k == steps - 1):
            log(f"train step {k}: loss {losses[-1]:.4e}")
    net.synchronize()
    return losses


def evaluate(net: mg.Cnn, runs, steps, every=10, seed=99, device=0, mode=mg.MODE_MIXED, tol=1e-8, log=None):
    """V-cycles and device times to `tol` on held-out streamer runs from four initial
    guesses: zero, the previous potential, the extrapolation phi_{n-1} + delta_{n-1},
    and the learned guess (the library keeps the best of the last three)."""
    import torch
    rows = []
    warmed = {}
    for r in range(runs):
        s = Streamer(seed=1000 * seed + r, device=device)
        hist = None
        for k in range(steps):
            phi_prev, b_prev = s.advance()
            kw = mg.TUNED if mode != mg.MODE_FP64 else {}
            if hist is None or k % every:
                s.phi.copy_(phi_prev)
                mg.solve(s.ctx, s.phi, s.b, s.s, s.geom, s.bc, tol=tol, mode=mode, **kw)
                hist = (phi_prev, b_prev)
                continue
            phi2, b2 = hist
            res = {}

            def run(u):
                torch.cuda.synchronize()
                st = mg.solve(s.ctx, u, s.b, s.s, s.geom, s.bc, tol=tol, mode=mode, **kw)
                return (st["cycles"], st["device_ms"], st["initial_rel"])

            res["zero"] = run(torch.zeros_like(phi_prev))
            res["prev"] = run(phi_prev.clone())
            res["extrapolated"] = run(2 * phi_prev - phi2)
            if not warmed.get(r):
                # one untimed prediction per run first: the first call of a context sizes
                # its work buffers and sets up the network's launch attributes
                mg.cnn_predict(s.ctx, net, phi_prev.clone(), s.b, b_prev, phi2, b2, s.s, s.geom, s.bc)
                warmed[r] = True
            u = phi_prev.clone()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            which = mg.cnn_predict(s.ctx, net, u, s.b, b_prev, phi2, b2, s.s, s.geom, s.bc)
            t_pred = (time.perf_counter() - t0) * 1e3
            c, ms, ini = run(u)
            res["learned"] = (c, ms + t_pred, ini)
            res["which"] = which
            res["active"] = mg.lib().srmg_cnn_last_active(s.ctx.handle) / mg.lib().srmg_cnn_leaf_blocks(s.ctx.handle)
            res["predict_ms"] = t_pred
            rows.append(res)
            s.phi.copy_(u)
            hist = (phi_prev, b_prev)
        if log:
            log(f"eval run {r}: {len(rows)} solves so far")
        s.ctx.close()
    out = {}
    for key in ("zero", "prev", "extrapolated", "learned"):
        c = np.array([r[key][0] for r in rows], dtype=float)
        ms = np.array([r[key][1] for r in rows], dtype=float)
        ini = np.array([r[key][2] for r in rows], dtype=float)
        out[key] = {"mean_cycles": float(c.mean()), "mean_ms": float(ms.mean()),
                    "median_initial_rel": float(np.median(ini))}
    w = np.array([r["which"] for r in rows])
    out["kept"] = {"previous": float(np.mean(w == 0)), "extrapolated": float(np.mean(w == 1)),
                   "learned": float(np.mean(w == 2))}
    out["predict_ms"] = float(np.mean([r["predict_ms"] for r in rows]))
    out["predict_ms_median"] = float(np.median([r["predict_ms"] for r in rows]))
    out["active_block_fraction"] = float(np.mean([r["active"] for r in rows]))
    out["solves"] = len(rows)
    out["cycles_saved_vs_prev"] = out["prev"]["mean_cycles"] - out["learned"]["mean_cycles"]
    out["cycles_saved_vs_zero"] = out["zero"]["mean_cycles"] - out["learned"]["mean_cycles"]
    out["cycles_saved_vs_extrapolation"] = out["extrapolated"]["mean_cycles"] - out["learned"]["mean_cycles"]
    return out
