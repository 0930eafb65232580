"""The full-size timestep field solve (config 5): on the refined multi-branched channel
tree (8-12M leaf cells), every time step solves the Poisson potential and three
photoionization Helmholtz terms, as the reference's derivs! does
(src/streamer.jl:322-334 and src/photo.jl), while the densities move.

Per step:
  * the densities advance one step (libsrmg's streamer stepper on every leaf block);
  * Poisson: learned warm start from the two previous potentials (the network runs on
    the blocks where the charge's second difference is significant), then the
    mixed-precision solve to 1e-8;
  * Helmholtz: the three terms (k = lambda_j, s = h_1^2, photo boundary table) with
    the ionisation rate of the step as the source, solved together as one batch of 3
    items from the linear extrapolation of their two previous solutions, mixed
    precision, to 1e-8.
Timed beside: the plain FP64 GPU solves of the same step (Poisson from the previous
potential, the three Helmholtz terms one by one from their previous solutions) on
sampled steps, and the FP64 error of the mixed results against tight FP64 solves.
"""
from __future__ import annotations

import time

import numpy as np

from . import gen
from . import multigrid as mg
from .streamer import Streamer

LAMBDAS = (1.5e2, 1.2e3, 9.0e3)   # screening constants, 1/m (inside the 1e2-1e4 range)
PHOTO_COEF = (1.0e-4, 6.0e-3, 3.0e-2)  # source weights of the three terms


def leaf_mask(tree, nblk):
    m = np.zeros((nblk, 20, 20), dtype=bool)
    for layer in tree:
        for cc, blk in layer.index.items():
            if tree.isleaf(layer.level, cc):
                m[blk - 1, 2:18, 2:18] = True
    return m


def run(net, steps=200, sample_every=50, device=0, log=None, problem=None):
    import torch
    dev = torch.device("cuda", device)
    stream = torch.cuda.Stream(device=dev)
    t0 = time.time()
    p = problem if problem is not None else gen.config5()
    t_gen = time.time() - t0
    from .tree import leaf_cells
    nleaf = leaf_cells(p.tree)
    with torch.cuda.stream(stream):
        s = Streamer(seed=5, device=device, problem=p, stream=stream)
        s.ctx.set_option("cnn_active_ppm", 100)
        nblk = s.nblk
        h1 = p.h1
        # Helmholtz items on the same tree, one batch
        bc_photo = gen.BC_PHOTO
        batch = mg.Batch([(s.ctx, h1 * h1, ("helmholtz", lam * lam), bc_photo) for lam in LAMBDAS],
                         p.geom, device=device)
        batch.set_stream(stream.cuda_stream)
        psi = [torch.zeros((nblk, 20, 20), dtype=torch.float64, device=dev) for _ in LAMBDAS]
        src = [torch.zeros_like(s.b) for _ in LAMBDAS]
    mask_t = torch.from_numpy(leaf_mask(p.tree, nblk)).to(dev)
    ev0, ev1, ev2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    rec = {"poisson_ms": [], "photo_ms": [], "poisson_cycles": [], "photo_cycles": [], "which": []}
    samples = []
    hist = None
    psi_old = None  # the Helmholtz solutions of the step before the previous one
    opts = dict(tol=1e-8, ndown=2, ntop=4, nup=2, max_cycles=5000)

    def photo_sources():
        # ionisation rate of the last step (the stepper's dn+/dt) on leaf cells, weighted
        rate = s.work[nblk * 400:2 * nblk * 400].view(nblk, 20, 20)
        for j, c in enumerate(PHOTO_COEF):
            src[j].copy_(torch.where(mask_t, c * rate, torch.zeros_like(rate)))
        torch.cuda.current_stream().synchronize()
        for j in range(len(LAMBDAS)):
            for l in range(len(p.tree), 1, -1):
                s.ctx.check(mg.lib().srmg_restrict_level_dev(s.ctx.handle, src[j].data_ptr(), nblk, l))

    for k in range(steps):
        with torch.cuda.stream(stream):
            phi_prev, b_prev = s.advance()
            photo_sources()
            stream.synchronize()
            ev0.record(stream)
            if hist is not None:
                phi2, b2 = hist
                which = mg.cnn_predict(s.ctx, net, s.phi, s.b, b_prev, phi2, b2, s.s, s.geom, s.bc)
            else:
                which = -1
            st = mg.solve(s.ctx, s.phi, s.b, s.s, s.geom, s.bc, mode=mg.MODE_MIXED, **opts)
            ev1.record(stream)
            sampled = k % sample_every == sample_every - 1
            psi_prev = [x.clone() for x in psi] if sampled else None
            # Helmholtz initial guesses: linear extrapolation from the two previous
            # solutions (the sources move smoothly with the streamer); the solve
            # iterates to the same tolerance from whatever guess it is given
            if psi_old is not None:
                for j in range(len(LAMBDAS)):
                    nxt = 2.0 * psi[j] - psi_old[j]
                    psi_old[j].copy_(psi[j])
                    psi[j].copy_(nxt)
            elif k > 0:
                psi_old = [x.clone() for x in psi]
            sts = batch.solve(psi, src, mode=mg.MODE_MIXED, **opts)
            ev2.record(stream)
            ev2.synchronize()
        rec["poisson_ms"].append(ev0.elapsed_time(ev1))
        rec["photo_ms"].append(ev1.elapsed_time(ev2))
        rec["poisson_cycles"].append(st["cycles"])
        rec["photo_cycles"].append(max(x["cycles"] for x in sts))
        rec["which"].append(which)
        if sampled:
            samples.append(fp64_sample(s, psi, psi_prev, src, phi_prev, stream, opts, mask_t))
            if log:
                log(f"step {k}: poisson {np.mean(rec['poisson_ms'][-sample_every:]):.2f} ms "
                    f"({np.mean(rec['poisson_cycles'][-sample_every:]):.1f} cycles), photo "
                    f"{np.mean(rec['photo_ms'][-sample_every:]):.2f} ms; fp64 {samples[-1]['fp64_step_ms']:.1f} ms")
        hist = (phi_prev, b_prev)
    out_problem = p
    w = np.array(rec["which"][1:])
    step_ms = np.array(rec["poisson_ms"]) + np.array(rec["photo_ms"])
    fp64_ms = np.mean([x["fp64_step_ms"] for x in samples])
    fp64_cyc = np.mean([x["fp64_poisson_cycles"] for x in samples])
    out = {
        "workload": "config5: refined multi-branched channel tree, Poisson + 3 photoionization Helmholtz "
                    "terms per step, densities advanced by the streamer stepper between steps",
        "leaf_cells": int(nleaf), "blocks": int(nblk), "levels": len(p.tree), "steps": steps,
        "generate_s": t_gen,
        "mixed_learned": {"step_ms": float(step_ms.mean()), "poisson_ms": float(np.mean(rec["poisson_ms"])),
                          "photo_ms": float(np.mean(rec["photo_ms"])),
                          "poisson_cycles": float(np.mean(rec["poisson_cycles"])),
                          "photo_cycles_max": float(np.mean(rec["photo_cycles"])),
                          "kept": {"previous": float(np.mean(w == 0)), "extrapolated": float(np.mean(w == 1)),
                                   "learned": float(np.mean(w == 2))}},
        "fp64_gpu": {"step_ms": float(fp64_ms), "poisson_cycles": float(fp64_cyc),
                     "photo_cycles": [float(np.mean([x["fp64_photo_cycles"][j] for x in samples]))
                                      for j in range(len(LAMBDAS))]},
        "speedup_vs_fp64_gpu": float(fp64_ms / step_ms.mean()),
        "error_vs_fp64": {"poisson_rel_l2_max": max(x["err_poisson"] for x in samples),
                          "photo_rel_l2_max": max(x["err_photo"] for x in samples)},
    }
    out["solves_per_s"] = {"mixed_learned": 4 * 1e3 / step_ms.mean(), "fp64_gpu": 4 * 1e3 / fp64_ms}
    batch.close()
    s.ctx.close()
    return out, out_problem


def fp64_sample(s, psi, psi_prev, src, phi_prev, stream, opts, mask_t):
    """The same step in plain FP64 on the GPU (from the previous potential and the
    previous Helmholtz solutions), timed, and the FP64 error of the mixed results psi
    and s.phi against FP64 solves to 1e-11."""
    import torch
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        u = phi_prev.clone()
        ps = [x.clone() for x in psi_prev]
        stream.synchronize()
        ev0.record(stream)
        st = mg.solve(s.ctx, u, s.b, s.s, s.geom, s.bc, mode=mg.MODE_FP64, **opts)
        photo_cycles = []
        for j, lam in enumerate(LAMBDAS):
            sth = mg.solve(s.ctx, ps[j], src[j], batch_s(s), s.geom, gen.BC_PHOTO, ("helmholtz", lam * lam),
                           mode=mg.MODE_FP64, **opts)
            photo_cycles.append(sth["cycles"])
        ev1.record(stream)
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1)
        tight = dict(opts, tol=1e-11)
        mg.solve(s.ctx, u, s.b, s.s, s.geom, s.bc, mode=mg.MODE_FP64, **tight)
        err_p = float(((s.phi - u)[mask_t]).norm() / u[mask_t].norm())
        err_h = 0.0
        for j, lam in enumerate(LAMBDAS):
            mg.solve(s.ctx, ps[j], src[j], batch_s(s), s.geom, gen.BC_PHOTO, ("helmholtz", lam * lam),
                     mode=mg.MODE_FP64, **tight)
            n = ps[j][mask_t].norm()
            if n > 0:
                err_h = max(err_h, float(((psi[j] - ps[j])[mask_t]).norm() / n))
    return {"fp64_step_ms": ms, "fp64_poisson_cycles": st["cycles"], "fp64_photo_cycles": photo_cycles,
            "err_poisson": err_p, "err_photo": err_h}


def batch_s(s):
    return s.problem.h1 * s.problem.h1
