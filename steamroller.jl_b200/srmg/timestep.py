"""The full-size timestep field solve (config 5): on the refined multi-branched channel
tree (8-12M leaf cells), every time step is one SSPRK3 step of step!
(src/streamer.jl:386-425), and each of its three stages solves the Poisson potential
and three photoionization Helmholtz terms, as the reference's derivs! does
(src/streamer.jl:322-334 and src/photo.jl), while the densities move.

Per stage:
  * Poisson: stage 1 from the learned warm start (the network runs on the blocks where
    the charge's second difference is significant, guarded by the previous potential
    and the time extrapolation); stages 2 and 3 from the previous stage's potential;
    mixed precision to 1e-8;
  * Helmholtz: the three terms (k = lambda_j, s = h_1^2, photo boundary table) with the
    stage's ionisation rate as the source, solved together as one batch of 3 items from
    the linear extrapolation of the same stage's solutions of the two previous steps,
    mixed precision, to 1e-8;
  * the densities' rates (libsrmg's flux!, chemderivs!, fluxderivs! kernels) between.
Timed beside: on sampled steps, the plain FP64 GPU solves of every stage (the same
guesses), and the FP64 error of the first stage's mixed results against tight FP64
solves.
"""
from __future__ import annotations

import time

import numpy as np

from . import gen
from . import multigrid as mg
from .streamer import Streamer

LAMBDAS = (1.5e2, 1.2e3, 9.0e3)   # screening constants, 1/m (inside the 1e2-1e4 range)
PHOTO_COEF = (1.0e-4, 6.0e-3, 3.0e-2)  # source weights of the three terms
STAGES = 3


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
        batch = mg.Batch([(s.ctx, h1 * h1, ("helmholtz", lam * lam), gen.BC_PHOTO) for lam in LAMBDAS],
                         p.geom, device=device)
        batch.set_stream(stream.cuda_stream)
        zf = lambda: torch.zeros((nblk, 20, 20), dtype=torch.float64, device=dev)
        # per stage: the Helmholtz solutions of the last step and of the step before
        psi = [[zf() for _ in LAMBDAS] for _ in range(STAGES)]
        psi_old = [None] * STAGES
        src = [zf() for _ in LAMBDAS]
    mask_t = torch.from_numpy(leaf_mask(p.tree, nblk)).to(dev)
    opts = dict(tol=1e-8, max_cycles=5000, **mg.TUNED)          # mixed solves: the tuned smoother
    # one untimed solve of each kind first: a context builds the inverse of its direct
    # coarsest solve (per operator, on the host) the first time it solves
    with torch.cuda.stream(stream):
        mg.solve(s.ctx, s.phi.clone(), s.b.clone(), s.s, s.geom, s.bc, mode=mg.MODE_MIXED, **dict(opts, max_cycles=1))
        batch.solve([zf() for _ in LAMBDAS], [zf() for _ in LAMBDAS], mode=mg.MODE_MIXED, **dict(opts, max_cycles=1))
    stream.synchronize()
    ref_opts = dict(tol=1e-8, ndown=2, ntop=4, nup=2, max_cycles=5000)  # plain FP64: the reference's cycle
    rec = {"poisson_ms": [], "photo_ms": [], "poisson_cycles": [], "photo_cycles": [], "which": [],
           "stage_poisson_cycles": [[] for _ in range(STAGES)]}
    samples = []
    prev1 = prev2 = None
    ev_pairs = []  # (kind, start event, end event) of the current step

    def timed(kind, fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        out = fn()
        b.record(stream)
        ev_pairs.append((kind, a, b))
        return out

    def photo(stage, fp64):
        """The stage's three Helmholtz terms (source: the stage's ionisation rate)."""
        rate = s.ionisation_rate(stage)
        for j, c in enumerate(PHOTO_COEF):
            src[j].copy_(torch.where(mask_t, c * rate, torch.zeros_like(rate)))
        stream.synchronize()
        for j in range(len(LAMBDAS)):
            mg.restrict_full_(s.ctx, src[j])
        k = stage - 1
        if psi_old[k] is not None:
            for j in range(len(LAMBDAS)):
                nxt = 2.0 * psi[k][j] - psi_old[k][j]
                psi_old[k][j].copy_(psi[k][j])
                psi[k][j].copy_(nxt)
        elif rec_steps[0] > 0:
            psi_old[k] = [x.clone() for x in psi[k]]
        guesses = [x.clone() for x in psi[k]] if fp64 is not None else None
        sts = timed("photo", lambda: batch.solve(psi[k], src, mode=mg.MODE_MIXED, **opts))
        cur["photo_cycles"] = max(cur["photo_cycles"], max(x["cycles"] for x in sts))
        if fp64 is not None:
            fp64_stage_photo(s, guesses, src, stream, ref_opts, fp64)

    def poisson(stage, fp64):
        guess = s.phi.clone() if fp64 is not None else None
        st = timed("poisson", lambda: mg.solve(s.ctx, s.phi, s.b, s.s, s.geom, s.bc, mode=mg.MODE_MIXED,
                                               **opts))
        rec["stage_poisson_cycles"][stage - 1].append(st["cycles"])
        cur["poisson_cycles"] += st["cycles"]
        if fp64 is not None:
            fp64_stage_poisson(s, guess, stream, ref_opts, fp64)
        return st

    rec_steps = [0]
    for k in range(steps):
        ev_pairs.clear()
        cur = {"poisson_cycles": 0, "photo_cycles": 0}
        sampled = k % sample_every == sample_every - 1
        fp64 = {"ms": 0.0, "poisson_cycles": [], "photo_cycles": []} if sampled else None
        with torch.cuda.stream(stream):
            # stage 1: the Poisson solve of the current charge, learned warm start
            # s.phi holds the previous step's stage-1 potential; prev1/prev2 the stage-1
            # (potential, charge) of the last two steps
            if prev2 is not None:
                which = timed("poisson", lambda: mg.cnn_predict(s.ctx, net, s.phi, s.b, prev1[1], prev2[0],
                                                                prev2[1], s.s, s.geom, s.bc))
            else:
                which = -1
            guess1 = s.phi.clone() if sampled else None
            poisson(1, fp64)
            if sampled:
                samples.append(error_sample(s, guess1, stream, ref_opts, mask_t))
            phi_prev, b_prev = s.advance(on_stage=lambda st_: photo(st_, fp64),
                                         poisson=lambda st_: poisson(st_, fp64))
            stream.synchronize()
        ms = {"poisson": 0.0, "photo": 0.0}
        for kind, a, b in ev_pairs:
            ms[kind] += a.elapsed_time(b)
        rec["poisson_ms"].append(ms["poisson"])
        rec["photo_ms"].append(ms["photo"])
        rec["poisson_cycles"].append(cur["poisson_cycles"])
        rec["photo_cycles"].append(cur["photo_cycles"])
        rec["which"].append(which)
        if sampled:
            samples[-1]["fp64_step_ms"] = fp64["ms"]
            samples[-1]["fp64_poisson_cycles"] = fp64["poisson_cycles"]
            samples[-1]["fp64_photo_cycles"] = fp64["photo_cycles"]
            if log:
                log(f"step {k}: poisson {np.mean(rec['poisson_ms'][-sample_every:]):.2f} ms "
                    f"({np.mean(rec['poisson_cycles'][-sample_every:]):.1f} cycles), photo "
                    f"{np.mean(rec['photo_ms'][-sample_every:]):.2f} ms; fp64 {fp64['ms']:.1f} ms")
        prev2, prev1 = prev1, (phi_prev, b_prev)
        rec_steps[0] += 1
    w = np.array(rec["which"][2:])
    step_ms = np.array(rec["poisson_ms"]) + np.array(rec["photo_ms"])
    fp64_ms = np.mean([x["fp64_step_ms"] for x in samples])
    out = {
        "workload": "config5: refined multi-branched channel tree; per time step one SSPRK3 step of 3 stages, "
                    "each stage a Poisson solve + 3 photoionization Helmholtz terms (12 solves per step), densities "
                    "advanced by libsrmg's flux!/chemderivs!/fluxderivs! kernels",
        "leaf_cells": int(nleaf), "blocks": int(nblk), "levels": len(p.tree), "steps": steps,
        "stages_per_step": STAGES, "solves_per_step": STAGES * (1 + len(LAMBDAS)), "generate_s": t_gen,
        "mixed_learned": {"step_ms": float(step_ms.mean()), "poisson_ms": float(np.mean(rec["poisson_ms"])),
                          "photo_ms": float(np.mean(rec["photo_ms"])),
                          "poisson_cycles_per_step": float(np.mean(rec["poisson_cycles"])),
                          "poisson_cycles_by_stage": [float(np.mean(c)) for c in rec["stage_poisson_cycles"]],
                          "photo_cycles_max": float(np.mean(rec["photo_cycles"])),
                          "kept": {"previous": float(np.mean(w == 0)), "extrapolated": float(np.mean(w == 1)),
                                   "learned": float(np.mean(w == 2))}},
        "fp64_gpu": {"step_ms": float(fp64_ms), "sampled_steps": len(samples),
                     "poisson_cycles_by_stage": [float(np.mean([x["fp64_poisson_cycles"][i] for x in samples]))
                                                 for i in range(STAGES)],
                     "photo_cycles": [float(np.mean([x["fp64_photo_cycles"][i] for x in samples]))
                                      for i in range(STAGES * len(LAMBDAS))]},
        "speedup_vs_fp64_gpu": float(fp64_ms / step_ms.mean()),
        "error_vs_fp64": {"poisson_rel_l2_max": max(x["err_poisson"] for x in samples),
                          "reference": "mixed stage-1 Poisson result against an FP64 GPU solve to 1e-11 from the "
                                       "same guess, sampled steps"},
    }
    n_solves = STAGES * (1 + len(LAMBDAS))
    out["solves_per_s"] = {"mixed_learned": n_solves * 1e3 / step_ms.mean(), "fp64_gpu": n_solves * 1e3 / fp64_ms}
    batch.close()
    s.ctx.close()
    return out, p


def error_sample(s, guess, stream, opts, mask_t):
    """The FP64 error of the stage-1 mixed Poisson result s.phi against an FP64 solve to
    1e-11 from the same guess."""
    with torch_stream(stream):
        u = guess.clone()
        mg.solve(s.ctx, u, s.b, s.s, s.geom, s.bc, mode=mg.MODE_FP64, **dict(opts, tol=1e-11))
        err = float(((s.phi - u)[mask_t]).norm() / u[mask_t].norm())
    return {"err_poisson": err}


def torch_stream(stream):
    import torch
    return torch.cuda.stream(stream)


def fp64_stage_poisson(s, guess, stream, opts, acc):
    """The stage's Poisson solve again in plain FP64 from the same guess, timed."""
    import torch
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    u = guess.clone()
    a.record(stream)
    st = mg.solve(s.ctx, u, s.b, s.s, s.geom, s.bc, mode=mg.MODE_FP64, **opts)
    b.record(stream)
    b.synchronize()
    acc["ms"] += a.elapsed_time(b)
    acc["poisson_cycles"].append(st["cycles"])


def fp64_stage_photo(s, guesses, src, stream, opts, acc):
    """The stage's three Helmholtz terms again in plain FP64, one by one, from the same
    guesses, timed."""
    import torch
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ps = [x.clone() for x in guesses]
    a.record(stream)
    cyc = []
    for j, lam in enumerate(LAMBDAS):
        st = mg.solve(s.ctx, ps[j], src[j], s.problem.h1 * s.problem.h1, s.geom, gen.BC_PHOTO,
                      ("helmholtz", lam * lam), mode=mg.MODE_FP64, **opts)
        cyc.append(st["cycles"])
    b.record(stream)
    b.synchronize()
    acc["ms"] += a.elapsed_time(b)
    acc["photo_cycles"].extend(cyc)


