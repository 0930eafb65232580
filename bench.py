"""Benchmark: field solves/s to 1e-8 relative residual on the refined channel tree.

Workload (one "step"): one Poisson field solve L u + s b = 0 from a zero initial guess
to resnorm(u)/leafnorm(b) <= 1e-8 on the refined channel tree of ~1.5M leaf cells
(config 2: base uniform tree to level 5 plus 4 refined levels, cylindrical r-z,
order-2 stencil, Neumann axis/outer radius, Dirichlet electrodes).  Synthetic, seeded
data with the shapes of the reference's own setup (no published data exists).

  value      mixed-precision solves/s (FP32 V-cycles + FP64 defect correction, FP64
             direct coarsest-level solve) with fields resident in HBM
  fp64       the plain FP64 GPU multigrid (the reference's V-cycle, repeated to the
             same tolerance) on the same tree
  roofline   the timed kernel (one mixed-solve launch per step): algorithmic bytes
             of the model (srmg.model.mixed_solve_bytes) / its event-timed duration,
             against the measured HBM copy peak; roofline_fp64_vcycle the same for
             one plain FP64 V-cycle (srmg.model.vcycle_bytes)
  e2e        the same solve through the C ABI with host arrays (H2D of u and b and
             D2H of u inside the timed region, every step): srmg_solve_async /
             srmg_solve_wait on two contexts of the tree, each step's copies
             overlapping the other context's solve; e2e.sync gives srmg_solve one call
             at a time
  cpu_baseline  the oracle (C restatement of the reference FP64 solve, OpenMP) on
             the host cores: complete solves from a zero guess to the tolerance
  error_vs_fp64  each GPU result's relative L2 error on the leaf cells against the
             oracle's FP64 solution of the same problem to 1e-11

`--impl reference` times the reference's CPU algorithm (the oracle, since Julia is not
available) on the same workload.  Multi-GPU: replicas (independent solves per rank,
no data-path collective), weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "steamroller.jl_b200"))

import numpy as np  # noqa: E402

TOL = 1e-8
SEED = 2
TARGET_LEAF = 1_500_000
METRIC = "field solves/sec at 1e-8 rel residual (mixed-precision multigrid; plain FP64 GPU alongside)"
# DRAM bytes of one plain FP64 V-cycle launch on the config-2 tree, from an ncu capture
# (57.52 MB read + 40.66 MB written)
TRAFFIC_VCYCLE_CONFIG2 = 98.18e6
# DRAM bytes of one mixed-solve launch on the config-2 tree (the tuned V(1,1) cycle,
# 9 V-cycles in 3 defect-correction steps, the direct solve on level 2), from an ncu
# capture (170.85 MB read + 137.01 MB written)
TRAFFIC_MIXED_CONFIG2 = 307.87e6


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons while the timed region runs: NVML
    polled every 5 ms (nvidia-smi's fastest loop, 200 ms, would see one sample of a
    40 ms region) plus `nvidia-smi -lms 200` beside it for the reasons.  A failing NVML
    call is recorded (`nvml_error`) and the other sources keep going."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits (nvml.h: nvmlClocksEventReason*)
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
            "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}

    def __init__(self, index, period_s=0.005):
        self.index = index
        self.period = period_s
        self.sm, self.mx, self.reasons = [], [], set()
        self.smi_sm, self.smi_mx = [], []
        self.proc = None
        self.nvml = None
        self.error = None
        self.stop_ev = threading.Event()
        self.threads = []

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _note(self, e):
        if self.error is None:
            self.error = f"{type(e).__name__}: {e}"

    def start(self):
        self.stop_ev.clear()
        try:
            self.nvml, self.h = self._handle()
            self.threads.append(threading.Thread(target=self._poll, daemon=True))
        except Exception as e:
            self._note(e)
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.threads.append(threading.Thread(target=self._read, daemon=True))
        except Exception:
            self.proc = None
        for t in self.threads:
            t.start()
        return self

    def _poll(self):
        nv = self.nvml
        getters = [getattr(nv, n) for n in ("nvmlDeviceGetCurrentClocksEventReasons",
                                             "nvmlDeviceGetCurrentClocksThrottleReasons") if hasattr(nv, n)]
        try:
            mx = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))
        except Exception as e:
            self._note(e)
            mx = None
        while True:
            try:
                self.sm.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
                if mx is not None:
                    self.mx.append(mx)
            except Exception as e:
                self._note(e)
            while getters:
                try:
                    bits = int(getters[0](self.h))
                    for name, bit in self.BITS.items():
                        if bits & bit:
                            self.reasons.add(name)
                    break
                except Exception as e:
                    self._note(e)
                    getters.pop(0)
            if self.stop_ev.wait(self.period):
                break

    def _read(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.proc.stdout:
            r = [x.strip() for x in line.split(",")]
            if len(r) > 8 and r[1].replace(".", "").isdigit():
                self.smi_sm.append(float(r[1]))
                self.smi_mx.append(float(r[2]))
                for k, n in enumerate(names):
                    if r[5 + k].lower() == "active":
                        self.reasons.add(n)

    def stop(self):
        self.stop_ev.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        for t in self.threads:
            t.join(timeout=5)

    def __enter__(self):
        return self.start()

    def __exit__(self, *a):
        self.stop()

    def summary(self):
        sm = self.sm if self.sm else self.smi_sm
        mx = self.mx + self.smi_mx
        out = {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
               "reasons": sorted(self.reasons), "samples": len(self.sm), "smi_samples": len(self.smi_sm),
               "source": "nvml every 5 ms + nvidia-smi every 200 ms"}
        if self.error:
            out["nvml_error"] = self.error
        return out


def dist_setup(backend=None, timeout_s=120):
    """One process per GPU (torchrun env); NCCL on GPUs, gloo on the host (tests).  A
    rank that dies or never joins makes the others' next collective end with an error
    within timeout_s instead of waiting for good."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group(backend or "nccl", timeout=datetime.timedelta(seconds=timeout_s))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(x, pg, device):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, device):
    import torch
    if pg is not None:
        if device.type == "cuda":
            pg.barrier(device_ids=[device.index])
        else:
            pg.barrier()
    if device.type == "cuda":
        torch.cuda.synchronize()


def shard(n, rank, world):
    """Independent work units (trees) of this rank: round-robin, no exchange needed."""
    return list(range(rank, n, world))


def _oracle(problem, threads):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc_mod
    orc_mod.build() if not os.path.exists(orc_mod._LIB_PATH) else None
    return orc_mod.Oracle(problem, threads=threads)


def oracle_solve(problem, tol, threads=None, u0=None, max_cycles=5000):
    """One complete reference-algorithm FP64 solve (the oracle: V-cycles (2, 2, 4) with
    resnorm after each, src/multigrid.jl:60-106, 391-417) from u0 (zero if None) to
    resnorm/leafnorm(b) <= tol.  Returns (u, cycles, rel_residual, wall seconds)."""
    orc = _oracle(problem, threads or os.cpu_count())
    u = np.zeros_like(problem.b) if u0 is None else u0.copy()
    b = problem.b.copy()
    t0 = time.perf_counter()
    c, rel = orc.solve(u, b, tol, max_cycles=max_cycles, ndown=2, ntop=4, nup=2)
    return u, c, rel, time.perf_counter() - t0


def run_cpu_reference(problem, steps=1, warm=0, threads=None, budget_s=None):
    """Time complete reference-algorithm solves (the oracle, OpenMP over blocks per
    level, as the reference's @batch loops) from a zero guess to 1e-8 on the host cores:
    `warm` untimed solves, then `steps` timed ones (with budget_s: as many as fit, at
    least one).  Every solve is run to the tolerance; nothing is extrapolated."""
    threads = threads or os.cpu_count()
    for _ in range(warm):
        oracle_solve(problem, TOL, threads)
    times, cycles, rels = [], [], []
    t_start = time.perf_counter()
    while True:
        _, c, rel, dt = oracle_solve(problem, TOL, threads)
        times.append(dt)
        cycles.append(c)
        rels.append(rel)
        if budget_s is None:
            if len(times) >= steps:
                break
        elif time.perf_counter() - t_start + dt > budget_s:
            break
    total = float(np.sum(times))
    n = len(times)
    return {"value": n / total, "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": f"{n} complete FP64 solves of this tree from a zero guess to rel. residual {TOL:g} "
                      f"({cycles[0]} V-cycles each, {total:.1f} s)",
            "ms_per_solve": 1e3 * total / n, "cycles_per_solve": int(cycles[0]),
            "rel_residual": float(max(rels)), "solves": n}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="srmg", choices=["srmg", "reference"])
    ap.add_argument("--target-leaf", type=int, default=TARGET_LEAF)
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched config-3 section")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned warm-start (config-4) section")
    ap.add_argument("--learned-pairs", type=int, default=20000, help="solve pairs generated for training")
    ap.add_argument("--no-config5", action="store_true", help="skip the full-size timestep (config-5) section")
    ap.add_argument("--config5-steps", type=int, default=200)
    ap.add_argument("--no-rows", action="store_true", help="skip the order-4, 3D and free-boundary section")
    ap.add_argument("--no-autotune", action="store_true",
                    help="mixed solve with the stored tuned smoother (srmg.multigrid.TUNED) instead of autotuning "
                         "first (profiling runs: the timed launches are then the first engine launches)")
    ap.add_argument("--only", default=None, choices=[None, "vcycle", "smooth", "cnn", "rows"],
                    help="vcycle: time plain FP64 V-cycles only; smooth: GS iterations on the finest "
                         "level only; cnn: the warm-start network's inference forward, mma.sync and "
                         "tcgen05 (profiling runs); rows: the order-4, 3D and free-boundary section")
    ap.add_argument("--samples", type=int, default=4096, help="--only cnn: block samples per forward")
    ap.add_argument("--config", default="config2", choices=["config1", "config2", "config5"])
    args = ap.parse_args()
    if args.only in ("vcycle", "smooth"):
        return vcycle_only(args)
    if args.only == "cnn":
        return cnn_only(args)
    if args.only == "rows":
        print(json.dumps({"only": "rows", **run_rows(0)}))
        return

    from srmg import gen, model
    from srmg.tree import leaf_cells

    world, rank, local, pg = dist_setup()
    problem = gen.config2(seed=SEED, target_leaf=args.target_leaf)
    nleaf = leaf_cells(problem.tree)
    cfg = {"workload": "config2: refined channel tree, Poisson, cylindrical r-z, tol 1e-8",
           "leaf_cells": nleaf, "blocks": problem.tree.nblocks(), "levels": problem.tree.finest_level(),
           "block": "16x16 + 2 ghosts", "tol": TOL,
           "vcycle": "(ndown,nup,ntop)=(2,2,4), omega 1 for the plain FP64 leg and the reference arm; "
                     "the mixed and FP64 + direct legs use 'tuned'",
           "parallelism": f"replicas x{world}", "l2": "flushed between timed steps (256 MB write)"}

    if args.impl == "reference":
        if rank != 0:
            return
        # one step = one complete FP64 solve of the reference algorithm (the oracle) from
        # a zero guess to the tolerance, wall-timed on the host cores
        cpu = run_cpu_reference(problem, steps=args.steps, warm=args.warmup)
        line = {"impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": "solves/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": cpu["ms_per_solve"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
                "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": cpu["value"], "unit": "solves/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0},
                "fp64_cycles_per_solve": {"cycles": cpu["cycles_per_solve"], "extrapolated": False,
                                          "rel_residual": cpu["rel_residual"]}}
        print(json.dumps(line))
        return

    import torch
    from srmg import multigrid as mg
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = mg.Context(local).set_tree(problem.tree, problem.conn)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)
    nblk = problem.nblk
    b = torch.from_numpy(problem.b).to(dev)
    u = torch.zeros_like(b)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    s, geom, bc = problem.s, problem.geom, problem.bc

    # the project's autotuner picks the launch shape, sweep counts and Gauss-Seidel
    # relaxation factor of the mixed solve on this problem (untimed; the plain FP64 leg
    # keeps the reference's V(2,2) cycle with 4 top sweeps and omega = 1)
    with torch.cuda.stream(stream):
        u.zero_()
    stream.synchronize()
    launch_opts = {}  # the tuned launch shape (set on ctx by the autotuner), for a second context
    if args.no_autotune:
        tuned, inner = dict(mg.TUNED), 3  # the autotuner's choice on this tree
    else:
        chosen, trials = mg.autotune(ctx, u, b, s, geom, bc, tol=TOL, mode=mg.MODE_MIXED)
        tuned = {k: chosen[k] for k in ("ndown", "nup", "ntop", "omega")}
        inner = chosen["inner_cycles"]
        if trials:
            best = min(trials, key=lambda t: t["ms"])
            launch_opts = {"engine_ctas": best["engine_ctas"], "local_max_blocks": best["local_max_blocks"]}
    cfg["tuned"] = dict(tuned, inner_cycles=inner)
    ref_cycle = dict(ndown=2, nup=2, ntop=4, omega=1.0)
    opts_of = {mg.MODE_MIXED: dict(tuned, inner_cycles=inner), mg.MODE_FP64_DIRECT: tuned, mg.MODE_FP64: ref_cycle}

    def one_solve(mode, max_cycles=5000):
        u.zero_()
        return mg.solve(ctx, u, b, s, geom, bc, tol=TOL, mode=mode, max_cycles=max_cycles, **opts_of[mode])

    def timed(mode, steps, warm, clk=None):
        for _ in range(warm):
            with torch.cuda.stream(stream):
                st = one_solve(mode)
        barrier(pg, dev)
        total_ms, stats = 0.0, None
        l0 = ctx.launches()
        if clk is not None:
            clk.start()
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                u.zero_()
            stream.synchronize()
            st = mg.solve(ctx, u, b, s, geom, bc, tol=TOL, mode=mode, max_cycles=5000, **opts_of[mode])
            total_ms += st["device_ms"]
            stats = st
        if clk is not None:
            clk.stop()
        barrier(pg, dev)
        return total_ms, stats, ctx.launches() - l0

    clk = ClockSampler(local)
    mixed_ms, mixed_st, launches = timed(mg.MODE_MIXED, args.steps, args.warmup, clk)
    fp64_steps = max(1, args.fp64_steps)
    fp64_ms, fp64_st, _ = timed(mg.MODE_FP64, fp64_steps, 1)
    # FP64 V-cycles with the mixed mode's direct coarsest solve: the precision effect alone
    fpd_ms, fpd_st, _ = timed(mg.MODE_FP64_DIRECT, args.steps, 1)
    mixed_ms = max_over_ranks(mixed_ms, pg, dev)
    fp64_ms = max_over_ranks(fp64_ms, pg, dev)
    fpd_ms = max_over_ranks(fpd_ms, pg, dev)
    value = world * args.steps / (mixed_ms / 1e3)
    fp64_value = world * fp64_steps / (fp64_ms / 1e3)
    fpd_value = world * args.steps / (fpd_ms / 1e3)

    # error of each result on the leaf cells against the FP64 oracle's solution of the
    # same problem to 1e-11 (the oracle's complete solve on the host cores, rank 0); with
    # --no-cpu, against the plain FP64 GPU path's solve to 1e-11 instead
    from srmg.timestep import leaf_mask
    leaf_np = leaf_mask(problem.tree, problem.nblk)
    leaf = torch.from_numpy(leaf_np).to(dev)
    sols = {}
    for name, mode, tol in (("fp64_tight", mg.MODE_FP64, 1e-11), ("mixed", mg.MODE_MIXED, TOL),
                            ("fp64", mg.MODE_FP64, TOL)):
        with torch.cuda.stream(stream):
            u.zero_()
        stream.synchronize()
        mg.solve(ctx, u, b, s, geom, bc, tol=tol, mode=mode, max_cycles=5000, **opts_of[mode])
        sols[name] = u[leaf].cpu().numpy()
    if rank == 0 and not args.no_cpu:
        uo, oc, orel, ot = oracle_solve(problem, 1e-11)
        ref = uo[leaf_np]
        ref_name = (f"FP64 oracle solve to 1e-11 from zero ({oc} V-cycles, rel. residual {orel:.2e}, "
                    f"{ot:.1f} s on {os.cpu_count()} host cores); leaf cells, relative L2")
    else:
        ref = sols["fp64_tight"]
        ref_name = "FP64 GPU solve to 1e-11 (leaf cells, relative L2)"
    nref = float(np.linalg.norm(ref))
    err = {k: float(np.linalg.norm(sols[k] - ref)) / nref for k in ("mixed", "fp64", "fp64_tight")}
    err["reference"] = ref_name

    # roofline of the plain FP64 V-cycle (model bytes / event-timed V-cycle)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r_, u1_ = torch.zeros_like(b), torch.zeros_like(b)
    bw = b.clone()
    nv = 20
    with torch.cuda.stream(stream):
        u.zero_()
        mg.vcycle_(ctx, u, bw, r_, u1_, s, geom, bc, ndown=2, ntop=4, nup=2, ncycles=3)
        flush.fill_(2.0)
        ev0.record(stream)
        mg.vcycle_(ctx, u, bw, r_, u1_, s, geom, bc, ndown=2, ntop=4, nup=2, ncycles=nv)
        ev1.record(stream)
    ev1.synchronize()
    vc_ms = ev0.elapsed_time(ev1) / nv
    bytes_vc = model.vcycle_bytes(problem.tree, 8, 2, 2, 4)
    hbm, src = peaks()
    achieved = bytes_vc / (vc_ms / 1e3) / 1e9
    # the timed kernel: one mixed-solve launch per step, event-timed on the context's stream
    bytes_mx = model.mixed_solve_bytes(problem.tree, mixed_st["cycles"], mixed_st["outer"], ndown=tuned["ndown"],
                                       nup=tuned["nup"])
    achieved_mx = bytes_mx / (mixed_ms / args.steps / 1e3) / 1e9

    # e2e through the host-pointer C ABI, from page-locked host buffers
    uh = torch.zeros(problem.b.shape, dtype=torch.float64).pin_memory().numpy()
    bh = torch.from_numpy(np.ascontiguousarray(problem.b)).pin_memory().numpy()
    e2e_t = []
    for i in range(args.warmup + args.steps):
        uh[:] = 0.0
        t0 = time.perf_counter()
        mg.solve(ctx, uh, bh, s, geom, bc, tol=TOL, mode=mg.MODE_MIXED, **opts_of[mg.MODE_MIXED])
        if i >= args.warmup:
            e2e_t.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(float(np.sum(e2e_t)), pg, dev)
    # the same through srmg_solve_async / srmg_solve_wait: two contexts on the tree
    # alternate, so that each step's copies overlap the other context's solve; every
    # step copies its own zero guess and b in and its solution out (page-locked buffers
    # zeroed before timing), results checked against the synchronous solve's
    ctx2 = mg.Context(local).set_tree(problem.tree, problem.conn)
    for k, v in launch_opts.items():
        ctx2.set_option(k, v)
    ctxs = (ctx, ctx2)
    nbuf = args.warmup + args.steps
    uhs = [torch.zeros(problem.b.shape, dtype=torch.float64).pin_memory().numpy() for _ in range(nbuf)]
    bhs = [bh, torch.from_numpy(np.ascontiguousarray(problem.b)).pin_memory().numpy()]
    kw_async = dict(tol=TOL, mode=mg.MODE_MIXED, **opts_of[mg.MODE_MIXED])
    pending = [False, False]
    t_pipe = 0.0
    for i in range(nbuf):
        if i == args.warmup:  # the timed steps start from an empty pipeline
            for k in (0, 1):
                if pending[k]:
                    mg.solve_wait(ctxs[k])
                    pending[k] = False
            t_pipe = time.perf_counter()
        if pending[i % 2]:
            mg.solve_wait(ctxs[i % 2])
        mg.solve_async(ctxs[i % 2], uhs[i], bhs[i % 2], s, geom, bc, **kw_async)
        pending[i % 2] = True
    for k in (0, 1):
        if pending[k]:
            mg.solve_wait(ctxs[k])
    t_pipe = time.perf_counter() - t_pipe
    uref = uh.copy()  # the last synchronous solve's result
    pipe_ok = all(np.array_equal(uhs[i].view(np.uint64), uref.view(np.uint64)) for i in range(nbuf))
    ctx2.close()
    pipe_s = max_over_ranks(t_pipe, pg, dev)
    e2e = {"value": world * args.steps / pipe_s, "unit": "solves/s",
           "h2d_bytes_per_step": 2 * nblk * 400 * 8, "d2h_bytes_per_step": nblk * 400 * 8,
           "host_memory": "pinned",
           "api": "srmg_solve_async/srmg_solve_wait on two contexts, copies overlapping the other's solve",
           "results_equal_sync": bool(pipe_ok),
           "sync": {"value": world * args.steps / e2e_s, "unit": "solves/s",
                    "api": "srmg_solve, one call at a time"}}

    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mixed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": cfg,
            "fp64": {"value": fp64_value, "unit": "solves/s", "cycles_per_solve": fp64_st["cycles"],
                     "ms_per_solve": fp64_ms / fp64_steps, "rel_residual": fp64_st["rel_residual"]},
            "mixed": {"cycles_per_solve": mixed_st["cycles"], "outer_steps": mixed_st["outer"],
                      "rel_residual": mixed_st["rel_residual"]},
            "fp64_direct_coarse": {"value": fpd_value, "unit": "solves/s", "cycles_per_solve": fpd_st["cycles"],
                                   "ms_per_solve": fpd_ms / args.steps, "rel_residual": fpd_st["rel_residual"],
                                   "what": "FP64 V-cycles with the mixed mode's direct FP64 coarsest solve"},
            "speedup_vs_fp64": value / fp64_value,
            "speedup_split": {"coarse_solve": fpd_value / fp64_value, "precision": value / fpd_value},
            "roofline": {"bound": "hbm", "achieved": achieved_mx, "peak": hbm, "unit": "GB/s",
                         "frac": achieved_mx / hbm,
                         "traffic": TRAFFIC_MIXED_CONFIG2 if nleaf == 1503232 else None,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one mixed-solve "
                                           "launch on this tree (most of the working set stays in L2)",
                         "peak_source": src,
                         "kernel": "mixed-precision solve (one persistent launch per solve: the timed kernel)",
                         "bytes_per_launch": bytes_mx, "ms_per_launch": mixed_ms / args.steps,
                         "bytes_model": "srmg.model.mixed_solve_bytes(tree, cycles=%d, steps=%d, ndown=%d, nup=%d)"
                                        % (mixed_st["cycles"], mixed_st["outer"], tuned["ndown"], tuned["nup"])},
            "roofline_fp64_vcycle": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                                     "frac": achieved / hbm,
                                     "traffic": TRAFFIC_VCYCLE_CONFIG2 if nleaf == 1503232 else None,
                                     "peak_source": src, "kernel": "plain FP64 V-cycle (whole cycle)",
                                     "bytes_per_launch": bytes_vc, "ms_per_vcycle": vc_ms},
            "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(), "error_vs_fp64": err}
    all_cells = sum(len(layer) for layer in problem.tree) * 256
    line["cells_vcycles_per_s"] = {
        "leaf": nleaf * mixed_st["cycles"] * value, "all_levels": all_cells * mixed_st["cycles"] * value,
        "fp64_leaf": nleaf * fp64_st["cycles"] * fp64_value, "note": "cells x V-cycles per second"}
    line["config1"] = run_config1(local, args.steps, args.warmup, cpu=(rank == 0 and not args.no_cpu))
    line["dropin_vcycle"] = run_dropin(ctx, problem, args.steps, args.warmup, stream)
    if not args.no_batch:
        line["batch"] = run_batch(local, stream, min(args.steps, 3), rank, world, pg, dev)
    if not args.no_learned:
        line["learned"], net = run_learned(local, args.learned_pairs)
        if not args.no_config5:
            line["config5"] = run_config5(local, net, args.config5_steps, cpu=(rank == 0 and not args.no_cpu))
        net.close()
    if not args.no_rows:
        line["rows"] = run_rows(local)
    if rank == 0 and world == 1 and not args.no_cpu:
        # complete oracle solves from zero to 1e-8 for about 20 s (at least one)
        cpu = run_cpu_reference(problem, budget_s=20.0)
        line["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        line["cpu_baseline"]["cycles_per_solve"] = cpu["cycles_per_solve"]
        # the same on one host core (the oracle's OpenMP loops with one thread): one solve
        cpu1 = run_cpu_reference(problem, steps=1, threads=1)
        line["cpu_baseline_1core"] = {k: cpu1[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if pg is not None:
        pg.destroy_process_group()


def run_dropin(ctx, problem, steps, warm, stream):
    """The drop-in call as run_from_input makes it: derivs! runs poisson_iter = 2
    vcycle! per stage (src/streamer.jl:322-334) on Julia-owned, pageable host arrays,
    which the shim hands to srmg_vcycle.  Wall time per call (H2D of u and b, 2 V-cycles,
    D2H of u), from pageable numpy arrays: with b copied back (the reference's in/out
    b), without it (the default), and with the arrays page-locked by srmg_host_register;
    beside it the device time of the same 2 V-cycles."""
    from srmg import multigrid as mg
    p = problem
    u0 = np.zeros_like(p.b)
    out = {"workload": "config2 tree, srmg_vcycle x 2 V-cycles (poisson_iter = 2) on pageable host arrays",
           "bytes_per_call": {"h2d": 2 * p.b.nbytes, "d2h_u": p.b.nbytes}}
    cases = (("pageable_b_copied_back", 1, False), ("pageable", 0, False), ("registered", 0, True))
    for name, copy_back, register in cases:
        ctx.set_option("b_copy_back", copy_back)
        u, b = u0.copy(), p.b.copy()
        r, u1 = np.zeros_like(u), np.zeros_like(u)
        if register:
            for a in (u, b):
                ctx.check(mg.lib().srmg_host_register(ctx.handle, a.ctypes.data, a.nbytes))
        ts = []
        for i in range(warm + steps):
            t0 = time.perf_counter()
            mg.vcycle_(ctx, u, b, r, u1, p.s, p.geom, p.bc, ndown=2, ntop=4, nup=2, ncycles=2)
            if i >= warm:
                ts.append(time.perf_counter() - t0)
        if register:
            for a in (u, b):
                ctx.check(mg.lib().srmg_host_unregister(ctx.handle, a.ctypes.data))
        out[name] = {"ms_per_call": 1e3 * float(np.mean(ts)), "ms_min": 1e3 * float(np.min(ts))}
    ctx.set_option("b_copy_back", 0)
    import torch
    bg = torch.from_numpy(p.b).cuda()
    ug = torch.zeros_like(bg)
    rg, u1g = torch.zeros_like(bg), torch.zeros_like(bg)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):  # the context's stream: the events bracket its launches
        mg.vcycle_(ctx, ug, bg, rg, u1g, p.s, p.geom, p.bc, ndown=2, ntop=4, nup=2, ncycles=2)
        ev0.record(stream)
        for _ in range(steps):
            mg.vcycle_(ctx, ug, bg, rg, u1g, p.s, p.geom, p.bc, ndown=2, ntop=4, nup=2, ncycles=2)
        ev1.record(stream)
    ev1.synchronize()
    out["device_ms_per_call"] = ev0.elapsed_time(ev1) / steps
    return out


def run_config1(local, steps, warm, cpu=True):
    """Config 1: the uniform level-5 tree (256 x 256 cells, 341 blocks), FP64 Poisson
    solve from a zero guess to 1e-10 (the reference's own CPU-runnable case), through
    the persistent engine in plain FP64, FP64 with the direct coarsest solve, and mixed
    precision; event-timed per solve on the context's stream; beside it one complete
    oracle solve on the host cores."""
    import torch
    from srmg import gen, multigrid as mg
    p = gen.config1()
    tol = 1e-10
    ctx = mg.Context(local).set_tree(p.tree, p.conn)
    b = torch.from_numpy(p.b).cuda(local)
    u = torch.zeros_like(b)
    out = {"workload": "config1: uniform level-5 tree (256 x 256 cells, 341 blocks), Poisson, cylindrical r-z, "
                       "tol 1e-10", "blocks": p.tree.nblocks(), "tol": tol}
    for mode, name in ((mg.MODE_FP64, "fp64"), (mg.MODE_FP64_DIRECT, "fp64_direct_coarse"), (mg.MODE_MIXED, "mixed")):
        ms, st = [], None
        for i in range(warm + steps):
            u.zero_()
            torch.cuda.synchronize()
            st = mg.solve(ctx, u, b, p.s, p.geom, p.bc, tol=tol, mode=mode, max_cycles=5000)
            if i >= warm:
                ms.append(st["device_ms"])
        out[name] = {"value": 1e3 / float(np.mean(ms)), "unit": "solves/s", "ms_per_solve": float(np.mean(ms)),
                     "cycles": st["cycles"], "rel_residual": st["rel_residual"]}
    if cpu:
        _, c, rel, dt = oracle_solve(p, tol)
        out["cpu_baseline"] = {"value": 1.0 / dt, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
                               "cycles": c, "rel_residual": rel,
                               "sample": f"one complete oracle FP64 solve from a zero guess to {tol:g} ({c} V-cycles)"}
    ctx.close()
    return out


def run_batch(local, stream, steps, rank=0, world=1, pg=None, dev=None):
    """Config 3: 16 independent trees with leaf counts log-uniform in [1e5, 3e6], each
    with one Poisson and three photoionization Helmholtz right-hand sides: 64 solves to
    1e-8 in ONE persistent launch (graph-captured batch), against the same 64 solves
    run one by one in plain FP64 and in mixed precision.  With several ranks the trees
    are shared out round-robin (no exchange); times are the max over ranks and the
    solves/s count every rank's items (strong scaling: the 64 solves are fixed)."""
    import torch
    from srmg import gen, multigrid as mg
    from srmg.tree import leaf_cells
    all_trees = gen.config3_tree_problems()
    trees = [all_trees[i] for i in shard(len(all_trees), rank, world)]
    n_total = 4 * len(all_trees)
    ctxs, items = [], []
    for pois, terms in trees:
        c = mg.Context(local).set_tree(pois.tree, pois.conn)
        c.set_stream(stream.cuda_stream)
        ctxs.append(c)
        for p in [pois] + terms:
            items.append((c, p))
    disc = lambda p: ("helmholtz", p.k2) if p.op else None
    batch = mg.Batch([(c, p.s, disc(p), p.bc) for c, p in items], gen.GEOM_CYL1, device=local)
    batch.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        us = [torch.zeros(p.b.shape, dtype=torch.float64, device="cuda") for _, p in items]
        bs = [torch.from_numpy(p.b).cuda() for _, p in items]
    stream.synchronize()
    ref_opts = dict(tol=TOL, ndown=2, ntop=4, nup=2, max_cycles=5000)   # plain FP64: the reference's cycle
    tuned_opts = dict(tol=TOL, max_cycles=5000, **mg.TUNED)               # mixed: the tuned smoother
    opts_of = {mg.MODE_MIXED: tuned_opts, mg.MODE_FP64: ref_opts}

    def zero():
        with torch.cuda.stream(stream):
            for u in us:
                u.zero_()
        stream.synchronize()

    batch.set_option("graph", 1)
    res = {}
    for mode, name in ((mg.MODE_MIXED, "mixed"), (mg.MODE_FP64, "fp64")):
        zero()
        batch.solve(us, bs, mode=mode, **opts_of[mode])  # warm-up (capture)
        ms = []
        n = steps if mode == mg.MODE_MIXED else 1
        for _ in range(n):
            zero()
            st = batch.solve(us, bs, mode=mode, **opts_of[mode])
            ms.append(st[0]["device_ms"])
        t = max_over_ranks(float(np.mean(ms)), pg, dev)
        res[name + "_batched"] = {"value": n_total / (t / 1e3), "unit": "solves/s",
                                  "ms_per_batch": t,
                                  "max_cycles": max(x["cycles"] for x in st),
                                  "max_rel_residual": max(x["rel_residual"] for x in st)}
    for mode, name in ((mg.MODE_MIXED, "mixed"), (mg.MODE_FP64, "fp64")):
        tot = 0.0
        for k, (c, p) in enumerate(items):
            with torch.cuda.stream(stream):
                us[k].zero_()
            stream.synchronize()
            st = mg.solve(c, us[k], bs[k], p.s, p.geom, p.bc, disc(p), mode=mode, **opts_of[mode])
            tot += st["device_ms"]
        tot = max_over_ranks(tot, pg, dev)
        res[name + "_solo"] = {"value": n_total / (tot / 1e3), "unit": "solves/s", "ms_total": tot}
    out = {"workload": "config3: 16 trees (leaf cells log-uniform 1e5-3e6) x (Poisson + 3 Helmholtz "
                       "photoionization terms), cylindrical r-z, tol 1e-8, one graph-captured persistent launch",
           "items": n_total, "leaf_cells": int(sum(leaf_cells(p.tree) for p, _ in all_trees)),
           "scaling": "strong", "ranks": world,
           "blocks": batch.total_blocks, **res,
           "speedup_mixed_batched_vs_fp64_solo": res["mixed_batched"]["value"] / res["fp64_solo"]["value"],
           "speedup_mixed_batched_vs_fp64_batched": res["mixed_batched"]["value"] / res["fp64_batched"]["value"]}
    batch.close()
    for c in ctxs:
        c.close()
    return out


def run_learned(local, npairs):
    """Config 4: the learned warm start.  Solve pairs from seeded streamer runs on
    config-1-sized trees (1.5 MV/m applied field), generated by the library's own solver;
    the BF16 network trained by the library's kernels; then on held-out runs every 20th
    step is solved to 1e-8 from a zero guess, the previous-step potential, the time
    extrapolation, and the learned guess (mixed precision), plus the plain FP64 solve
    from the previous-step potential.  Times include the prediction."""
    import torch
    from srmg import learn, multigrid as mg
    runs = max(1, npairs // 2500)
    t0 = time.time()
    pairs = learn.generate(runs=runs, steps=(npairs + runs - 1) // runs + 2, seed=1, device=local)
    t_gen = time.time() - t0
    net = mg.Cnn(local, seed=5)
    t0 = time.time()
    losses = learn.train(net, pairs, steps=3000, batch=4, lr=1e-3, mu=0.001)
    torch.cuda.synchronize()
    t_train = time.time() - t0
    ev = learn.evaluate(net, runs=2, steps=1500, every=20, seed=77, device=local)
    ev_fp64 = learn.evaluate(net, runs=1, steps=600, every=20, seed=78, device=local, mode=mg.MODE_FP64)
    out = {"workload": "config4: streamer runs on the uniform level-5 tree (256 x 256 cells), 1.5 MV/m, "
                       "Poisson solves to 1e-8 along held-out runs",
           "pairs": int(pairs.n), "generate_s": t_gen, "train_steps": 3000, "train_s": t_train,
           "loss_first": losses[0], "loss_last": float(np.mean(losses[-100:])),
           "mixed": ev, "fp64": {k: ev_fp64[k] for k in ("zero", "prev", "extrapolated", "learned")}}
    fp64_prev_ms = ev_fp64["prev"]["mean_ms"]
    out["solves_per_s"] = {"mixed_learned": 1e3 / ev["learned"]["mean_ms"],
                           "mixed_prev": 1e3 / ev["prev"]["mean_ms"],
                           "fp64_prev": 1e3 / fp64_prev_ms,
                           "fp64_zero": 1e3 / ev_fp64["zero"]["mean_ms"]}
    out["speedup_mixed_learned_vs_fp64_prev"] = fp64_prev_ms / ev["learned"]["mean_ms"]
    out["speedup_mixed_learned_vs_fp64_zero"] = ev_fp64["zero"]["mean_ms"] / ev["learned"]["mean_ms"]
    del pairs
    torch.cuda.empty_cache()
    return out, net


def run_config5(local, net, steps, cpu=True):
    """Config 5: the full-size timestep field solve (Poisson + 3 Helmholtz per step,
    learned warm start + mixed precision) on the 8-12M-leaf tree, beside the plain FP64
    GPU solves of sampled steps and, on rank 0, one complete oracle FP64 Poisson solve of
    the same tree on the host cores (from a zero guess to 1e-8)."""
    from srmg import timestep
    out, problem = timestep.run(net, steps=steps, device=local)
    if cpu:
        _, c, rel, dt = oracle_solve(problem, TOL)
        out["cpu_baseline"] = {"value": 1.0 / dt, "unit": "Poisson solves/s", "cores": os.cpu_count(),
                               "kind": "port", "cycles": c, "rel_residual": rel, "s_per_solve": dt,
                               "sample": f"one complete oracle FP64 Poisson solve of this tree from a zero guess "
                                         f"to {TOL:g} ({c} V-cycles, {dt:.1f} s)"}
    return out


def run_rows(local):
    """The widened rows, FP64 on the per-operation kernels (replayed from CUDA graphs;
    the sequencer's single launch alongside), event-timed on one stream:
    the compact order-4 Laplacian on a refined BoxStencil tree (beside the order-2
    Laplacian on the same tree and path), a uniform level-4 octree (512 finest blocks,
    order-2 and order-4), and the free-boundary step on the config-2 tree at the
    transform lengths of a level-9 and a level-11 tree.  Roofline: the V-cycle byte
    model (srmg.model.vcycle_bytes, 3w per cell per GS iteration whatever the stencil)
    against the measured copy peak."""
    import torch
    from srmg import gen, gen3, model, multigrid as mg
    from srmg.tree3 import Tree3, populate, connectivity as connectivity3, STAR3, BOX3
    hbm, _ = peaks()
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)

    def time_vcycles(ctx, b_np, s, geom, bc, lpl, n=8):
        ctx.set_stream(stream.cuda_stream)
        b = torch.from_numpy(b_np).to(dev)
        u, r, u1 = torch.zeros_like(b), torch.zeros_like(b), torch.zeros_like(b)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            # warm-up with the timed call's own key: its graph or sequence is recorded here
            mg.vcycle_(ctx, u, b, r, u1, s, geom, bc, lpl, ndown=2, ntop=4, nup=2, ncycles=n)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            l0 = ctx.launches()
            e0.record(stream)
            mg.vcycle_(ctx, u, b, r, u1, s, geom, bc, lpl, ndown=2, ntop=4, nup=2, ncycles=n)
            e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / n, (ctx.launches() - l0) / n

    def line(tree, ms, launches, extra=None):
        B = model.vcycle_bytes(tree, 8, 2, 2, 4)
        d = {"blocks": tree.nblocks(), "ms_per_vcycle": ms, "launches_per_vcycle": launches, "model_bytes": B,
             "achieved_GBps": B / (ms / 1e3) / 1e9, "frac_of_measured_hbm": B / (ms / 1e3) / 1e9 / hbm}
        d.update(extra or {})
        return d

    out = {}
    p = gen.order4_problem(seed=41, geom=gen.GEOM_CYL1, base_level=6, extra=3)
    ctx = mg.Context(local).set_tree(p.tree, p.conn)
    ms4, l4 = time_vcycles(ctx, p.b, p.s, p.geom, p.bc, "laplacian4")
    ms2, l2 = time_vcycles(ctx, p.b, p.s, p.geom, p.bc, None)
    # the same cycles as one sequencer launch instead of a replayed CUDA graph
    ctx.set_option("op_sequencer", 1)
    ms4q, l4q = time_vcycles(ctx, p.b, p.s, p.geom, p.bc, "laplacian4")
    ctx.set_option("op_sequencer", 0)
    out["order4_2d"] = {"workload": f"{p.name}: compact order-4 Laplacian, cylindrical r-z, BoxStencil tree",
                        "order4": line(p.tree, ms4, l4), "order2_same_tree_per_op": line(p.tree, ms2, l2),
                        "order4_sequencer": line(p.tree, ms4q, l4q)}
    ctx.close()
    t = Tree3((1, 1, 1), 4)
    populate(t, 4)
    for name, op, st in (("order2", 0, STAR3), ("order4", 2, BOX3)):
        conn = connectivity3(t, st)
        p3 = gen3.make_problem3(t, conn, lambda x, y, z: np.sin(3 * x) * np.cos(2 * y) * z, (1.0 / 16) ** 2, op=op)
        ctx = mg.Context(local, D=3).set_tree(t, conn)
        lpl = {0: None, 2: "laplacian4"}[op]
        ms, ln = time_vcycles(ctx, p3.b, p3.s, 0, p3.bc, lpl)
        ctx.set_option("op_sequencer", 1)
        msq, lnq = time_vcycles(ctx, p3.b, p3.s, 0, p3.bc, lpl)
        row = out.setdefault("octree_3d", {"workload": "uniform level-4 octree (585 blocks, 2.1M finest cells), "
                                                       "Cartesian, Dirichlet"})
        row[name] = line(t, ms, ln)
        row[name + "_sequencer"] = line(t, msq, lnq)
        ctx.close()
    from srmg import freebc as fbc
    p = gen.config2(seed=2, target_leaf=1_500_000)
    ctx = mg.Context(local).set_tree(p.tree, p.conn)
    ctx.set_stream(stream.cuda_stream)
    q = torch.from_numpy(p.b).to(dev)
    u = torch.from_numpy(np.random.default_rng(0).standard_normal(p.b.shape)).to(dev)
    torch.cuda.synchronize()
    fb = {}
    for level in (9, 11):
        n, _, _, f = fbc.kernel(1, level, (1, 1), p.h1)
        mg.freebc_set(ctx, 1, level, (1, 1), f)
        with torch.cuda.stream(stream):
            for _ in range(2):
                mg.freebc_(ctx, q, u, p.h1, p.s)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(5):
                mg.freebc_(ctx, q, u, p.h1, p.s)
            e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / 5
        fb[str(n)] = {"ms": ms, "fp64_GFLOPs": 4.0 * n * n / (ms / 1e3) / 1e9}
    out["freebc"] = {"workload": "freebc! on the config-2 tree (outer column gather, DST-II, times f, DST-III, "
                                 "setouter), transform length n", "by_n": fb}
    ctx.close()
    return out


def vcycle_only(args):
    """Plain FP64 V-cycles (the persistent engine) on one config: W warm-up cycles, then
    K timed cycles with CUDA events; prints one JSON line.  Used for ncu captures."""
    import torch
    from srmg import gen, model, multigrid as mg
    problem = {"config1": gen.config1, "config2": lambda: gen.config2(seed=SEED, target_leaf=args.target_leaf),
               "config5": gen.config5}[args.config]()
    ctx = mg.Context(0).set_tree(problem.tree, problem.conn)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    b = torch.from_numpy(problem.b).cuda()
    u, r, u1 = torch.zeros_like(b), torch.zeros_like(b), torch.zeros_like(b)
    torch.cuda.synchronize()
    if args.only == "smooth":
        import ctypes
        L = problem.tree.finest_level()
        sl = problem.s / 4 ** (L - 1)
        bca = np.ascontiguousarray(problem.bc, dtype=np.int8)
        run = lambda n: ctx.check(mg.lib().srmg_gs_iter_dev(ctx.handle, u.data_ptr(), b.data_ptr(), problem.nblk, L,
                                                            1.0, sl, n, problem.op, problem.k2, problem.geom,
                                                            bca.ctypes.data))
        with torch.cuda.stream(stream):
            run(args.warmup)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run(args.steps)
            e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / max(1, args.steps)
        nb = len(problem.tree[L - 1])
        byts = nb * 256 * 24  # model: read u, b; write u per iteration
        print(json.dumps({"only": "smooth", "config": args.config, "level": L, "blocks": nb,
                          "us_per_iteration": ms * 1e3, "model_GBps": byts / (ms / 1e3) / 1e9}))
        ctx.close()
        return
    with torch.cuda.stream(stream):
        mg.vcycle_(ctx, u, b, r, u1, problem.s, problem.geom, problem.bc, ndown=2, ntop=4, nup=2,
                   ncycles=args.warmup)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        mg.vcycle_(ctx, u, b, r, u1, problem.s, problem.geom, problem.bc, ndown=2, ntop=4, nup=2,
                   ncycles=args.steps)
        e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / max(1, args.steps)
    B = model.vcycle_bytes(problem.tree, 8, 2, 2, 4)
    print(json.dumps({"only": "vcycle", "config": args.config, "blocks": problem.tree.nblocks(),
                      "ms_per_vcycle": ms, "model_bytes": B, "model_GBps": B / (ms / 1e3) / 1e9}))
    ctx.close()


def cnn_only(args):
    """The warm-start network's inference forward on --samples random BF16 block samples:
    W untimed calls, then K timed calls of each forward (mma.sync, tcgen05) with CUDA
    events on the network's stream; prints one JSON line.  Used for ncu captures."""
    import torch
    from srmg import multigrid as mg
    net = mg.Cnn(0, seed=7)
    g = torch.Generator(device="cuda")
    g.manual_seed(SEED)
    x = torch.randn((args.samples, 400, 2), generator=g, device="cuda").to(torch.bfloat16)
    torch.cuda.synchronize()
    out = {"only": "cnn", "samples": args.samples, "params": net.nparams,
           "macs_per_sample": 2 * 9 * 32 * 400 + 4 * 9 * 32 * 32 * 400 + 9 * 32 * 400}
    for name, fwd in (("mma_sync", net.forward), ("tcgen05", net.forward_tc)):
        for _ in range(args.warmup):
            fwd(x)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            y = fwd(x)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) / max(1, args.steps) * 1e3
        # each call synchronises the network's stream, so the wall clock brackets the
        # device work plus one launch and synchronisation
        out[name] = {"ms_per_forward": ms, "tflops": 2 * out["macs_per_sample"] * args.samples / (ms / 1e3) / 1e12,
                     "finite": bool(torch.isfinite(y).all()), "timing": "wall clock around synchronous calls"}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
