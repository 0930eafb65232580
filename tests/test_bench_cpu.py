"""bench.py on the host: the reference arm (the oracle timed on the CPU) prints one
JSON line with the contract's keys, and the roofline byte model matches its stated
figures."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_json_line():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "1", "--target-leaf", "20000"],
                         capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config"):
        assert k in line, k
    assert line["value"] > 0 and line["unit"] == "solves/s" and line["higher_is_better"] is True
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    # every step is a complete solve to the tolerance: measured, not extrapolated
    cyc = line["fp64_cycles_per_solve"]
    assert cyc["extrapolated"] is False and cyc["cycles"] > 0 and cyc["rel_residual"] <= 1e-8
    assert abs(line["ms_per_step"] - 1e3 / line["value"]) <= 1e-6 * line["ms_per_step"]


def test_byte_model_figures():
    from srmg import gen, model
    from srmg.tree3 import Tree3, populate
    # config 1 (uniform level 5): 15.17 MB per FP64 V-cycle (164 B per level-l cell +
    # 40 B per level-(l-1) cell for (2,2,4))
    p = gen.config1()
    assert abs(model.vcycle_bytes(p.tree, 8, 2, 2, 4) - 15.17e6) < 0.01e6
    # the mixed solve's model: 8 FP32 V-cycles plus 5 defect, 5 restriction, 4 update passes
    n = model.level_cells(p.tree)
    N, N2 = sum(n), sum(n[1:])
    want = 8 * model.vcycle_bytes(p.tree, 4, 2, 2, 4) + 5 * (24 * N + 10 * N2) + 4 * 20 * N
    assert abs(model.mixed_solve_bytes(p.tree, 8, 4) - want) < 1.0
    # three dimensions: M^3 cells per block
    t = Tree3((1, 1, 1), 2)
    populate(t, 2)
    assert model.level_cells(t) == [16 ** 3, 8 * 16 ** 3]
