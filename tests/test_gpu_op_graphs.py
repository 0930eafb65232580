"""Per-operation V-cycles run three ways -- kernel by kernel, replayed from a captured
CUDA graph (option `op_graphs`), and as one cooperative launch of the sequencer (option
`op_sequencer`, on by default) -- give bit-identical results for every key (fields,
operator, sweep counts, tree): a BoxStencil order-4 tree, a StarStencil tree with the
persistent engine off, and an octree (order-2 and order-4 stencils)."""
import numpy as np
import pytest

from conftest import gpu_available
from srmg import gen, gen3, multigrid as mg
from srmg.tree3 import Tree3, populate, connectivity as connectivity3, STAR3, BOX3

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]


def cases():
    p4 = gen.order4_problem(seed=51, geom=gen.GEOM_CYL1)
    yield "order4_box", (lambda: mg.Context(0).set_tree(p4.tree, p4.conn)), p4.b, p4.s, p4.geom, p4.bc, "laplacian4"
    p2 = gen.config2(seed=5, target_leaf=40_000, extra=3)

    def star_no_engine():
        return mg.Context(0).set_tree(p2.tree, p2.conn).set_option("engine", 0)
    yield "star_engine_off", star_no_engine, p2.b, p2.s, p2.geom, p2.bc, None
    t = Tree3((1, 1, 1), 3)
    populate(t, 3)
    conn = connectivity3(t, STAR3)
    p3 = gen3.make_problem3(t, conn, lambda x, y, z: np.cos(4 * x) * y * (1 - z), (1.0 / 16) ** 2)
    yield "octree", (lambda: mg.Context(0, D=3).set_tree(t, conn)), p3.b, p3.s, 0, p3.bc, None
    conn4 = connectivity3(t, BOX3)
    p34 = gen3.make_problem3(t, conn4, lambda x, y, z: np.sin(3 * x) * y * (1 - z), (1.0 / 16) ** 2, op=2)
    yield "octree_order4", (lambda: mg.Context(0, D=3).set_tree(t, conn4)), p34.b, p34.s, 0, p34.bc, "laplacian4"


MODES = {"kernels": dict(op_graphs=0, op_sequencer=0), "graphs": dict(op_graphs=1, op_sequencer=0),
         "sequencer": dict(op_graphs=0, op_sequencer=1)}


@pytest.mark.parametrize("case", list(cases()), ids=lambda c: c[0])
def test_replay_and_sequencer_are_bit_identical(case):
    import torch
    _, make, b0, s, geom, bc, lpl = case
    results = {}
    for mode, opts in MODES.items():
        ctx = make()
        for k, v in opts.items():
            ctx.set_option(k, v)
        b = torch.from_numpy(b0).cuda()
        u, r, u1 = torch.zeros_like(b), torch.zeros_like(b), torch.zeros_like(b)
        torch.cuda.synchronize()
        outs = []
        l0 = ctx.launches()
        # two calls of the same key (record / capture, then replay), then a new key (other s)
        for ss in (s, s, 0.5 * s):
            mg.vcycle_(ctx, u, b, r, u1, ss, geom, bc, lpl, ndown=2, ntop=4, nup=2, ncycles=2)
            ctx.synchronize()
            outs.append(u.cpu().numpy().copy())
        results[mode] = (outs, ctx.launches() - l0)
        ctx.close()
    for mode in ("graphs", "sequencer"):
        for a, g in zip(results["kernels"][0], results[mode][0]):
            np.testing.assert_array_equal(a.view(np.uint64), g.view(np.uint64), err_msg=mode)
    assert results["sequencer"][1] == 3  # one launch per call
