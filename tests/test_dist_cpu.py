"""Multi-process plumbing of bench.py on the host: two gloo ranks (no GPU) exercise the
process-group setup, the max-over-ranks timing, the barrier and the round-robin
sharding of independent trees.  The solve itself has no cross-rank exchange (replicas
of the config-2 solve, trees shared out for the config-3 batch).  Failure: a rank that
exits without joining the barrier makes the other's barrier end with an error, within
the process group's timeout, instead of waiting for good."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import torch
    import bench
    w, r, local, pg = bench.dist_setup(backend="gloo")
    dev = torch.device("cpu")
    m = bench.max_over_ranks(1.5 + r, pg, dev)
    bench.barrier(pg, dev)
    mine = bench.shard(16, r, w)
    q.put((r, w, m, mine))
    pg.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=100) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    out.sort()
    assert [o[1] for o in out] == [2, 2]
    assert all(o[2] == 2.5 for o in out)          # max over ranks seen by every rank
    shards = [set(o[3]) for o in out]
    assert shards[0].isdisjoint(shards[1]) and shards[0] | shards[1] == set(range(16))


def _worker_dies(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import time
    import torch
    import bench
    w, r, local, pg = bench.dist_setup(backend="gloo", timeout_s=10)
    dev = torch.device("cpu")
    bench.barrier(pg, dev)  # both ranks are up
    if r == 1:
        os._exit(0)  # leaves between steps, never joins the next barrier
    t0 = time.time()
    try:
        bench.barrier(pg, dev)
        q.put(("no error", time.time() - t0))
    except Exception as e:  # noqa: BLE001 -- any error ends the wait; the kind varies
        q.put((type(e).__name__, time.time() - t0))


@pytest.mark.timeout(120)
def test_rank_that_leaves_is_detected():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_dies, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    kind, waited = q.get(timeout=100)
    for p in procs:
        p.join(timeout=30)
    assert kind != "no error"
    assert waited < 60
