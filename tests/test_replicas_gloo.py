"""The multi-process path of bench.py (replicas: one process per GPU, no
collective on the data path) on CPU ranks over gloo: the process group,
the max over ranks that device times go through, the barrier, and the
whole-job value of N replicas."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist, r, w, local = bench.dist_init(world, backend="gloo")
    ms = 10.0 + 5.0 * r            # each rank's device time; the slowest bounds the job
    slowest = bench.allmax(dist, ms)
    bench.barrier(dist)
    q.put((r, w, slowest, bench.replica_value(w, 1000, 4, slowest)))
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_replicas_take_the_slowest_rank(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    slowest = 10.0 + 5.0 * (world - 1)
    for r, (rr, w, s, v) in enumerate(out):
        assert (rr, w) == (r, world)
        assert s == slowest
        assert abs(v - world * 1000 * 4 / (slowest / 1e3) / 1e9) < 1e-15


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.dist_init(1) == (None, 0, 1, 0)
    assert bench.allmax(None, 3.5) == 3.5
