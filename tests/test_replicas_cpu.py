"""The multi-process path of bench.py on the CPU: two ranks over gloo
(127.0.0.1), as torchrun launches them. The time step does not shard, so
N GPUs run N independent replicas; the only cross-rank steps are the barrier
around the timed region and the maximum of the per-rank times, which these
tests exercise."""
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


def _rank(rank, ws, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import bench
    w, r, local = bench._dist()
    dist = bench._maybe_init(w, local)
    try:
        bench._barrier(dist)
        mx = bench._max_over_ranks(dist, float(10 + 5 * rank))
        q.put((r, w, mx))
    finally:
        dist.destroy_process_group()


def test_two_ranks_barrier_and_max():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == [(0, 2, 15.0), (1, 2, 15.0)]


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench._maybe_init(1, 0) is None
    assert bench._max_over_ranks(None, 3.5) == 3.5
