"""The N > 1 host path of bench.py (replicas, no collective on the data path) with two gloo
ranks on CPU: rendezvous, distinct replica problems, barrier and max-over-ranks timing."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    import torch.distributed as dist
    from tensorsvm_b200 import synth
    w, r, local = bench.dist_setup()
    X, y = synth.two_gaussians(256, 18, seed=bench.replica_seed(r), noise=bench.NOISE)
    bench.barrier(w)
    m = bench.dist_max([float(r + 1), float(-r)], w)
    out.put((r, m, float(X[0, 0]), dist.get_backend()))
    dist.destroy_process_group()


def test_two_gloo_ranks_max_over_ranks_and_distinct_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, x0, be0), (r1, m1, x1, be1) = res
    assert m0 == m1 == [2.0, 0.0]
    assert x0 != x1                      # each replica trains its own problem
    assert be0 == be1 == "gloo"
