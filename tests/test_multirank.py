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


# ---- row-sharded training restated in FP64 on gloo ranks --------------------------------

def _sharded_rank(rank, world, port, out, n, k):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import numpy as np
    import torch
    import torch.distributed as dist
    from oracle import oracle as orc
    from oracle import sharded
    from tensorsvm_b200 import synth
    from tensorsvm_b200.shard import partition
    dist.init_process_group("gloo", rank=rank, world_size=world)

    def allreduce(a, op):
        t = torch.from_numpy(a)
        dist.all_reduce(t, op=dist.ReduceOp.SUM if op == "sum" else dist.ReduceOp.MIN)

    X, y = synth.two_gaussians(n, 6, seed=31, noise=0.1)
    g, C = 0.2, 4.0
    row0, nr = partition(n, world)[rank]
    rows = slice(row0, row0 + nr)
    f = sharded.lra(X, y, g, k, row0, nr, allreduce)
    U = np.zeros((n, k))
    U[rows] = f.U
    allreduce(U, "sum")                  # assembled factor, for the comparison only
    r = sharded.mpc(U[rows], y[rows], C, allreduce, rel_gap_tol=None)
    x = np.zeros(n)
    x[rows] = r.x
    allreduce(x, "sum")
    b, bstd, counts = sharded.bias_rbf(U[rows], y[rows], r.x, C, rank, world, allreduce)
    out.put((rank, U, x, r.iters, r.log[-1], r.status, b, bstd, counts))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_row_sharded_lra_mpc_bias_reproduce_one_rank(world):
    """The row-sharded factor, interior-point solve and bias (every exchange the library's
    tsvm_comm path makes: Gram matrices, C, the gathered basis, k-vectors, scalars, minima,
    the capacitance matrix, the free-SV terms) on 2 and 3 gloo ranks -- 3 splits 1501 rows
    unevenly -- reproduce the single-process oracle: the same iteration count and objective to
    1e-12, the same factor and solution."""
    import numpy as np
    from oracle import oracle as orc
    from tensorsvm_b200 import synth
    n, k = 1501, 24
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_rank, args=(r, world, port, q, n, k))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    X, y = synth.two_gaussians(n, 6, seed=31, noise=0.1)
    f = orc.lra(X, y, 0.2, k, c_as_float32=False)
    G = f.U @ f.U.T
    for _, U, x, iters, last, status, b, bstd, counts in res:
        assert np.linalg.norm(U @ U.T - G) / np.linalg.norm(G) < 1e-10
    U = res[0][1]
    r1 = orc.mpc(U, y, 4.0)
    b1, bstd1 = orc.bias_rbf(U, y, r1.x, 4.0)
    sv, free = orc.sv_sets(r1.x, 4.0)
    for _, _, x, iters, last, status, b, bstd, counts in res:
        assert iters == r1.iters and status == r1.status
        assert abs(last[5] - r1.log[-1][5]) <= 1e-12 * abs(r1.log[-1][5])
        assert abs(last[6] - r1.log[-1][6]) <= 1e-12 * abs(r1.log[-1][6])
        assert np.max(np.abs(x - r1.x)) < 1e-8
        assert abs(b - b1) < 1e-9 and abs(bstd - bstd1) < 1e-9
        assert tuple(counts) == (len(sv), len(free))


def test_partition_is_contiguous_balanced_and_in_rank_order():
    from tensorsvm_b200.shard import partition
    for n, w in [(10, 3), (1_000_000, 8), (7, 7), (1501, 2)]:
        parts = partition(n, w)
        assert parts[0][0] == 0 and sum(nr for _, nr in parts) == n
        assert all(parts[i][0] + parts[i][1] == parts[i + 1][0] for i in range(w - 1))
        assert max(nr for _, nr in parts) - min(nr for _, nr in parts) <= 1
    with pytest.raises(ValueError):
        partition(3, 4)
