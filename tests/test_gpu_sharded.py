"""The row-sharded path of the library (tsvm_set_comm, tsvm_factor_rows, tsvm_ipm and tsvm_bias
on a rank's rows) against the single-process solve on the same GPU.

Two ranks run as two processes on the one GPU of the test box.  Their collectives go through
gloo on the host (TorchComm stages each buffer through host memory): no kernel of one process
waits on the other's, every exchange is a host-side all-reduce between launches.  On a
multi-GPU node the same code runs one process per GPU with NCCL.
"""
import os
import socket

import numpy as np
import pytest

from tensorsvm_b200 import _lib, api, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")

N, D, K, GAMMA, C = 6000, 18, 64, 0.05, 8.0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, prec, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch
    import torch.distributed as dist
    from tensorsvm_b200 import _lib, api, synth
    from tensorsvm_b200.shard import TorchComm, factor_rows, partition, set_comm
    try:
        import datetime
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=120))
        torch.cuda.set_device(0)
        X, y = synth.two_gaussians(N, D, seed=17, noise=0.1)
        Xd, yd = torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda()
        row0, nr = partition(N, world)[rank]
        comm = TorchComm()
        with _lib.Context(0) as ctx:
            set_comm(ctx, comm)
            Z, info = factor_rows(ctx, Xd, yd, row0, nr, GAMMA, K, prec)
            yl = yd[row0:row0 + nr].contiguous()
            alpha, _, _, st = api.ipm(ctx, Z, yl, K, C, rel_gap_tol=1e-8,
                                      precision=_lib.PREC_FP32 if prec == "fp32" else _lib.PREC_BF16)
            b, bstd, nsv, nfree = api.bias(ctx, Z, yl, alpha, K, C)
            out.put((rank, Z.cpu().numpy(), alpha.cpu().numpy(), st["iters"], st["pobj"],
                     st["dobj"], b, nsv, nfree, info["eig_min"], comm.calls, None))
        dist.destroy_process_group()
    except BaseException as e:  # report, do not hang the parent
        out.put((rank, None, None, 0, 0, 0, 0, 0, 0, 0, 0, repr(e)))


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_two_ranks_reproduce_single_process(ctx, prec):
    """Two ranks' factor rows, IPM and bias against one process on the whole problem: the
    assembled factor's Z Z^T, the IPM on it (same iterations, objective), the bias and counts."""
    world = 2
    spawn = mp.get_context("spawn")
    q = spawn.Queue()
    port = _free_port()
    procs = [spawn.Process(target=_rank, args=(r, world, port, prec, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        res = sorted((q.get(timeout=600) for _ in range(world)), key=lambda t: t[0])
    finally:
        for p in procs:
            p.join(timeout=120)
            if p.is_alive():   # a rank stuck on the host (its collective peer failed)
                p.kill()
    errors = [r[-1] for r in res if r[-1]]
    assert not errors, errors
    assert all(p.exitcode == 0 for p in procs)
    # the whole problem in this process
    X, y = synth.two_gaussians(N, D, seed=17, noise=0.1)
    Xd, yd = torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda()
    Z1, info1 = api.factor(ctx, Xd, yd, GAMMA, K, prec)
    Zs = np.concatenate([r[1] for r in res])[:, :K].astype(np.float64)
    Z1h = Z1.cpu().numpy()[:, :K].astype(np.float64)
    G1 = Z1h @ Z1h.T
    assert np.linalg.norm(Zs @ Zs.T - G1) / np.linalg.norm(G1) < 2e-5
    # the IPM on the assembled sharded factor, in one process
    Zsd = torch.from_numpy(np.ascontiguousarray(np.concatenate([r[1] for r in res]))).cuda()
    a1, _, _, st1 = api.ipm(ctx, Zsd, yd, K, C, rel_gap_tol=1e-8,
                            precision=_lib.PREC_FP32 if prec == "fp32" else _lib.PREC_BF16)
    b1, _, nsv1, nfree1 = api.bias(ctx, Zsd, yd, a1, K, C)
    alpha = np.concatenate([r[2] for r in res])
    for r in res:
        _, _, _, iters, pobj, dobj, b, nsv, nfree, _, calls, _ = r
        assert iters == st1["iters"]
        assert abs(pobj - st1["pobj"]) <= 1e-9 * abs(st1["pobj"])
        assert abs(dobj - st1["dobj"]) <= 1e-9 * abs(st1["dobj"])
        assert (nsv, nfree) == (nsv1, nfree1)
        assert abs(b - b1) <= 1e-7
        assert calls > 0
    assert np.max(np.abs(alpha - a1.cpu().numpy())) <= 1e-6 * C
