"""Batched interior-point solve (tsvm_ipm_batched) against the single-problem solver on the same
factors: every problem of a small (C, gamma) grid of uneven sizes must end with the same status,
iteration count, objective and decision values as its own tsvm_ipm run."""
import numpy as np
import pytest

from oracle import oracle as orc
from tensorsvm_b200 import _lib, api, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def grid(ctx):
    # 8 problems, 600..9000 rows, k = 64 (two of them below one 4096-row work unit)
    probs = synth.grid_problems(count=8, lo=600, hi=9000, seed=7)
    k = 64
    Zs, ys, Cs = [], [], []
    for X, y, gamma, C in probs:
        Z, _ = api.factor(ctx, dev(X), dev(y), gamma, k, "fp32")
        Zs.append(Z)
        ys.append(dev(y))
        Cs.append(C)
    return Zs, ys, Cs, k


def decision(Z, k, a, y):
    Zh = Z.cpu().numpy()[:, :k].astype(np.float64)
    return Zh @ (Zh.T @ (a * y))


@pytest.mark.parametrize("rel_gap_tol", [0.0, 1e-6])
def test_batched_matches_single(ctx, grid, rel_gap_tol):
    Zs, ys, Cs, k = grid
    alphas, stats, info = api.ipm_batched(ctx, Zs, ys, k, Cs, rel_gap_tol=rel_gap_tol)
    assert info["units"] >= len(Zs) and info["unit_rows"] in (4096, 8192, 16384, 32768)
    assert info["graph_used"] == 1
    assert info["iters_max"] == max(s["iters"] for s in stats)
    for Z, y, C, a, s in zip(Zs, ys, Cs, alphas, stats):
        a1, _, _, s1 = api.ipm(ctx, Z, y, k, C, rel_gap_tol=rel_gap_tol)
        assert s["status"] == s1["status_code"]
        assert abs(s["iters"] - s1["iters"]) <= 1, (s["iters"], s1["iters"])
        assert abs(s["pobj"] - s1["pobj"]) <= 1e-8 * max(1.0, abs(s1["pobj"]))
        yh = y.cpu().numpy().astype(np.float64)
        f = decision(Z, k, a.cpu().numpy(), yh)
        f1 = decision(Z, k, a1.cpu().numpy(), yh)
        assert np.max(np.abs(f - f1)) <= 1e-5 * max(1.0, np.max(np.abs(f1)))
        sv, _ = orc.sv_sets(a.cpu().numpy(), C)
        sv1, _ = orc.sv_sets(a1.cpu().numpy(), C)
        assert len(set(sv.tolist()) ^ set(sv1.tolist())) <= max(1, len(sv1) // 1000)


@pytest.mark.parametrize("rel_gap_tol", [0.0, 1e-6])
def test_batched_mixed_matches_single_mixed(ctx, grid, rel_gap_tol):
    """The 16-bit precisions' batched solve (per work unit the tensor-core capacitance matrix
    of the rows with weight <= tau and the other rows exactly in FP64, one refinement sweep per
    capacitance solve, tau adapted per problem on the device) against the single-problem mixed
    solver on the same factors."""
    Zs, ys, Cs, k = grid
    alphas, stats, info = api.ipm_batched(ctx, Zs, ys, k, Cs, rel_gap_tol=rel_gap_tol,
                                          precision=_lib.PREC_BF16)
    assert info["graph_used"] == 1
    for Z, y, C, a, s in zip(Zs, ys, Cs, alphas, stats):
        a1, _, _, s1 = api.ipm(ctx, Z, y, k, C, rel_gap_tol=rel_gap_tol, precision=_lib.PREC_BF16)
        assert s1["mixed_syrk"] == 1
        assert s["status"] == s1["status_code"]
        assert abs(s["iters"] - s1["iters"]) <= 1, (s["iters"], s1["iters"])
        assert abs(s["pobj"] - s1["pobj"]) <= 1e-8 * max(1.0, abs(s1["pobj"]))
        yh = y.cpu().numpy().astype(np.float64)
        f = decision(Z, k, a.cpu().numpy(), yh)
        f1 = decision(Z, k, a1.cpu().numpy(), yh)
        assert np.max(np.abs(f - f1)) <= 1e-5 * max(1.0, np.max(np.abs(f1)))
        sv, _ = orc.sv_sets(a.cpu().numpy(), C)
        sv1, _ = orc.sv_sets(a1.cpu().numpy(), C)
        assert len(set(sv.tolist()) ^ set(sv1.tolist())) <= max(1, len(sv1) // 1000)


def test_batched_single_problem_and_launch_count(ctx, grid):
    Zs, ys, Cs, k = grid
    l0 = ctx.launches
    alphas, stats, info = api.ipm_batched(ctx, Zs[:1], ys[:1], k, Cs[:1])
    assert stats[0]["status"] == _lib.OK
    # every iteration is one replay of the captured graph: launches grow with iterations
    assert ctx.launches - l0 > 10 * stats[0]["iters"]


@pytest.mark.parametrize("prec,k", [("fp32", 64), ("fp16", 128), ("fp16_fast", 128), ("fp32", 130)])
def test_factor_batched_matches_single(ctx, prec, k):
    """tsvm_factor_batched (every problem through its projection, the eigenproblems in one
    launch, Z formed in place) gives the factor of tsvm_factor for each problem: the same
    kernels on the same data, the same eigensolver per problem (k = 130 takes the grid
    eigensolver one problem after the other)."""
    probs = synth.grid_problems(count=6, lo=700, hi=6000, seed=11)
    Xs = [dev(X) for X, _, _, _ in probs]
    ys = [dev(y) for _, y, _, _ in probs]
    gs = [g for _, _, g, _ in probs]
    Zb, infos = api.factor_batched(ctx, Xs, ys, gs, k, prec)
    for X, y, g, Z, info in zip(Xs, ys, gs, Zb, infos):
        Z1, info1 = api.factor(ctx, X, y, g, k, prec)
        assert info["realk"] == info1["realk"]
        assert abs(info["eig_min"] - info1["eig_min"]) <= 1e-9 * abs(info1["eig_max"])
        assert torch.allclose(Z, Z1, rtol=0, atol=1e-6 * float(Z1.abs().max()))
