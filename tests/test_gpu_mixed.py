"""Mixed-precision capacitance matrix M = I + Z^T D^-1 Z: the tensor-core SYRK of the BF16 split
(rows with small weight) plus the exact FP64 sum of the others, against numpy FP64; and the IPM
that uses it (with refinement of every solve) against the FP64 IPM on the same Z."""
import ctypes

import numpy as np
import pytest

from conftest import jaccard
from oracle import oracle as orc
from tensorsvm_b200 import _lib, api, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def syrk_mixed(ctx, Z, k, dinv, tau, ways):
    n, ldz = Z.shape
    Zd, dd = dev(Z), dev(dinv)
    M = torch.empty((k, k), dtype=torch.float64, device="cuda")
    cnt = ctypes.c_int32()
    _lib.check(ctx.lib.tsvm_test_syrk_mixed(ctx.handle, Zd.data_ptr(), ldz, n, k, dd.data_ptr(),
                                            float(tau), ways, M.data_ptr(), ctypes.byref(cnt)),
               "syrk_mixed")
    return M.cpu().numpy(), cnt.value


# n not a multiple of the 64-row chunk, k both below and at the 128/256 strip sizes, ldz > k;
# k > 256 through column windows (3 groups up to 384, 5 groups up to 425)
@pytest.mark.parametrize("n,k,ways", [(70001, 256, 2), (70001, 256, 3), (5000, 100, 2),
                                      (4096, 32, 3), (130, 256, 2), (64, 200, 2),
                                      (9001, 300, 2), (20000, 400, 2), (777, 425, 3)])
@pytest.mark.parametrize("tau", [100.0, float("inf"), 0.0])
def test_syrk_mixed_accuracy(ctx, n, k, ways, tau):
    rng = np.random.default_rng(n + k + ways)
    ldz = (k + 3) // 4 * 4 + 4
    Z = rng.standard_normal((n, ldz)).astype(np.float32)
    dinv = np.exp(rng.uniform(np.log(1e-4), np.log(1e4), n))
    M, cnt = syrk_mixed(ctx, Z, k, dinv, tau, ways)
    Zk = Z[:, :k].astype(np.float64)
    ref = np.eye(k) + (Zk * dinv[:, None]).T @ Zk
    assert cnt == int(np.sum(dinv > tau))
    assert np.array_equal(M, M.T)
    scale = np.sqrt(np.outer(np.diag(ref), np.diag(ref)))
    err = np.max(np.abs(M - ref) / scale)
    # BF16 hi+lo keeps ~16 significant bits (lo*lo dropped), hi+mid+lo ~24, both summed in
    # FP32 by the tensor cores; rows above tau are exact
    tol = 1e-12 if tau == 0.0 else (1e-4 if ways == 2 else 2e-5)
    assert err < tol, err


@pytest.mark.parametrize("n,k", [(70001, 256), (130, 256), (5000, 128), (3001, 250), (64, 64)])
@pytest.mark.parametrize("tau", [100.0, float("inf")])
def test_syrk_fused_matches_two_kernel_path(ctx, n, k, tau):
    """With ldz <= 256 the 2-way SYRK scales and splits Z inside the tensor-core kernel; with a
    wider ldz it runs the separate split kernel and the TMA-fed SYRK.  Both feed the same BF16
    parts to the same MMAs over the same row ranges, so M must agree bit for bit, and both must
    meet the FP64 bound."""
    rng = np.random.default_rng(3 * n + k)
    ldz_fused = (k + 3) // 4 * 4
    Z = rng.standard_normal((n, ldz_fused + 260)).astype(np.float32)
    dinv = np.exp(rng.uniform(np.log(1e-4), np.log(1e4), n))
    Mf, cf = syrk_mixed(ctx, np.ascontiguousarray(Z[:, :ldz_fused]), k, dinv, tau, 2)
    Mp, cp = syrk_mixed(ctx, Z, k, dinv, tau, 2)
    assert cf == cp
    assert np.array_equal(Mf, Mp)
    Zk = Z[:, :k].astype(np.float64)
    ref = np.eye(k) + (Zk * dinv[:, None]).T @ Zk
    scale = np.sqrt(np.outer(np.diag(ref), np.diag(ref)))
    assert np.max(np.abs(Mf - ref) / scale) < 1e-4


@pytest.fixture(scope="module")
def prob(ctx):
    X, y = synth.two_gaussians(20000, 18, seed=2, noise=0.1)
    Z, _ = api.factor(ctx, dev(X), dev(y), 0.05, 128, "fp32")
    return X, y, Z


def test_ipm_mixed_wide_k_matches_fp64(ctx):
    # k = 400 (the d = 54 configuration's rank): the capacitance matrix through four windows.
    # The benchmark's stopping rule: on this flat kernel the absolute 1e-7 residual rule can end
    # in max/min(D) > 1e18 (WARN_ILL_CONDITIONED) before the residual rule is met.
    X, y, g, C, _ = synth.make("c3", n=20000)
    k = 400
    Z, _ = api.factor(ctx, dev(X), dev(y), g, k, "fp32")
    yd = dev(y)
    a64, _, _, s64 = api.ipm(ctx, Z, yd, k, C, precision=_lib.PREC_FP32, rel_gap_tol=1e-6)
    am, _, _, sm = api.ipm(ctx, Z, yd, k, C, precision=_lib.PREC_BF16, rel_gap_tol=1e-6)
    assert s64["mixed_syrk"] == 0 and sm["mixed_syrk"] == 1
    assert s64["status_code"] == _lib.OK and sm["status_code"] == _lib.OK, (s64, sm)
    assert abs(sm["iters"] - s64["iters"]) <= 2, (sm["iters"], s64["iters"])
    assert abs(sm["pobj"] - s64["pobj"]) / abs(s64["pobj"]) < 1e-6
    Zh = Z.cpu().numpy()[:, :k].astype(np.float64)
    f64 = Zh @ (Zh.T @ (a64.cpu().numpy() * y))
    fm = Zh @ (Zh.T @ (am.cpu().numpy() * y))
    assert np.max(np.abs(fm - f64)) < 1e-4 * max(1.0, np.max(np.abs(f64)))


@pytest.mark.parametrize("sweeps", [1, 2])
def test_ipm_mixed_matches_fp64(ctx, prob, sweeps):
    X, y, Z = prob
    n, k, C = len(y), 128, 32.0
    yd = dev(y)
    a64, _, _, s64 = api.ipm(ctx, Z, yd, k, C, precision=_lib.PREC_FP32)
    am, _, _, sm = api.ipm(ctx, Z, yd, k, C, precision=_lib.PREC_BF16, refine_sweeps=sweeps)
    assert s64["mixed_syrk"] == 0 and sm["mixed_syrk"] == 1
    assert sm["status_code"] == _lib.OK, sm
    assert abs(sm["iters"] - s64["iters"]) <= 2, (sm["iters"], s64["iters"])
    assert abs(sm["pobj"] - s64["pobj"]) / abs(s64["pobj"]) < 1e-7
    assert abs(sm["dobj"] - s64["dobj"]) / abs(s64["dobj"]) < 1e-7
    assert sm["exact_rows_mean"] < 0.1 * n
    assert sm["refine_res_max"] < 1e-2
    a64, am = a64.cpu().numpy(), am.cpu().numpy()
    Zh = Z.cpu().numpy()[:, :k].astype(np.float64)
    f64 = Zh @ (Zh.T @ (a64 * y))
    fm = Zh @ (Zh.T @ (am * y))
    assert np.max(np.abs(fm - f64)) < 1e-4 * max(1.0, np.max(np.abs(f64)))
    sv64, _ = orc.sv_sets(a64, C)
    svm, _ = orc.sv_sets(am, C)
    assert jaccard(sv64, svm) >= 0.999


def test_ipm_mixed_rel_gap_stop(ctx, prob):
    X, y, Z = prob
    k, C = 128, 32.0
    _, _, _, sm = api.ipm(ctx, Z, dev(y), k, C, precision=_lib.PREC_BF16, rel_gap_tol=1e-6)
    assert sm["status_code"] == _lib.OK
    assert sm["rel_gap"] <= 1e-6 and sm["t_rel_gap_1e6_ms"] > 0
