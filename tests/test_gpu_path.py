"""Training-path parity on the GPU: factor vs the oracle's LRA on the same sketch, the IPM vs the
oracle's mpc on the same Z, bias, and end to end vs the reference's own model files."""
import os
import subprocess

import numpy as np
import pytest

from conftest import jaccard, ref_fixture, ref_log
from oracle import oracle as orc
from tensorsvm_b200 import _lib, api, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def c1():
    X, y, g, C, k = synth.make("c1")
    return X, y, g, C, k


@pytest.fixture(scope="module")
def c1_factor(ctx, c1):
    X, y, g, C, k = c1
    Z, info = api.factor(ctx, dev(X), dev(y), g, k, "fp32")
    return Z, info


def test_factor_fp32_matches_oracle_lra(c1, c1_factor):
    X, y, g, C, k = c1
    Z, info = c1_factor
    Zh = Z.cpu().numpy()[:, :k].astype(np.float64)
    assert np.all(Z.cpu().numpy()[:, k:] == 0)
    f = orc.lra(X, y, g, k)
    G, Gr = Zh @ Zh.T, f.U @ f.U.T
    err = np.linalg.norm(G - Gr) / np.linalg.norm(Gr)
    assert err < 1e-4, err
    assert info["realk"] == f.realk == k
    assert abs(info["eig_max"] - f.eigvals[-1]) / f.eigvals[-1] < 1e-5


def test_factor_error_vs_exact_kernel(c1, c1_factor):
    X, y, g, C, k = c1
    Z, _ = c1_factor
    Zh = Z.cpu().numpy()[:2048, :k].astype(np.float64)
    K = orc.rbf_block(X[:2048], X[:2048], y[:2048], y[:2048], g)
    f = orc.lra(X, y, g, k)
    e_gpu = np.linalg.norm(K - Zh @ Zh.T) / np.linalg.norm(K)
    e_orc = np.linalg.norm(K - f.U[:2048] @ f.U[:2048].T) / np.linalg.norm(K)
    assert abs(e_gpu - e_orc) < 1e-4 * max(1.0, e_orc)


def test_ipm_matches_oracle_mpc_on_same_z(ctx, c1, c1_factor):
    X, y, g, C, k = c1
    Z, _ = c1_factor
    alpha, xi, ym, st = api.ipm(ctx, Z, dev(y), k, C, want_xi=True)
    Zh = Z.cpu().numpy()[:, :k].astype(np.float64)
    r = orc.mpc(Zh, y, C, kernel="rbf")
    a = alpha.cpu().numpy()
    assert st["iters"] == r.iters
    assert abs(st["pobj"] - r.log[-1][5]) / abs(r.log[-1][5]) < 1e-9
    assert abs(st["dobj"] - r.log[-1][6]) / abs(r.log[-1][6]) < 1e-9
    assert np.max(np.abs(a - r.x)) < 1e-4
    b_gpu, _, nsv, nfree = api.bias(ctx, Z, dev(y), alpha, k, C)
    b_orc, _ = orc.bias_rbf(Zh, y, r.x, C)
    assert abs(b_gpu - b_orc) < 1e-6
    sv, free = orc.sv_sets(a, C)
    assert (nsv, nfree) == (len(sv), len(free))
    Xt = synth.make("c1_test")[0]
    dv_g = orc.decision_values_dense(a, y, X, g, b_gpu, Xt)
    dv_o = orc.decision_values_dense(r.x, y, X, g, b_orc, Xt)
    assert np.max(np.abs(dv_g - dv_o)) < 1e-4


def test_train_end_to_end_matches_reference(ctx, c1):
    X, y, g, C, k = c1
    m = api.train(ctx, X, y, _lib.KERNEL_RBF, g, C, k, "fp32")
    last = ref_log("ref_c1_rbf")[-1]
    st = m.ipm_stats
    assert abs(st["pobj"] - last[5]) / abs(last[5]) < 1e-5
    assert abs(st["dobj"] - last[6]) / abs(last[6]) < 1e-5
    idx, coef, rho, _ = ref_fixture("ref_c1_rbf")
    sv, _ = orc.sv_sets(m.alpha, C)
    # the FP64 oracle itself agrees with the reference build on SV Jaccard 0.9958 here (alpha
    # moves along the dual's nearly flat optimal face with the factor's rounding), so 0.999
    # would hold no exact solver; the prediction bar below is the 99.9 % one
    assert jaccard(sv, idx) > 0.99
    ref_alpha = np.zeros(len(X))
    ref_alpha[idx] = coef * y[idx]
    Xt = synth.make("c1_test")[0]
    dv = orc.decision_values_dense(m.alpha, y, X, g, m.b, Xt)
    dv_r = orc.decision_values_dense(ref_alpha, y, X, g, -rho, Xt)
    assert np.mean(np.sign(dv) == np.sign(dv_r)) >= 0.999


def test_linear_end_to_end_matches_reference(ctx, c1, tmp_path):
    X, y, g, C, k = c1
    m = api.train(ctx, X, y, _lib.KERNEL_LINEAR, 0.0, 1.0, 0, "fp32")
    r, w, b = orc.train_linear(X, y, 1.0)
    assert m.ipm_stats["iters"] == r.iters
    assert np.max(np.abs(m.alpha - r.x)) < 1e-6
    assert abs(m.b - b) < 1e-7
    path = tmp_path / "lin.model"
    api.write_model(str(path), m, X, y, 1, -1)
    got = path.read_text().split("\n")
    ref = open(os.path.join(os.path.dirname(__file__), "golden", "ref_c1_lin.model")).read().split("\n")
    assert got[:6] == ref[:6]
    assert np.allclose([float(v) for v in got[6:25]], [float(v) for v in ref[6:25]], atol=1e-8)


@pytest.mark.parametrize("n,k", [(1000, 50), (777, 33), (64, 8), (2500, 130)])
def test_ragged_shapes_match_oracle(ctx, n, k):
    X, y = synth.two_gaussians(n, 7, seed=n)
    g, C = 0.1, 4.0
    Z, info = api.factor(ctx, dev(X), dev(y), g, k, "fp32")
    f = orc.lra(X, y, g, k)
    Zh = Z.cpu().numpy()[:, :k].astype(np.float64)
    G, Gr = Zh @ Zh.T, f.U @ f.U.T
    assert np.linalg.norm(G - Gr) / np.linalg.norm(Gr) < 1e-4
    alpha, _, _, st = api.ipm(ctx, Z, dev(y), k, C)
    r = orc.mpc(Zh, y, C, kernel="rbf")
    assert abs(st["pobj"] - r.log[-1][5]) / max(1.0, abs(r.log[-1][5])) < 1e-8
    assert np.max(np.abs(alpha.cpu().numpy() - r.x)) < 1e-4 * C


def test_rel_gap_stop_and_stats(ctx, c1, c1_factor):
    X, y, g, C, k = c1
    Z, _ = c1_factor
    alpha, _, _, st = api.ipm(ctx, Z, dev(y), k, C, rel_gap_tol=1e-6)
    assert st["status_code"] == _lib.OK
    assert st["rel_gap"] <= 1e-6 and st["t_rel_gap_1e6_ms"] > 0


def test_ipm_iteration_cap_returns_its_own_status(ctx, c1, c1_factor):
    # the reference's 100-iteration cap (T:1603) as a distinct warning, outputs still valid
    X, y, g, C, k = c1
    Z, _ = c1_factor
    alpha, _, _, st = api.ipm(ctx, Z, dev(y), k, C, max_iter=3)
    assert st["status_code"] == _lib.WARN_MAX_ITER
    assert st["iters"] == 3
    a = alpha.cpu().numpy()
    assert np.all(np.isfinite(a)) and a.min() > 0.0 and a.max() < C


def test_allocation_failure_returns_status_and_context_recovers():
    # injected on the host, in a fresh context (every scratch buffer still to be allocated):
    # the failing allocation surfaces as TSVM_ERR_OUT_OF_MEMORY, not a crash, at the first
    # allocation and in the middle of a factorisation; with the hook off the same context works
    X, y = synth.two_gaussians(2000, 8, seed=4)
    with _lib.Context(0) as c:
        Xd, yd = dev(X), dev(y)
        for after in (0, 3):
            _lib.check(c.lib.tsvm_test_fail_alloc(c.handle, after), "fail_alloc")
            with pytest.raises(_lib.TsvmError) as err:
                api.factor(c, Xd, yd, 0.1, 32, "fp32")
            assert err.value.status == _lib.ERR_OUT_OF_MEMORY
        _lib.check(c.lib.tsvm_test_fail_alloc(c.handle, -1), "fail_alloc")
        Z, info = api.factor(c, Xd, yd, 0.1, 32, "fp32")
        alpha, _, _, st = api.ipm(c, Z, yd, 32, 1.0, rel_gap_tol=1e-6)
        assert st["status_code"] == _lib.OK and bool(torch.isfinite(alpha).all())


def test_ipm_nan_input_reports_not_spd(ctx):
    X, y = synth.two_gaussians(256, 3, seed=2)
    Z = torch.zeros((256, 64), dtype=torch.float32, device="cuda")
    Z[:, :3] = dev(X)
    Z[5, 1] = float("nan")
    alpha, _, _, st = api.ipm(ctx, Z, dev(y), 3, 1.0)
    assert st["status_code"] == _lib.ERR_NOT_SPD
    assert st["iters"] == 1


def test_cli_end_to_end(tmp_path):
    X, y = synth.two_gaussians(3000, 18, seed=11, noise=0.05)
    y = -y  # first label -1 becomes POS, as in the reference's remap
    train = tmp_path / "t.train"
    synth.write_libsvm(str(train), X, y)
    model = tmp_path / "t.model"
    p = subprocess.run([_lib.CLI_PATH, "-k", "32", "-c", "8", "-g", "0.05", "-t", "2", str(train),
                        str(model)], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    m = orc.parse_model(model.read_text())
    assert m["header"]["label"] == [str(int(y[0])), str(int(-y[0]))]
    assert m["header"]["kernel_type"] == ["rbf"]
    yy, pos, neg = orc.remap_labels(y)
    f, r, b = orc.train_rbf(X, yy, 0.05, 8.0, 32)
    sv, _ = orc.sv_sets(r.x, 8.0)
    assert abs(int(m["header"]["total_sv"][0]) - len(sv)) <= 0.01 * len(sv)
    dv = orc.decision_values(m, X[:500], 18)
    dv_o = orc.decision_values_dense(r.x, yy, X, 0.05, b, X[:500])
    assert np.mean(np.sign(dv) == np.sign(dv_o)) >= 0.995


# Z Z^T of the tensor-core factor against the FP64 oracle's.  Split forms (the kernel block as
# hi + lo in the range-finder pass, the basis as hi + lo in the projection pass): about FP32
# accuracy; one-product forms: the 16-bit rounding of both operands.
FACTOR_TOL = {"fp16": 5e-5, "bf16": 5e-4, "fp16_fast": 2e-3, "bf16_fast": 2e-2}


@pytest.mark.parametrize("prec", ["fp16", "bf16", "fp16_fast", "bf16_fast"])
def test_factor_tensor_core_matches_oracle(ctx, c1, prec):
    X, y, g, C, k = c1
    Z, info = api.factor(ctx, dev(X), dev(y), g, k, prec)
    Zh = Z.cpu().numpy()[:, :k].astype(np.float64)
    f = orc.lra(X, y, g, k)
    G, Gr = Zh @ Zh.T, f.U @ f.U.T
    err = np.linalg.norm(G - Gr) / np.linalg.norm(Gr)
    assert err < FACTOR_TOL[prec], err


@pytest.mark.parametrize("prec", ["fp16", "bf16", "fp16_fast", "bf16_fast"])
def test_factor_tensor_core_wide_features(ctx, prec):
    # d = 54 (the covtype-shaped config): Gram K = 192 on the tensor cores
    X, y, g, C, k = synth.make("c3", n=3000)
    k = 64
    Z, info = api.factor(ctx, dev(X), dev(y), g, k, prec)
    Zh = Z.cpu().numpy()[:, :k].astype(np.float64)
    f = orc.lra(X, y, g, k)
    G, Gr = Zh @ Zh.T, f.U @ f.U.T
    err = np.linalg.norm(G - Gr) / np.linalg.norm(Gr)
    assert err < FACTOR_TOL[prec], err


# Against the FP64 oracle (same sketch, same algorithm) on config 1's test split: objective
# and decision-value signs of the exact-kernel model (the model file's decision function).
# The FP16 split form is held to the bars of the tensor-core form (objective 1e-5, >= 99.9%
# signs); the others are held to what they measure, stated here.
@pytest.mark.parametrize("prec,pobj_tol,signs", [("fp16", 1e-5, 0.999), ("bf16", 2e-5, 0.99),
                                                 ("fp16_fast", 1e-4, 0.98)])
def test_train_tensor_core_against_fp64_oracle(ctx, c1, prec, pobj_tol, signs):
    X, y, g, C, k = c1
    m = api.train(ctx, X, y, _lib.KERNEL_RBF, g, C, k, prec)
    f, r, b = orc.train_rbf(X, y, g, C, k)
    st = m.ipm_stats
    assert abs(st["pobj"] - r.log[-1][5]) / abs(r.log[-1][5]) < pobj_tol
    Xt = synth.make("c1_test")[0]
    dv = orc.decision_values_dense(m.alpha, y, X, g, m.b, Xt)
    dv_o = orc.decision_values_dense(r.x, y, X, g, b, Xt)
    # k = 32 keeps eigen-directions down to 3.6e-4 of the largest; the flat rank-32 dual moves
    # alpha along them when the factor's weak directions move, which the 16-bit rounding of
    # the kernel block (range finder) and of the basis (projection) does in the fast form
    assert np.mean(np.sign(dv) == np.sign(dv_o)) >= signs


@pytest.fixture(scope="module")
def flat_kernel_oracle():
    # d = 54 one-hot + uniform features at gamma = 0.02: every kernel entry lies in about
    # [0.75, 1], and C's eigenvalues span 18057 .. 0.052 (ratio 2.9e-6) at n = 20000, k = 400
    X, y, g, C, _ = synth.make("c3", n=20000)
    k = 400
    f, r, b = orc.train_rbf(X, y, g, C, k, rel_gap_tol=1e-6)
    fv = f.U @ (f.U.T @ (r.x * y)) + b
    return X, y, g, C, k, f.eigvals, r.log[-1][5], fv


# fp16 is held to the bar of the tensor-core form (objective 1e-5; measured 6.8e-6 with the
# one-launch wide kernel, eigenvalue 0.05160 against 0.05163); bf16 measured 5.5e-5
@pytest.mark.parametrize("prec,pobj_tol,eig_tol", [("fp16", 1e-5, 0.01), ("bf16", 1e-4, 0.05),
                                                   ("fp16_fast", 3e-4, 0.05),
                                                   ("bf16_fast", 5e-2, 0.7)])
def test_flat_kernel_tensor_core_against_fp64_oracle(ctx, flat_kernel_oracle, prec, pobj_tol,
                                                     eig_tol):
    # 16-bit rounding of entries near 1 would put noise of ~2 sigma sqrt(n) = 0.04 on the kernel,
    # the size of its weakest kept eigenvalue (measured before the mean shift: fp16 objective
    # 5.3e-2 off, smallest eigenvalue -0.001); with the sampled mean taken off every entry before
    # rounding, measured 6.6e-5 and 0.0509 (fp16), 1.5e-2 (bf16); the FP32 form 3.2e-4
    X, y, g, C, k, w, pobj_o, fv_o = flat_kernel_oracle
    Z, info = api.factor(ctx, dev(X), dev(y), g, k, prec)
    assert abs(info["eig_min"] - w.min()) <= eig_tol * w.min()
    yd = dev(y)
    a, _, _, st = api.ipm(ctx, Z, yd, k, C, rel_gap_tol=1e-6, precision=_lib.PREC_BF16)
    assert abs(st["pobj"] - pobj_o) <= pobj_tol * abs(pobj_o), (st["pobj"], pobj_o)
    b = api.bias(ctx, Z, yd, a, k, C)[0]
    Zk = Z[:, :k].double()
    fv = (Zk @ (Zk.T @ (a * yd.double())) + b).cpu().numpy()
    assert np.mean(np.sign(fv) == np.sign(fv_o)) >= 0.999
    if prec in ("fp16", "fp16_fast"):
        assert np.max(np.abs(fv - fv_o)) <= 2e-3 * np.max(np.abs(fv_o))


def _heldout_predictions(ctx, m, X, y, g, C):
    """Decision values of a trained model on the held-out points of synth "c2_test"."""
    sv, _ = orc.sv_sets(m.alpha, C)
    Xt, *_ = synth.make("c2_test")
    coef = dev(m.alpha[sv] * y[sv].astype(np.float64))
    return api.decision_values(ctx, _lib.KERNEL_RBF, dev(X[sv]), coef, -m.b, g,
                               dev(Xt)).cpu().numpy()


def test_full_size_two_gaussians_against_reference_run(ctx):
    """The benchmark workload itself (n = 1M, d = 18, k = 256, gamma 0.05, C 32, seed 2, 10%
    label noise) through the FP16 tensor-core form and the FP32 form, against the reference
    build's own run on the same file (tests/golden/ref_c2_1000000.log and .model.head): its last
    logged iterate pobj -2.481707792e7 / dobj -2.481707797e7 (T:1645), 785,145 SVs (19,396 free)
    and rho 0.060243 (T:384-396), and its model's decision values on 20,000 held-out points
    (tests/golden/ref_c2_1000000_heldout.npz, made by tests/golden/make_ref_heldout.py).  The
    reference file's first label is -1, which it maps to +1 (T:880-895): its labels are ours
    negated, the dual (alpha, objective) is the same and its b is ours negated, so its rho
    (= -b_ref) is our b and its f is -f here.
    The reference's run never met its 1e-7 residual rule (||rd|| = 2e-5 at the end) and stopped
    on max/min(D) > 1e18 at iteration 25; these runs are taken to the same end (tol 0), since the
    SV counts at alpha > 1e-6 and alpha < C - 1e-6 are those of the last interior iterate.
    The dual's optimal face is nearly flat (Q has rank k << n), so alpha and the decision values
    move with the factor's rounding: the reference's FP32 LRA is itself one such rounding.
    Measured on the 20,000 held-out points: the FP32 form agrees with the reference on 99.94 %
    of the predictions, the FP16 form on 99.855 %, and the two forms with each other on 99.845 %
    (decision values within 0.25 % of max |f|); max |d alpha| / C is ~1 between any two of them.
    Carrying the sketch as hi + lo in the range finder as well (a third product) does not close
    the gap (99.78 % with the reference, 99.79 % with the FP32 form): the spread is that of the
    problem under rounding of the factor at the 2^-22 level, not of one rounding in particular."""
    X, y, g, C, k = synth.make("c2")
    last = ref_log("ref_c2_1000000")[-1]
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_c2_1000000_heldout.npz"))
    f_ref = ref["f"]
    pred_ref = np.where(f_ref > 0, ref["labels"][0], ref["labels"][1])
    res = {}
    for prec in ("fp16", "fp32"):
        m = api.train(ctx, X, y, _lib.KERNEL_RBF, g, C, k, prec, tol=0.0)
        st = m.ipm_stats
        info = (prec, st["iters"], st["mu"], m.status)
        assert m.status == _lib.WARN_ILL_CONDITIONED, info
        assert abs(st["pobj"] - last[5]) / abs(last[5]) < 1e-5, (st["pobj"], last[5], info)
        assert abs(st["dobj"] - last[6]) / abs(last[6]) < 1e-5, (st["dobj"], last[6], info)
        sv, free = orc.sv_sets(m.alpha, C)
        f = _heldout_predictions(ctx, m, X, y, g, C)
        res[prec] = dict(f=f, nsv=len(sv), nfree=len(free), b=m.b, info=info,
                         agree=float(np.mean(np.where(f > 0, 1.0, -1.0) == pred_ref)),
                         dmax=float(np.max(np.abs(f + f_ref)) / np.max(np.abs(f_ref))))
    summary = {p: {q: v for q, v in r.items() if q != "f"} for p, r in res.items()}
    f16, f32 = res["fp16"]["f"], res["fp32"]["f"]
    assert np.mean(np.sign(f16) == np.sign(f32)) >= 0.998, summary
    assert np.max(np.abs(f16 - f32)) <= 5e-3 * np.max(np.abs(f32)), summary
    assert res["fp32"]["agree"] >= 0.999, summary
    assert res["fp16"]["agree"] >= 0.998, summary
    for prec in ("fp16", "fp32"):
        r = res[prec]
        assert r["dmax"] < 5e-3, summary
        assert abs(r["nsv"] - int(ref["total_sv"])) <= 1e-2 * int(ref["total_sv"]), summary
        # b is a mean over the first 50 free SVs, whose spread is 0.014 in the reference's run
        assert abs(r["b"] - float(ref["rho"])) < 0.01, summary
