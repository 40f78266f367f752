"""The CPU oracle, pinned against the reference trainer's own outputs (tests/golden/, produced by
tests/golden/make_ref_goldens.sh running the compiled reference on a B200) and against
known-answer problems.  No GPU needed."""
import ctypes
import ctypes.util
import os

import numpy as np
import pytest

from conftest import GOLDEN, jaccard, ref_fixture, ref_log
from oracle import oracle as orc
from tensorsvm_b200 import synth


def test_glibc_generator_restatement_matches_libc():
    # the recurrence the GPU sketch kernel jumps ahead on == glibc rand() (tensorsvm-train.cu:2629)
    a = orc.glibc_rand(20000)
    b = orc.glibc_rand_restated(20000)
    assert np.array_equal(a, b)


def test_polar_sketch_follows_gaussrand_float_arithmetic():
    # independent restatement of tensorsvm-train.cu:2621-2643 with numpy float32 ops + libm logf
    libm = ctypes.CDLL(ctypes.util.find_library("m"))
    libm.logf.restype = ctypes.c_float
    libm.logf.argtypes = [ctypes.c_float]
    r = orc.glibc_rand(4000)
    out, j = [], 0
    while len(out) < 1000:
        u1 = np.float32(r[j]) / np.float32(2147483647)
        u2 = np.float32(r[j + 1]) / np.float32(2147483647)
        j += 2
        v1 = np.float32(2) * u1 - np.float32(1)
        v2 = np.float32(2) * u2 - np.float32(1)
        s = v1 * v1 + v2 * v2
        if s >= 1 or s == 0:
            continue
        f = np.sqrt(np.float32(-2) * np.float32(libm.logf(s)) / s, dtype=np.float32)
        out += [v1 * f, v2 * f]
    q = orc.polar_sketch(1, 1000).ravel()
    assert np.array_equal(q, np.asarray(out[:1000], dtype=np.float32))


def test_synthetic_data_is_deterministic():
    X, y, *_ = synth.make("c1")
    assert X.shape == (8192, 18) and set(np.unique(y)) == {-1.0, 1.0}
    assert abs(float(y.sum())) == 0.0  # balanced
    X2, y2, *_ = synth.make("c1")
    assert np.array_equal(X, X2) and np.array_equal(y, y2)


@pytest.fixture(scope="module")
def c1_oracle():
    X, y, g, C, k = synth.make("c1")
    yy, pos, neg = orc.remap_labels(y)
    f, r, b = orc.train_rbf(X, yy, g, C, k)
    return X, yy, g, C, k, f, r, b


def test_oracle_rbf_matches_reference_objective(c1_oracle):
    X, y, g, C, k, f, r, b = c1_oracle
    last = ref_log("ref_c1_rbf")[-1]
    assert int(last[0]) == r.iters                       # both stop at iteration 17
    assert abs(r.log[-1][5] - last[5]) / abs(last[5]) < 1e-5   # pobj
    assert abs(r.log[-1][6] - last[6]) / abs(last[6]) < 1e-5   # dobj


def test_oracle_rbf_matches_reference_model(c1_oracle):
    X, y, g, C, k, f, r, b = c1_oracle
    idx, coef, rho, hdr = ref_fixture("ref_c1_rbf")
    sv, free = orc.sv_sets(r.x, C)
    # SV membership flips only for alphas within rounding of the 1e-6 threshold
    assert jaccard(sv, idx) > 0.99
    ref_alpha = np.zeros(len(X))
    ref_alpha[idx] = coef * y[idx]
    Xt = synth.make("c1_test")[0]
    dv_o = orc.decision_values_dense(r.x, y, X, g, b, Xt)
    dv_r = orc.decision_values_dense(ref_alpha, y, X, g, -rho, Xt)
    assert np.mean(np.sign(dv_o) == np.sign(dv_r)) >= 0.999
    assert abs(b - (-rho)) < 1e-3
    assert "label 1 -1" in hdr and "gamma 0.0100000" in hdr


def test_oracle_rbf_matches_reference_larger():
    X, y = synth.two_gaussians(32768, 18, seed=7, noise=0.10)
    yy, pos, neg = orc.remap_labels(y)
    f, r, b = orc.train_rbf(X, yy, 0.05, 32.0, 64)
    last = ref_log("ref_m32k_rbf")[-1]
    assert abs(r.log[-1][5] - last[5]) / abs(last[5]) < 1e-5
    idx, coef, rho, _ = ref_fixture("ref_m32k_rbf")
    sv, _ = orc.sv_sets(r.x, 32.0)
    assert jaccard(sv, idx) > 0.998
    assert abs(b - (-rho)) < 1e-3


def test_oracle_linear_matches_reference():
    X, y, *_ = synth.make("c1")
    r, w, b = orc.train_linear(X, y, 1.0)
    lines = open(os.path.join(GOLDEN, "ref_c1_lin.model")).read().split("\n")
    i = lines.index("w")
    ref_w = np.array([float(v) for v in lines[i + 1:i + 19]])
    ref_b = float(lines[i + 19])
    assert np.max(np.abs(w - ref_w)) < 1e-8
    assert abs(b - ref_b) < 1e-8
    assert int(ref_log("ref_c1_lin")[-1][0]) == r.iters == 30


def test_mpc_two_point_known_answer():
    # x+ = (1, 0), x- = (-1, 0): hard-margin solution alpha = 2/||x+ - x-||^2 = 0.5 each, b = 0
    X = np.array([[1.0, 0.0], [-1.0, 0.0]])
    y = np.array([1.0, -1.0])
    r = orc.mpc(X * y[:, None], y, 10.0, kernel="linear", tol=1e-10)
    assert r.status == "converged" or r.status == "ill_conditioned"
    assert np.allclose(r.x, [0.5, 0.5], atol=1e-6)
    w, b = orc.linear_w_b(X, y, r.x, 10.0)
    assert np.allclose(w, [1.0, 0.0], atol=1e-6) and abs(b) < 1e-6


def test_mpc_four_point_known_answer():
    # x = +-1 and +-2 on a line, labels by sign: the hard-margin support vectors are +-1 with
    # alpha = 2/||x+ - x-||^2 = 0.5, the outer points carry alpha = 0; w = (1, 0), b = 0
    X = np.array([[1.0, 0.0], [-1.0, 0.0], [2.0, 0.0], [-2.0, 0.0]])
    y = np.array([1.0, -1.0, 1.0, -1.0])
    r = orc.mpc(X * y[:, None], y, 10.0, kernel="linear", tol=1e-10)
    assert r.status in ("converged", "ill_conditioned")
    assert np.allclose(r.x, [0.5, 0.5, 0.0, 0.0], atol=1e-6)
    w, b = orc.linear_w_b(X, y, r.x, 10.0)
    assert np.allclose(w, [1.0, 0.0], atol=1e-6) and abs(b) < 1e-6


def test_rbf_full_rank_matches_sklearn_exact_kernel():
    # k = n: the factor reproduces the labelled kernel, so the dual is the exact-kernel SVM's;
    # sklearn's SVC (libsvm SMO) is an independent solver of it
    from sklearn.svm import SVC
    X, y = synth.two_gaussians(160, 4, seed=11)
    g, C = 0.3, 2.0
    f = orc.lra(X, y, g, 160)
    r = orc.mpc(f.U, y, C, tol=1e-10)
    K = orc.labelled_kernel(X, y, g)
    m = SVC(kernel="rbf", gamma=g, C=C, tol=1e-12).fit(X.astype(np.float64), y)
    a = np.zeros(len(y))
    a[m.support_] = np.abs(m.dual_coef_.ravel())
    obj = lambda al: 0.5 * al @ K @ al - al.sum()
    assert abs(obj(r.x) - obj(a)) / abs(obj(a)) < 1e-7   # measured 3.8e-9
    assert jaccard(set(np.where(r.x > 1e-6 * C)[0]), set(m.support_)) > 0.98   # measured 0.991


def test_mpc_linear_matches_sklearn_objective():
    from sklearn.svm import SVC
    X, y = synth.two_gaussians(400, 5, seed=3)
    C = 2.0
    r = orc.mpc(X.astype(np.float64) * y[:, None], y, C, kernel="linear", tol=1e-9)
    m = SVC(kernel="linear", C=C, tol=1e-10).fit(X, y)
    a = np.zeros(len(y))
    a[m.support_] = np.abs(m.dual_coef_.ravel())
    Z = X.astype(np.float64) * y[:, None]
    obj = lambda al: 0.5 * np.sum((Z.T @ al) ** 2) - al.sum()
    assert abs(obj(r.x) - obj(a)) / abs(obj(a)) < 1e-6


def test_lra_full_rank_reproduces_kernel():
    X, y = synth.two_gaussians(96, 4, seed=9)
    f = orc.lra(X, y, 0.3, 96)
    K = orc.labelled_kernel(X, y, 0.3)
    assert np.linalg.norm(f.U @ f.U.T - K) / np.linalg.norm(K) < 1e-5


def test_philox_restatement_known_answers():
    """The oracle's Philox4x32-10 against the generator's published known-answer vectors
    (counter, key) -> output words."""
    kat = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
           ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
           ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
            (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for ctr, key, want in kat:
        got = orc.philox4x32_10([np.array([v], np.uint64) for v in ctr], key)[:, 0]
        assert tuple(int(v) for v in got) == want


def test_philox_sketch_moments_and_seeds():
    z = orc.philox_sketch(7, 1_000_003)
    assert abs(z.mean()) < 5e-3 and abs(z.var() - 1.0) < 5e-3
    assert abs(np.mean(z ** 4) - 3.0) < 3e-2                 # Gaussian kurtosis
    assert np.array_equal(z[:1000], orc.philox_sketch(7, 1000))
    assert not np.allclose(z[:1000], orc.philox_sketch(8, 1000))
