"""Decision values (tsvm_decision_values / tsvm_predict), the FP64 Frobenius residual
(tsvm_kernel_residual, the reference's -analysis) and the two command-line tools on the GPU,
against FP64 numpy restatements."""
import re
import subprocess

import numpy as np
import pytest

from oracle import oracle as orc
from tensorsvm_b200 import _lib, api, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

PREDICT = _lib.CLI_PATH.replace("tensorsvm-train", "tensorsvm-predict")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def rbf_fp64(S, coef, rho, gamma, X):
    d2 = ((X.astype(np.float64)[:, None, :] - S.astype(np.float64)[None, :, :]) ** 2).sum(-1)
    K = np.exp(-gamma * d2)
    return K @ coef - rho, np.abs(K) @ np.abs(coef)


# d = 5, 18, 30, 54 take the register kernels (16, 24, 32, 64 features), 100 the chunked one
@pytest.mark.parametrize("d", [5, 18, 30, 54, 100])
def test_rbf_decision_values_match_fp64(ctx, d):
    rng = np.random.default_rng(d)
    nsv, m = 700, 1500
    S = rng.standard_normal((nsv, d)).astype(np.float32)
    X = rng.standard_normal((m, d)).astype(np.float32)
    coef = rng.uniform(-32, 32, nsv)
    gamma, rho = 0.5 / d, 0.375
    f = api.decision_values(ctx, _lib.KERNEL_RBF, dev(S), dev(coef), rho, gamma, dev(X))
    f_o, scale = rbf_fp64(S, coef, rho, gamma, X)
    # FP32 distances and exp, FP64 over tiles: each term within ~1e-6 relative
    assert np.all(np.abs(f.cpu().numpy() - f_o) <= 1e-5 * scale + 1e-12)


def test_linear_decision_values_and_empty_rows(ctx):
    rng = np.random.default_rng(3)
    w = rng.standard_normal(40).astype(np.float32)
    X = rng.standard_normal((999, 40)).astype(np.float32)
    f = api.decision_values(ctx, _lib.KERNEL_LINEAR, dev(w), None, -0.5, 0.0, dev(X))
    f_o = X.astype(np.float64) @ w.astype(np.float64) + 0.5
    assert np.max(np.abs(f.cpu().numpy() - f_o)) <= 1e-12 * np.max(np.abs(f_o)) * 40
    mf = api.ModelFile(kernel=_lib.KERNEL_LINEAR, pos=1, neg=-1, rho=-0.5, gamma=0.0, sv=w,
                       coef=np.zeros(0))
    assert api.predict(ctx, mf, X[:0]).shape == (0,)


def test_host_predict_pads_to_common_width(ctx):
    # SVs with fewer columns than the rows (the file omits trailing all-zero features)
    rng = np.random.default_rng(4)
    S = rng.standard_normal((300, 12)).astype(np.float32)
    X = rng.standard_normal((800, 18)).astype(np.float32)
    coef = rng.standard_normal(300)
    mf = api.ModelFile(kernel=_lib.KERNEL_RBF, pos=1, neg=-1, rho=0.1, gamma=0.05, sv=S, coef=coef)
    f = api.predict(ctx, mf, X)
    f_o, scale = rbf_fp64(np.pad(S, ((0, 0), (0, 6))), coef, 0.1, 0.05, X)
    assert np.all(np.abs(f - f_o) <= 1e-5 * scale + 1e-12)


@pytest.mark.parametrize("n,k", [(3000, 64), (1000, 50), (130, 7)])
def test_kernel_residual_matches_fp64(ctx, n, k):
    X, y, g, C, _ = synth.make("c1", n=n)
    Z, _ = api.factor(ctx, dev(X), dev(y), g, k, "fp32")
    fk, fr = api.kernel_residual(ctx, dev(X), dev(y), g, Z, k)
    Kt = orc.labelled_kernel(X, y, g)
    Zh = Z.cpu().numpy()[:, :k].astype(np.float64)
    fk_o = np.linalg.norm(Kt)
    fr_o = np.linalg.norm(Kt - Zh @ Zh.T)
    assert abs(fk - fk_o) <= 1e-11 * fk_o
    assert abs(fr - fr_o) <= 1e-9 * fk_o, (fr, fr_o)


def test_train_and_predict_cli(tmp_path):
    X, y, g, C, k = synth.make("c1")
    Xt, yt, *_ = synth.make("c1_test")
    train, test = tmp_path / "c1.train", tmp_path / "c1.test"
    synth.write_libsvm(str(train), X, y)
    synth.write_libsvm(str(test), Xt, yt)
    model, out = tmp_path / "c1.model", tmp_path / "c1.out"
    p = subprocess.run([_lib.CLI_PATH, "-k", str(k), "-c", str(C), "-g", str(g), "-t", "2",
                        "-analysis", "-test", str(test), str(train), str(model)],
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    mk = re.search(r"fnorm\(K\)=(\S+) fnorm\(K-U\*U=(\S+)'\)", p.stdout)
    assert mk, p.stdout
    yy, pos, neg = orc.remap_labels(y)
    fk_o = np.linalg.norm(orc.labelled_kernel(X, yy, g))
    assert abs(float(mk.group(1)) - fk_o) <= 1e-3 * fk_o        # printed with %.3e
    assert float(mk.group(2)) < 0.1 * fk_o
    acc = re.search(r"prediction accuracy (\S+) \((\d+)/(\d+)\)", p.stdout)
    # the FP64 oracle's model scores 0.572 on this split (Bayes rate 0.69; rank 32 underfits)
    f_m, r_m, b_m = orc.train_rbf(X, yy, g, C, k)
    acc_o = np.mean(np.sign(orc.decision_values_dense(r_m.x, yy, X, g, b_m, Xt)) == yt)
    assert acc and int(acc.group(3)) == len(yt)
    assert abs(int(acc.group(2)) / len(yt) - acc_o) <= 0.01, (acc.group(0), acc_o)
    p2 = subprocess.run([PREDICT, "-dec", str(test), str(model), str(out)], capture_output=True,
                        text=True, timeout=300)
    assert p2.returncode == 0, p2.stdout + p2.stderr
    rows = [ln.split() for ln in out.read_text().splitlines()]
    lab = np.array([int(r[0]) for r in rows])
    f = np.array([float(r[1]) for r in rows])
    m = orc.parse_model(model.read_text())
    f_o = orc.decision_values(m, Xt, X.shape[1])
    assert np.max(np.abs(f - f_o)) <= 1e-5 * np.sum(np.abs(m["coef"]))
    assert np.array_equal(lab[np.abs(f_o) > 1e-3], np.where(f_o > 0, pos, neg)[np.abs(f_o) > 1e-3])
    a2 = re.search(r"Accuracy = (\S+)% \((\d+)/(\d+)\)", p2.stdout)
    assert int(a2.group(2)) == int(np.sum(lab == yt.astype(int)))
    # the in-memory -test accuracy and the model-file accuracy agree to a few points near f = 0
    assert abs(int(a2.group(2)) - int(acc.group(2))) <= 0.01 * len(yt)
