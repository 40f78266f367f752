"""The FP64 hypergradient restatement (oracle.hypergrad) against central finite differences of
the FP64 pipeline it differentiates (range finder -> mpc -> bias -> validation loss), with the
bias' free-SV set held at the base point (the loss is only piecewise smooth across changes of
that set)."""
import numpy as np

from oracle import oracle as orc
from tensorsvm_b200 import synth


def test_oracle_hypergrad_matches_finite_differences():
    n, nv, k = 400, 150, 30
    X, y = synth.tanh_teacher(n, 28, seed=5)
    Xv, yv = synth.tanh_teacher(nv, 28, seed=55)
    X, Xv = X.astype(np.float64), Xv.astype(np.float64)
    y, yv = y.astype(np.float64), yv.astype(np.float64)
    Om = orc.polar_sketch(n, k)
    d2 = ((X[:, None, :] - X[None, :, :]) ** 2).sum(-1)
    d2tv = ((X[:, None, :] - Xv[None, :, :]) ** 2).sum(-1)

    def factor(g):
        Ky = y[:, None] * np.exp(-g * d2) * y[None, :]
        W, _ = np.linalg.qr(Ky @ Om)
        Cm = W.T @ Ky @ W
        w, V = np.linalg.eigh(0.5 * (Cm + Cm.T))
        return W @ (V * np.sqrt(np.maximum(w, 0.0)))

    def loss(lg, lc, F=None):
        g, C = np.exp(lg), np.exp(lc)
        Z = factor(g)
        r = orc.mpc(Z, y, C, tol=1e-10)
        if F is None:
            F = [i for i in range(n) if 1e-6 < r.x[i] < C - 1e-6][:50]
        b = np.mean([y[j] - y[j] * np.sum(r.x * (Z @ Z[j])) for j in F])
        f = np.exp(-g * d2tv).T @ (r.x * y) + b
        h = np.maximum(0.0, 1.0 - yv * f)
        return float(np.sum(h * h) / nv), r, b, F

    lg, lc = np.log(0.03), np.log(16.0)
    L0, r, b, F = loss(lg, lc)
    L, dg, dc, dxv = orc.hypergrad(X, y, Xv, yv, np.exp(lg), np.exp(lc), k, r.x, r.xi, r.s, b,
                                   Q=Om)
    assert abs(L - L0) <= 1e-12 * max(1.0, L0)
    h = 1e-4
    fd_c = (loss(lg, lc + h, F)[0] - loss(lg, lc - h, F)[0]) / (2 * h)
    fd_g = (loss(lg + h, lc, F)[0] - loss(lg - h, lc, F)[0]) / (2 * h)
    assert abs(dc - fd_c) <= 1e-2 * max(abs(fd_c), 1e-3 * L0), (dc, fd_c)
    assert abs(dg - fd_g) <= 1e-2 * max(abs(fd_g), 1e-3 * L0), (dg, fd_g)
    # dL/dXv: FD on one coordinate of one validation point (alpha, b do not depend on Xv)
    v, c = 3, 5
    e = np.zeros_like(Xv)
    e[v, c] = 1e-5

    def lv(Xv2):
        d2v = ((X[:, None, :] - Xv2[None, :, :]) ** 2).sum(-1)
        f = np.exp(-np.exp(lg) * d2v).T @ (r.x * y) + b
        hh = np.maximum(0.0, 1.0 - yv * f)
        return float(np.sum(hh * hh) / nv)

    fd_x = (lv(Xv + e) - lv(Xv - e)) / 2e-5
    assert abs(dxv[v, c] - fd_x) <= 1e-4 * max(abs(fd_x), 1e-6)
