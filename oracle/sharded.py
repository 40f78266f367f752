"""Row-sharded restatement of the oracle's LRA, mpc and bias (test infrastructure only).

Each rank holds a contiguous range of the rows of Z (and of X, y, alpha, s, xi) in rank order;
``allreduce(array, op)`` completes a sum ("sum") or minimum ("min") over the ranks in place.
The exchanges are exactly the ones the library's row-sharded path makes (tsvm_comm):

  mpc  (tensorsvm-train.cu:1507-1785): per iteration the sums behind mu, sum x, sum xi, a^T x,
       ||rd||^2 and x^T Q x, the min/max of D, the k-vectors Z^T v of every SMW solve
       (tensorsvm-train.cu:1832-1836) and of Q x (1616-1617), the capacitance matrix
       I + Z^T D^-1 Z (the reference's DSYRK, 1674-1697, summed once with the identity counted
       once), a^T r7 and a^T b, the step-length minima and mu_aff;
  LRA  (tensorsvm-train.cu:1941-2249): the CholeskyQR Gram matrices and C = W^T (K W), and the
       basis W gathered once (as a sum of zero-padded rows) for the projection pass;
  bias (tensorsvm-train.cu:355-376): the SV counts, v = sum alpha_i Z_i, and the first <= 50
       free SVs' terms of every rank, taken in rank order.

Every rank takes the same collective steps in the same order: the control flow depends only on
reduced values.  Nothing in the product imports this file; tests compare it with the
single-process oracle (oracle.py) on gloo ranks.
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as orc


def _sum(allreduce, v):
    a = np.atleast_1d(np.asarray(v, dtype=np.float64)).copy()
    allreduce(a, "sum")
    return a if np.ndim(v) else float(a[0])


def _min(allreduce, v):
    a = np.array([float(v)])
    allreduce(a, "min")
    return float(a[0])


def _smw_solve(Z, D, Lm, b, allreduce):
    """(D + Z Z^T)^-1 b on this rank's rows: the k-vector Z^T D^-1 b is all-reduced."""
    from scipy.linalg import cho_solve
    b = b / D
    bb = _sum(allreduce, Z.T @ b)
    bb = cho_solve((Lm, True), bb)
    return b - (Z @ bb) / D


def _newton_step(Z, D, Lm, C, a, x, s, xi, rd, rp, rs, rxi, allreduce):
    r5 = rd - rs / x + rxi / (C - x)
    r7 = _smw_solve(Z, D, Lm, r5, allreduce)
    r6 = rp + _sum(allreduce, a @ r7)
    b = _smw_solve(Z, D, Lm, a, allreduce)
    dy = r6 / _sum(allreduce, a @ b)
    dx = _smw_solve(Z, D, Lm, a * dy - r5, allreduce)
    ds = (rs - s * dx) / x
    dxi = (rxi + xi * dx) / (C - x)
    return dx, dy, ds, dxi


def _ratio(x, s, xi, dx, ds, dxi, C, allreduce):
    """The step-length ratio test of tensorsvm-train.cu:1733-1739, minimum over the ranks."""
    alpha = 1.0
    m = dx < 0
    if m.any():
        alpha = min(alpha, float(np.min(-x[m] / dx[m])))
    m = dx > 0
    if m.any():
        alpha = min(alpha, float(np.min((C - x[m]) / dx[m])))
    m = ds < 0
    if m.any():
        alpha = min(alpha, float(np.min(-s[m] / ds[m])))
    m = dxi < 0
    if m.any():
        alpha = min(alpha, float(np.min(-xi[m] / dxi[m])))
    return _min(allreduce, alpha)


def mpc(Z, a, C, allreduce, kernel: str = "rbf", max_iter: int = orc.MAX_MPC_ITER,
        tol: float = 1e-7, rel_gap_tol: float | None = None) -> orc.MpcResult:
    """oracle.mpc on this rank's rows (Z: n_local x k, a: n_local labels)."""
    from scipy.linalg import cholesky
    Z = np.asarray(Z, dtype=np.float64)
    a = np.asarray(a, dtype=np.float64)
    n_loc, k = Z.shape
    n = _sum(allreduce, float(n_loc))
    y = 0.0
    e = np.ones(n_loc)
    if kernel == "rbf":
        q = _sum(allreduce, Z.T @ e)
        e2 = Z @ q
        s2 = _sum(allreduce, np.array([e2.sum(), e2 @ e2]))
        ox = s2[0] / s2[1]
    else:
        ox = 1.0
    if 0.01 * C < ox < 0.99 * C:
        x = np.full(n_loc, ox)
    elif ox > 0.99 * C:
        x = np.full(n_loc, 0.99 * C)
    else:
        x = np.full(n_loc, 0.01 * C)
    s = np.ones(n_loc)
    xi = np.ones(n_loc)
    if kernel != "rbf":
        t = Z @ _sum(allreduce, Z.T @ x) - a * y - 1.0
        s = s + np.where(t > 0, t, 0.0)
        xi = xi - np.where(t > 0, 0.0, t)
    log = []
    status = "max_iter"
    it = 0
    for it in range(max_iter):
        Qx = Z @ _sum(allreduce, Z.T @ x)
        rd = Qx - a * y - s + xi - 1.0
        D = s / x + xi / (C - x)
        sums = _sum(allreduce, np.array([np.sum(x * s + (C - x) * xi), a @ x, rd @ rd, x @ Qx,
                                         x.sum(), xi.sum()]))
        mu = sums[0] / (2 * n)
        rp = -sums[1]
        rs = -s * x
        rxi = -xi * (C - x)
        dmin = _min(allreduce, D.min())
        dmax = -_min(allreduce, -D.max())
        cond = dmax / dmin
        normdx = math.sqrt(sums[2])
        normdy = abs(rp)
        tmp = 0.5 * sums[3]
        pobj = tmp - sums[4]
        dobj = -tmp - C * sums[5]
        log.append((it, mu, normdx, normdy, cond, pobj, dobj))
        if mu < tol and normdx < tol and normdy < tol:
            status = "converged"
            break
        if rel_gap_tol is not None:
            rel_gap = (pobj - dobj) / max(1.0, abs(pobj))
            scale = 1.0 + math.sqrt(n)
            if rel_gap <= rel_gap_tol and normdx / scale <= rel_gap_tol \
                    and normdy / scale <= rel_gap_tol:
                status = "converged"
                break
        if cond > 1e18:
            status = "ill_conditioned"
            break
        Zs = Z / np.sqrt(D)[:, None]
        M = Zs.T @ Zs + np.eye(k)          # this rank's rows plus I ...
        M = _sum(allreduce, M) - (_sum(allreduce, 1.0) - 1.0) * np.eye(k)   # ... I counted once
        try:
            Lm = cholesky(M, lower=True)
        except np.linalg.LinAlgError:
            status = "not_spd"
            break
        dx_a, dy_a, ds_a, dxi_a = _newton_step(Z, D, Lm, C, a, x, s, xi, rd, rp, rs, rxi,
                                               allreduce)
        alpha = _ratio(x, s, xi, dx_a, ds_a, dxi_a, C, allreduce)
        mu_aff = _sum(allreduce, np.sum((x + alpha * dx_a) * (s + alpha * ds_a)
                                        + (C - x - alpha * dx_a) * (xi + alpha * dxi_a))) / (2 * n)
        sigma = (mu_aff / mu) ** 3
        rs_c = sigma * mu - dx_a * ds_a
        rxi_c = sigma * mu + dx_a * dxi_a
        dx_c, dy_c, ds_c, dxi_c = _newton_step(Z, D, Lm, C, a, x, s, xi, np.zeros(n_loc), 0.0,
                                               rs_c, rxi_c, allreduce)
        dx = dx_c + dx_a
        dy = dy_c + dy_a
        ds = ds_c + ds_a
        dxi = dxi_c + dxi_a
        alpha = 0.99 * _ratio(x, s, xi, dx, ds, dxi, C, allreduce)
        x = x + alpha * dx
        s = s + alpha * ds
        xi = xi + alpha * dxi
        y = y + alpha * dy
    return orc.MpcResult(x=x, xi=xi, s=s, y=y, iters=it, status=status, log=log)


def lra(X, y, gamma, k, row0, nr, allreduce, c_as_float32: bool = False) -> orc.LraResult:
    """oracle.lra's factor rows [row0, row0 + nr) (X, y: the whole training set on every rank).

    The whole sketch is drawn on every rank; the range basis is orthonormalised by CholeskyQR2
    with all-reduced Gram matrices (only range(W) enters Z Z^T, so any orthonormal basis of it
    gives oracle.lra's factor)."""
    n = X.shape[0]
    Q = orc.polar_sketch(n, k).astype(np.float64)
    rows = slice(row0, row0 + nr)

    def kermatmul_rows(A):
        W = np.zeros((nr, A.shape[1]))
        for j in range(0, n, 2048):
            jb = slice(j, min(n, j + 2048))
            W += orc.rbf_block(X[rows], X[jb], y[rows], y[jb], gamma) @ A[jb]
        return W

    W = kermatmul_rows(Q)
    for _ in range(2):
        G = _sum(allreduce, W.T @ W)
        L = np.linalg.cholesky(G)
        W = np.linalg.solve(L, W.T).T
    Wall = np.zeros((n, k))
    Wall[rows] = W
    allreduce(Wall, "sum")
    Q2 = kermatmul_rows(Wall)
    C = _sum(allreduce, W.T @ Q2)
    if c_as_float32:
        C32 = C.astype(np.float32)
        C = ((C32 + C32.T).astype(np.float32) * np.float32(0.5)).astype(np.float64)
    else:
        C = 0.5 * (C + C.T)
    w, V = np.linalg.eigh(C, UPLO="L")
    s = np.where(w > 0, np.sqrt(np.maximum(w, 0.0)), 0.0)
    return orc.LraResult(U=W @ (V * s[None, :]), eigvals=w, realk=int((w > 0).sum()), W=W, C=C)


def bias_rbf(U, labels, alpha, C, rank, world, allreduce):
    """oracle.bias_rbf on this rank's rows: every rank contributes its first <= 50 free SVs'
    terms; the first 50 over the ranks in rank order (= global index order) are averaged."""
    sv, free = orc.sv_sets(alpha, C)
    U = np.asarray(U, np.float64)
    labels = np.asarray(labels, np.float64)
    v = _sum(allreduce, alpha[sv] @ U[sv])
    m = min(len(free), 50)
    terms = np.zeros((world, 51))
    terms[rank, 0] = m
    for t in range(m):
        j = free[t]
        terms[rank, 1 + t] = labels[j] - labels[j] * float(v @ U[j])
    allreduce(terms, "sum")
    take = []
    for r in range(world):
        take.extend(terms[r, 1:1 + int(terms[r, 0])])
    take = np.array(take[:50])
    counts = _sum(allreduce, np.array([len(sv), len(free)], dtype=np.float64))
    if len(take) == 0:
        return float("nan"), float("nan"), counts
    b = take.mean()
    return float(b), float(np.sqrt(np.mean((take - b) ** 2))), counts
