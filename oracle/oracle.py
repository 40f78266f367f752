"""FP64 CPU oracle for the TensorSVM training path.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this module,
and only as the checker (or the timed CPU baseline), never as the product path.

It restates, in FP64 with host BLAS/LAPACK (numpy/scipy over OpenBLAS), the reference
trainer robbwu/tensorsvm ``tensorsvm-train.cu``:

* ``polar_sketch``          gaussrand + Q fill          tensorsvm-train.cu:2621-2643, 1966-1974
* ``rbf_block``             vecnorm + XIJ + rbf_kergen  tensorsvm-train.cu:2569-2581, 2506-2530, 2598-2612
* ``kermatmul``             RBF_KERMATMUL / rbf_kermatmul  tensorsvm-train.cu:1999-2063, 2476-2567
* ``lra``                   LRA                         tensorsvm-train.cu:1941-2249
* ``mpc``                   Mehrotra predictor-corrector tensorsvm-train.cu:1507-1785
* ``newton_step``           NewtonStep                  tensorsvm-train.cu:1794-1822
* ``smw_solve``             SMWSolve                    tensorsvm-train.cu:1824-1840
* ``bias_rbf`` / ``bias_linear`` / ``write_model``  writemodel  tensorsvm-train.cu:273-417
* ``read_libsvm``           libsvmread                  tensorsvm-train.cu:1162-1278
* ``remap_labels``          label remap in main         tensorsvm-train.cu:879-896

Pinning: the sketch is bit-exact against glibc (it *is* glibc rand()+logf); the end-to-end
result is pinned against the reference binary's own model files on config-1-shaped data
(tests/golden/, produced by tests/golden/make_ref_goldens.sh on a B200).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")
_SKETCH_SO = os.path.join(_BUILD, "liboracle_sketch.so")


def build(force: bool = False) -> str:
    """Compile oracle/sketch.c (gcc, no FMA contraction) into oracle/_build/."""
    os.makedirs(_BUILD, exist_ok=True)
    src = os.path.join(_HERE, "sketch.c")
    if force or not os.path.exists(_SKETCH_SO) or os.path.getmtime(_SKETCH_SO) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off",
                               src, "-o", _SKETCH_SO, "-lm"])
    return _SKETCH_SO


_sketch_lib = None


def _lib():
    global _sketch_lib
    if _sketch_lib is None:
        _sketch_lib = ctypes.CDLL(build())
        _sketch_lib.oracle_polar_sketch.restype = ctypes.c_long
        _sketch_lib.oracle_polar_sketch.argtypes = [ctypes.c_void_p, ctypes.c_long]
        _sketch_lib.oracle_rand_stream.restype = None
        _sketch_lib.oracle_rand_stream.argtypes = [ctypes.c_void_p, ctypes.c_long]
    return _sketch_lib


def polar_sketch(n: int, k: int) -> np.ndarray:
    """Q (n x k, float32, row-major): the reference's gaussrand() stream.

    tensorsvm-train.cu:1967-1973 fills Q[i*k+j] = gaussrand() for i then j."""
    out = np.empty(n * k, dtype=np.float32)
    _lib().oracle_polar_sketch(out.ctypes.data, out.size)
    return out.reshape(n, k)


def philox4x32_10(ctr, key):
    """Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC 2011) on vectors of counters: ctr is a
    (4, m) uint32 array, key a (2,) pair.  Restated from the paper's round function: two 32x32
    multiplications per round with the multipliers 0xD2511F53 and 0xCD9E8D57, Weyl key bumps
    0x9E3779B9 and 0xBB67AE85, ten rounds."""
    c = [np.asarray(v, dtype=np.uint64) for v in ctr]
    k0, k1 = np.uint64(key[0]), np.uint64(key[1])
    mask = np.uint64(0xFFFFFFFF)
    for _ in range(10):
        p0 = np.uint64(0xD2511F53) * c[0]
        p1 = np.uint64(0xCD9E8D57) * c[2]
        c = [(p1 >> np.uint64(32)) ^ c[1] ^ k0, p1 & mask, (p0 >> np.uint64(32)) ^ c[3] ^ k1,
             p0 & mask]
        k0 = (k0 + np.uint64(0x9E3779B9)) & mask
        k1 = (k1 + np.uint64(0xBB67AE85)) & mask
    return np.stack([v.astype(np.uint32) for v in c])


def philox_sketch(seed: int, count: int) -> np.ndarray:
    """The TSVM_SKETCH_PHILOX stream in FP64: block b = e // 4 of entry e is Philox4x32-10 of
    counter (b, 0, 0, 0) under key (seed low, seed high); words (w0, w1) and (w2, w3) give
    Box-Muller pairs r cos(2 pi u1), r sin(2 pi u1), r = sqrt(-2 ln u0), u = ((w >> 8) + 1/2) 2^-24."""
    blocks = (count + 3) // 4
    b = np.arange(blocks, dtype=np.uint64)
    ctr = [b & np.uint64(0xFFFFFFFF), b >> np.uint64(32), np.zeros_like(b), np.zeros_like(b)]
    w = philox4x32_10(ctr, (seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF))
    u = ((w >> np.uint32(8)).astype(np.float64) + 0.5) / 16777216.0
    out = np.empty((blocks, 4))
    for p in range(2):
        r = np.sqrt(-2.0 * np.log(u[2 * p]))
        out[:, 2 * p] = r * np.cos(2 * np.pi * u[2 * p + 1])
        out[:, 2 * p + 1] = r * np.sin(2 * np.pi * u[2 * p + 1])
    return out.ravel()[:count]


def glibc_rand(count: int) -> np.ndarray:
    """The glibc rand() stream from the default seed (1)."""
    out = np.empty(count, dtype=np.uint32)
    _lib().oracle_rand_stream(out.ctypes.data, count)
    return out


def glibc_rand_restated(count: int) -> np.ndarray:
    """Pure-numpy restatement of glibc's TYPE_3 additive generator (degree 31, separation 3).

    r[0]=seed; r[i] = 16807*r[i-1] mod (2^31-1) for i<31 (Schrage form, signed);
    r[i] = r[i-31] for 31<=i<34; r[i] = r[i-31] + r[i-3] mod 2^32 afterwards;
    output m is r[m+344] >> 1.  This is the recurrence the GPU sketch kernel jumps ahead on."""
    total = count + 344
    r = np.zeros(max(total, 34), dtype=np.int64)
    r[0] = 1
    for i in range(1, 31):
        hi, lo = divmod(int(r[i - 1]), 127773)
        word = 16807 * lo - 2836 * hi
        if word < 0:
            word += 2147483647
        r[i] = word
    for i in range(31, 34):
        r[i] = r[i - 31]
    ru = (r & 0xFFFFFFFF).astype(np.uint64)
    for i in range(34, total):
        ru[i] = (ru[i - 31] + ru[i - 3]) & 0xFFFFFFFF
    return (ru[344:344 + count] >> np.uint64(1)).astype(np.uint32)


# ----------------------------------------------------------------------------------------
# LIBSVM input (tensorsvm-train.cu:1162-1278) and label remap (tensorsvm-train.cu:879-896)
# ----------------------------------------------------------------------------------------

def read_libsvm(path: str, scale256: bool = False):
    """Dense row-major float32 instances and float32 labels, indices shifted by min_index."""
    labels, rows = [], []
    max_index, min_index = 0, 1
    with open(path) as f:
        for line in f:
            toks = line.split()
            if not toks:
                continue
            labels.append(float(toks[0]))
            feats = []
            for t in toks[1:]:
                idx, val = t.split(":")
                idx = int(idx)
                feats.append((idx, float(val)))
                min_index = min(min_index, idx)
                max_index = max(max_index, idx)
            rows.append(feats)
    nf = max_index - min_index + 1 if min_index == 0 else max_index
    X = np.zeros((len(rows), nf), dtype=np.float32)
    for i, feats in enumerate(rows):
        for idx, val in feats:
            X[i, idx - min_index] = np.float32(val) / np.float32(256) if scale256 else np.float32(val)
    return np.asarray(labels, dtype=np.float32), X


def remap_labels(labels: np.ndarray):
    """POS = first label, NEG = first different label; map to +1/-1 (tensorsvm-train.cu:880-895)."""
    pos = int(labels[0])
    neg = None
    for v in labels:
        if int(v) != pos:
            neg = int(v)
            break
    if neg is None:
        raise ValueError("training data has a single class")
    y = np.where(labels.astype(np.int64) == pos, 1.0, -1.0).astype(np.float32)
    bad = (labels.astype(np.int64) != pos) & (labels.astype(np.int64) != neg)
    if bad.any():
        raise ValueError("more than two classes in training data")
    return y, pos, neg


# ----------------------------------------------------------------------------------------
# Kernel factor (LRA)
# ----------------------------------------------------------------------------------------

def rbf_block(Xi, Xj, yi, yj, gamma):
    """y_i y_j exp(-gamma (||x_i||^2 + ||x_j||^2 - 2 x_i.x_j)) in FP64 (tensorsvm-train.cu:2608)."""
    Xi = np.asarray(Xi, dtype=np.float64)
    Xj = np.asarray(Xj, dtype=np.float64)
    ni = np.einsum("ij,ij->i", Xi, Xi)
    nj = np.einsum("ij,ij->i", Xj, Xj)
    d2 = ni[:, None] + nj[None, :] - 2.0 * (Xi @ Xj.T)
    return (np.asarray(yi, np.float64)[:, None] * np.asarray(yj, np.float64)[None, :]) * np.exp(-gamma * d2)


def kermatmul(X, y, gamma, A, block: int = 2048, threads: int = 1):
    """W = (Y K Y) A, K the RBF kernel of X (tensorsvm-train.cu:1999-2063 with 2476-2567).

    threads > 1 spreads the row blocks over host threads (numpy's exp and single-threaded BLAS
    inside each worker); every row block is still summed over the column blocks in order."""
    n = X.shape[0]
    A = np.asarray(A, dtype=np.float64)
    W = np.zeros((n, A.shape[1]), dtype=np.float64)

    def row_block(i):
        ib = slice(i, min(n, i + block))
        for j in range(0, n, block):
            jb = slice(j, min(n, j + block))
            W[ib] += rbf_block(X[ib], X[jb], y[ib], y[jb], gamma) @ A[jb]

    if threads <= 1:
        for i in range(0, n, block):
            row_block(i)
        return W
    from concurrent.futures import ThreadPoolExecutor
    from threadpoolctl import threadpool_limits
    with threadpool_limits(limits=1, user_api="blas"), ThreadPoolExecutor(threads) as ex:
        list(ex.map(row_block, range(0, n, block)))
    return W


def labelled_kernel(X, y, gamma):
    return rbf_block(X, X, y, y, gamma)


@dataclass
class LraResult:
    U: np.ndarray            # n x k labelled factor, U U^T ~= Y K Y
    eigvals: np.ndarray      # eigenvalues of C (ascending, like dsyevd)
    realk: int               # number of positive eigenvalues kept (tensorsvm-train.cu:2197-2211)
    W: np.ndarray = field(repr=False, default=None)
    C: np.ndarray = field(repr=False, default=None)


def lra(X, y, gamma, k, Q=None, c_as_float32: bool = True, threads: int = 1) -> LraResult:
    """Randomised range-finder factor of Y K Y (tensorsvm-train.cu:1941-2249), FP64.

    Steps: Q = sketch; W = K~ Q; W = orth(W); Q = K~ W; C = W^T Q (stored as float,
    tensorsvm-train.cu:1990, lower triangle averaged 2152-2156); C = V diag(w) V^T (dsyevd,
    lower); X = V diag(sqrt(max(w,0))); U = W X."""
    n = X.shape[0]
    if Q is None:
        Q = polar_sketch(n, k)
    W = kermatmul(X, y, gamma, Q, threads=threads)
    W, _ = np.linalg.qr(W)                       # any exact QR: only range(W) matters
    Q2 = kermatmul(X, y, gamma, W, threads=threads)
    C = W.T @ Q2
    if c_as_float32:
        C32 = C.astype(np.float32)
        C = ((C32 + C32.T).astype(np.float32) * np.float32(0.5)).astype(np.float64)
    else:
        C = 0.5 * (C + C.T)      # dsyevd('L') sees the averaged lower triangle
    w, V = np.linalg.eigh(C, UPLO="L")
    s = np.where(w > 0, np.sqrt(np.maximum(w, 0.0)), 0.0)
    realk = int((w > 0).sum())
    U = W @ (V * s[None, :])
    return LraResult(U=U, eigvals=w, realk=realk, W=W, C=C)


# ----------------------------------------------------------------------------------------
# Interior-point solver (tensorsvm-train.cu:1507-1840)
# ----------------------------------------------------------------------------------------

MAX_MPC_ITER = 100   # tensorsvm-train.cu:62


@dataclass
class MpcResult:
    x: np.ndarray
    xi: np.ndarray
    s: np.ndarray
    y: float
    iters: int
    status: str                       # "converged" | "ill_conditioned" | "not_spd" | "max_iter"
    log: list = field(default_factory=list)   # per iteration (iter, mu, normdx, normdy, cond, pobj, dobj)


def smw_solve(Z, D, Lm, b):
    """(D + Z Z^T)^{-1} b through M = I + Z^T D^{-1} Z = L L^T (tensorsvm-train.cu:1824-1840)."""
    from scipy.linalg import cho_solve
    b = b / D
    c = b.copy()
    bb = Z.T @ b
    bb = cho_solve((Lm, True), bb)
    return c - (Z @ bb) / D


def newton_step(Z, D, Lm, C, a, x, s, xi, rd, rp, rs, rxi):
    """Block elimination of the reduced KKT system (tensorsvm-train.cu:1794-1822).

    Returns (dx, dy, ds, dxi).  Three SMW solves, as in the reference."""
    r5 = rd - rs / x + rxi / (C - x)
    r7 = smw_solve(Z, D, Lm, r5)
    r6 = rp + a @ r7
    b = smw_solve(Z, D, Lm, a)
    dy = r6 / (a @ b)
    dx = smw_solve(Z, D, Lm, a * dy - r5)
    ds = (rs - s * dx) / x
    dxi = (rxi + xi * dx) / (C - x)
    return dx, dy, ds, dxi


def _ratio(x, s, xi, dx, ds, dxi, C):
    """Largest step in [0,1] keeping 0<=x<=C, s>=0, xi>=0 (tensorsvm-train.cu:1733-1739)."""
    alpha = 1.0
    neg = dx < 0
    if neg.any():
        alpha = min(alpha, float(np.min(-x[neg] / dx[neg])))
    pos = dx > 0
    if pos.any():
        alpha = min(alpha, float(np.min((C - x[pos]) / dx[pos])))
    m = ds < 0
    if m.any():
        alpha = min(alpha, float(np.min(-s[m] / ds[m])))
    m = dxi < 0
    if m.any():
        alpha = min(alpha, float(np.min(-xi[m] / dxi[m])))
    return alpha


def mpc(Z, a, C, kernel: str = "rbf", max_iter: int = MAX_MPC_ITER, tol: float = 1e-7,
        rel_gap_tol: float | None = None):
    """Mehrotra predictor-corrector on the SVM dual with Q = Z Z^T (tensorsvm-train.cu:1507-1785).

    ``kernel`` selects the reference's initialisation (RBF T:1535-1552, linear T:1553-1579).
    ``rel_gap_tol`` (not in the reference) adds a stop on rel_gap = (pobj-dobj)/max(1,|pobj|)
    together with ||rd||/(1+sqrt n) and |rp|/(1+sqrt n) below the same tolerance."""
    from scipy.linalg import cholesky
    Z = np.asarray(Z, dtype=np.float64)
    a = np.asarray(a, dtype=np.float64)
    n, k = Z.shape
    y = 0.0
    e = np.ones(n)
    if kernel == "rbf":
        q = Z.T @ e
        e2 = Z @ q
        ox = e2.sum() / (np.linalg.norm(e2) ** 2)
    else:
        ox = e.sum() / (np.linalg.norm(e) ** 2)
    if 0.01 * C < ox < 0.99 * C:
        x = np.full(n, ox)
    elif ox > 0.99 * C:
        x = np.full(n, 0.99 * C)
    else:
        x = np.full(n, 0.01 * C)
    s = np.ones(n)
    xi = np.ones(n)
    if kernel != "rbf":
        t = Z @ (Z.T @ x) - a * y - 1.0
        s = s + np.where(t > 0, t, 0.0)
        xi = xi - np.where(t > 0, 0.0, t)
    log = []
    status = "max_iter"
    it = 0
    for it in range(max_iter):
        mu = float(np.sum(x * s + (C - x) * xi)) / (2 * n)
        Qx = Z @ (Z.T @ x)
        rd = Qx - a * y - s + xi - 1.0
        rp = -float(a @ x)
        rs = -s * x
        rxi = -xi * (C - x)
        D = s / x + xi / (C - x)
        cond = float(D.max() / D.min())
        normdx = float(np.linalg.norm(rd))
        normdy = abs(rp)
        tmp = 0.5 * float(x @ Qx)
        pobj = tmp - float(x.sum())
        dobj = -tmp - C * float(xi.sum())
        log.append((it, mu, normdx, normdy, cond, pobj, dobj))
        if mu < tol and normdx < tol and normdy < tol:
            status = "converged"
            break
        if rel_gap_tol is not None:
            rel_gap = (pobj - dobj) / max(1.0, abs(pobj))
            scale = 1.0 + math.sqrt(n)
            if rel_gap <= rel_gap_tol and normdx / scale <= rel_gap_tol and normdy / scale <= rel_gap_tol:
                status = "converged"
                break
        if cond > 1e18:
            status = "ill_conditioned"
            break
        Zs = Z / np.sqrt(D)[:, None]
        M = Zs.T @ Zs + np.eye(k)
        try:
            Lm = cholesky(M, lower=True)
        except np.linalg.LinAlgError:
            status = "not_spd"
            break
        dx_a, dy_a, ds_a, dxi_a = newton_step(Z, D, Lm, C, a, x, s, xi, rd, rp, rs, rxi)
        alpha = _ratio(x, s, xi, dx_a, ds_a, dxi_a, C)
        mu_aff = float(np.sum((x + alpha * dx_a) * (s + alpha * ds_a)
                              + (C - x - alpha * dx_a) * (xi + alpha * dxi_a))) / (2 * n)
        sigma = (mu_aff / mu) ** 3
        rs_c = sigma * mu - dx_a * ds_a
        rxi_c = sigma * mu + dx_a * dxi_a
        dx_c, dy_c, ds_c, dxi_c = newton_step(Z, D, Lm, C, a, x, s, xi,
                                              np.zeros(n), 0.0, rs_c, rxi_c)
        dx = dx_c + dx_a
        dy = dy_c + dy_a
        ds = ds_c + ds_a
        dxi = dxi_c + dxi_a
        alpha = 0.99 * _ratio(x, s, xi, dx, ds, dxi, C)
        x = x + alpha * dx
        s = s + alpha * ds
        xi = xi + alpha * dxi
        y = y + alpha * dy
    return MpcResult(x=x, xi=xi, s=s, y=y, iters=it, status=status, log=log)


# ----------------------------------------------------------------------------------------
# Bias and model file (tensorsvm-train.cu:273-417)
# ----------------------------------------------------------------------------------------

def sv_sets(alpha, C):
    """SV: alpha > 1e-6; 'BSV' (the reference's name for free SVs): also alpha < C-1e-6."""
    sv = np.nonzero(alpha > 1e-6)[0]
    free = sv[alpha[sv] < C - 1e-6]
    return sv, free


def bias_rbf(U, labels, alpha, C):
    """Mean of y_j - sum_i alpha_i y_j (U_i.U_j) over the first <=50 free SVs (T:355-376).

    Returns (b, std); b is NaN when there is no free SV (T:372 divides by zero)."""
    sv, free = sv_sets(alpha, C)
    m = min(len(free), 50)
    if m == 0:
        return float("nan"), float("nan")
    U = np.asarray(U, np.float64)
    labels = np.asarray(labels, np.float64)
    Us = U[sv]
    bs = np.empty(m)
    for t in range(m):
        jj = free[t]
        sums = Us @ U[jj]
        bs[t] = labels[jj] - float(np.sum(alpha[sv] * labels[jj] * sums))
    b = bs.mean()
    return float(b), float(np.sqrt(np.mean((bs - b) ** 2)))


def linear_w_b(X, labels, alpha, C):
    """w = sum alpha_i y_i x_i over SVs; b = mean over the first <=5000 free SVs (T:301-332)."""
    sv, free = sv_sets(alpha, C)
    X = np.asarray(X, np.float64)
    labels = np.asarray(labels, np.float64)
    w = (alpha[sv] * labels[sv]) @ X[sv]
    m = min(len(free), 5000)
    b = 0.0
    if m > 0:
        bs = labels[free[:m]] - X[free[:m]] @ w
        b = float(bs.mean())
    return w, b


def format_model_rbf(alpha, labels, X, C, gamma, b, pos, neg) -> str:
    """LIBSVM/ThunderSVM text model exactly as tensorsvm-train.cu:384-406 writes it."""
    sv, free = sv_sets(alpha, C)
    out = ["svm_type c_svc\n", "kernel_type rbf\n", "gamma %.7f\n" % gamma, "nr_class 2\n",
           "total_sv %d\n" % len(sv), "rho %f\n" % (-b), "label %d %d\n" % (pos, neg),
           "nr_sv %d %d\n" % (len(free), len(sv) - len(free)), "SV\n"]
    for j in sv:
        parts = ["%7f " % (float(labels[j]) * float(alpha[j]))]
        for c in np.nonzero(X[j])[0]:
            parts.append("%d:%7f " % (c + 1, float(X[j, c])))
        out.append("".join(parts) + "\n")
    return "".join(out)


def format_model_linear(w, b, d, pos, neg) -> str:
    """LIBLINEAR text model as tensorsvm-train.cu:340-349 writes it."""
    out = ["solver_type L2R_L1LOSS_SVC_DUAL\n", "nr_class 2\n", "label %d %d\n" % (pos, neg),
           "nr_feature %d\n" % d, "bias %d\n" % 1, "w\n"]
    out += ["%.16f \n" % float(v) for v in w]
    out.append("%.16f\n" % b)
    return "".join(out)


def parse_model(text: str) -> dict:
    """Parse an RBF model file into header fields, SV coefficients and a dense SV matrix."""
    lines = text.splitlines()
    hdr = {}
    i = 0
    while lines[i].strip() != "SV":
        key, *vals = lines[i].split()
        hdr[key] = vals
        i += 1
    coefs, svs = [], []
    for ln in lines[i + 1:]:
        toks = ln.split()
        if not toks:
            continue
        coefs.append(float(toks[0]))
        svs.append({int(t.split(":")[0]): float(t.split(":")[1]) for t in toks[1:]})
    return {"header": hdr, "coef": np.asarray(coefs), "sv": svs,
            "rho": float(hdr["rho"][0]), "gamma": float(hdr["gamma"][0])}


def decision_values(model: dict, Xtest, d: int) -> np.ndarray:
    """f(x) = sum_i coef_i exp(-gamma ||sv_i - x||^2) - rho in FP64 (the ThunderSVM rule)."""
    S = np.zeros((len(model["sv"]), d))
    for r, feats in enumerate(model["sv"]):
        for c, v in feats.items():
            S[r, c - 1] = v
    Xt = np.asarray(Xtest, np.float64)
    out = np.empty(Xt.shape[0])
    for i in range(0, Xt.shape[0], 1024):
        blk = Xt[i:i + 1024]
        d2 = (blk * blk).sum(1)[:, None] + (S * S).sum(1)[None, :] - 2 * blk @ S.T
        out[i:i + 1024] = np.exp(-model["gamma"] * d2) @ model["coef"] - model["rho"]
    return out


def decision_values_dense(alpha, labels, X, gamma, b, Xtest) -> np.ndarray:
    """Exact-kernel decision values from in-memory alpha (no text rounding)."""
    sv = np.nonzero(alpha > 1e-6)[0]
    coef = np.asarray(alpha[sv], np.float64) * np.asarray(labels[sv], np.float64)
    S = np.asarray(X[sv], np.float64)
    Xt = np.asarray(Xtest, np.float64)
    out = np.empty(Xt.shape[0])
    for i in range(0, Xt.shape[0], 1024):
        blk = Xt[i:i + 1024]
        d2 = (blk * blk).sum(1)[:, None] + (S * S).sum(1)[None, :] - 2 * blk @ S.T
        out[i:i + 1024] = np.exp(-gamma * d2) @ coef + b
    return out


def train_rbf(X, labels, gamma, C, k, Q=None, **mpc_kw):
    """LRA + mpc + bias, the reference's RBF training path end to end (FP64)."""
    f = lra(X, labels, gamma, k, Q=Q)
    r = mpc(f.U, labels, C, kernel="rbf", **mpc_kw)
    b, bstd = bias_rbf(f.U, labels, r.x, C)
    return f, r, b


def train_linear(X, labels, C, **mpc_kw):
    """Z = diag(y) X, mpc with the linear initialisation, w and b (tensorsvm-train.cu:907-930)."""
    Z = np.asarray(X, np.float64) * np.asarray(labels, np.float64)[:, None]
    r = mpc(Z, labels, C, kernel="linear", **mpc_kw)
    w, b = linear_w_b(X, labels, r.x, C)
    return r, w, b


# ----------------------------------------------------------------------------------------
# Hypergradient (no reference counterpart): the FP64 restatement of tsvm_hypergrad's formulas
# ----------------------------------------------------------------------------------------

def hypergrad(X, y, Xv, yv, gamma, C, k, alpha, xi, s, b, Q=None):
    """Validation squared-hinge loss L and dL/dlog(gamma), dL/dlog(C), dL/dXv, in FP64 with
    exact kernels and a dense KKT solve.  The model is f(x) = sum_i alpha_i y_i K(x_i, x) + b
    with b = mean of y_j - y_j sum_i alpha_i Z_i.Z_j over the first <= 50 free SVs; the dual
    was solved on Q = Z Z^T = P Ky P from the range finder (B = Ky Omega, W R = B,
    P = W W^T), and the gamma derivative differentiates it with the sketch Omega fixed:
    dQ = dP Ky P + P dKy P + P Ky dP, dP x = (I-P) dB B+ x + B+^T dB^T (I-P) x, dB = dKy Omega.
    s, xi: the multipliers of the final iterate of the solver (D = s/alpha + xi/(C - alpha)).
    Returns (L, dL/dlog gamma, dL/dlog C, dL/dXv)."""
    X = np.asarray(X, np.float64); Xv = np.asarray(Xv, np.float64)
    y = np.asarray(y, np.float64); yv = np.asarray(yv, np.float64)
    alpha = np.asarray(alpha, np.float64); xi = np.asarray(xi, np.float64)
    n, m = len(y), len(yv)
    Om = polar_sketch(n, k) if Q is None else np.asarray(Q, np.float64)
    d2 = ((X[:, None, :] - X[None, :, :]) ** 2).sum(-1)
    Ky = y[:, None] * np.exp(-gamma * d2) * y[None, :]
    W, R = np.linalg.qr(Ky @ Om)
    Cm = W.T @ Ky @ W
    w, V = np.linalg.eigh(0.5 * (Cm + Cm.T))
    Z = W @ (V * np.sqrt(np.maximum(w, 0.0)))
    d2tv = ((X[:, None, :] - Xv[None, :, :]) ** 2).sum(-1)
    Ktv = np.exp(-gamma * d2tv)
    beta = alpha * y
    f = Ktv.T @ beta + b
    h = np.maximum(0.0, 1.0 - yv * f)
    L = float(np.sum(h * h) / m)
    g = -2.0 * yv * h / m
    Gb = float(g.sum())
    F = [i for i in range(n) if 1e-6 < alpha[i] < C - 1e-6][:50]
    zF = (y[F][:, None] * Z[F]).sum(0) if F else np.zeros(Z.shape[1])
    c = y * (Ktv @ g) - (Gb / len(F) if F else 0.0) * (Z @ zF)
    D = np.asarray(s, np.float64) / alpha + xi / (C - alpha)
    A = np.zeros((n + 1, n + 1))
    A[:n, :n] = Z @ Z.T + np.diag(D)
    A[:n, n] = y
    A[n, :n] = y
    lam = np.linalg.solve(A, np.concatenate([c, [0.0]]))[:n]
    dKy = y[:, None] * (-d2 * np.exp(-gamma * d2)) * y[None, :]
    P = lambda v: W @ (W.T @ v)
    Bp = lambda v: np.linalg.solve(R, W.T @ v)
    BpT = lambda v: W @ np.linalg.solve(R.T, v)
    u = P(alpha)
    E1 = Ky @ u
    D1 = dKy @ (Om @ Bp(E1)); D2 = dKy @ (E1 - P(E1)); D3 = dKy @ u
    D4 = dKy @ (Om @ Bp(alpha)); D5 = dKy @ (alpha - P(alpha))
    s2 = (D4 - P(D4)) + BpT(Om.T @ D5)
    r = (D1 - P(D1)) + BpT(Om.T @ D2) + P(D3) + P(Ky @ s2)
    dlogC = float(lam @ (C * xi / (C - alpha)))
    tv = (-d2tv * Ktv).T @ beta
    dlogg = -gamma * float(lam @ r) - (Gb * gamma * float(np.mean(y[F] * r[F])) if F else 0.0) \
        + gamma * float(g @ tv)
    S0 = Ktv.T @ beta
    S1 = Ktv.T @ (beta[:, None] * X)
    dXv = -2.0 * gamma * g[:, None] * (Xv * S0[:, None] - S1)
    return L, dlogg, dlogC, dXv
