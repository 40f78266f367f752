"""Python host side over the C ABI.

``factor`` / ``ipm`` / ``bias`` take CUDA tensors (anything with ``data_ptr()`` on the context's
device, e.g. torch tensors) and map to tsvm_factor / tsvm_ipm / tsvm_bias, which replace the
reference's LRA (tensorsvm-train.cu:1941), mpc (tensorsvm-train.cu:1507) and the bias part of
writemodel (tensorsvm-train.cu:355-376).  ``train`` runs the end-to-end path from host arrays
(tsvm_train, the path main() drives at tensorsvm-train.cu:907-1024) and ``write_model`` writes
the reference's LIBSVM / LIBLINEAR model text (tensorsvm-train.cu:334-409).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib

PRECISIONS = {"fp32": _lib.PREC_FP32, "bf16": _lib.PREC_BF16, "fp16": _lib.PREC_FP16,
              "bf16_fast": _lib.PREC_BF16_FAST, "fp16_fast": _lib.PREC_FP16_FAST}


def _ptr(t) -> int:
    return int(t.data_ptr()) if t is not None else 0


def _fields(struct) -> dict:
    return {name: getattr(struct, name) for name, _ in struct._fields_}


def factor(ctx, X, y, gamma: float, k: int, precision: str = "fp32", Q=None, ldz: int | None = None,
           philox_seed: int | None = None):
    """Z (n x ldz float32 CUDA tensor, ldz = round_up(k, 64) by default) with Z Z^T ~= Y K Y.
    The sketch is the reference's glibc stream, the caller's Q, or with philox_seed the
    counter-based Philox sketch of that seed."""
    import torch
    n, d = X.shape
    kp = ((k + 63) // 64) * 64
    ldz = ldz or kp
    Z = torch.empty((n, ldz), dtype=torch.float32, device=X.device)
    info = _lib.FactorInfo()
    sketch = _lib.SKETCH_USER if Q is not None else _lib.SKETCH_GLIBC
    if philox_seed is not None:
        _lib.check(ctx.lib.tsvm_set_sketch_seed(ctx.handle, int(philox_seed)), "tsvm_set_sketch_seed")
        sketch = _lib.SKETCH_PHILOX
    st = ctx.lib.tsvm_factor(ctx.handle, _ptr(X), _ptr(y), n, d, float(gamma), k,
                             PRECISIONS[precision], sketch, _ptr(Q), _ptr(Z), ldz,
                             ctypes.byref(info))
    _lib.check(st, "tsvm_factor")
    return Z, _fields(info)


def factor_batched(ctx, Xs, ys, gammas, k: int, precision: str = "fp32"):
    """Factors of many problems (tsvm_factor_batched): lists of CUDA tensors X (n_p x d), y and
    gammas; returns the list of Z (n_p x round_up(k, 64)) and of factor statistics."""
    import torch
    kp = ((k + 63) // 64) * 64
    count = len(Xs)
    d = Xs[0].shape[1]
    Zs = [torch.empty((X.shape[0], kp), dtype=torch.float32, device=X.device) for X in Xs]
    probs = (_lib.FactorProblem * count)()
    for p, (X, y, g, Z) in enumerate(zip(Xs, ys, gammas, Zs)):
        probs[p] = _lib.FactorProblem(_ptr(X), _ptr(y), X.shape[0], float(g), _ptr(Z))
    infos = (_lib.FactorInfo * count)()
    st = ctx.lib.tsvm_factor_batched(ctx.handle, probs, count, d, k, PRECISIONS[precision],
                                     _lib.SKETCH_GLIBC, kp, infos)
    _lib.check(st, "tsvm_factor_batched")
    return Zs, [_fields(i) for i in infos]


def ipm(ctx, Z, y, k: int, C: float, kernel: int = _lib.KERNEL_RBF, want_xi: bool = False, **opts):
    """Solve the dual with Q = Z Z^T; returns (alpha f64 CUDA tensor, xi or None, y_mult, stats).
    With want_xi the multipliers s of alpha >= 0 are returned as stats["s"] as well."""
    import torch
    n, ldz = Z.shape
    alpha = torch.empty(n, dtype=torch.float64, device=Z.device)
    xi = torch.empty(n, dtype=torch.float64, device=Z.device) if want_xi else None
    sv = torch.empty(n, dtype=torch.float64, device=Z.device) if want_xi else None
    o = _lib.default_options(kernel=kernel, **opts)
    ym = ctypes.c_double()
    stats = _lib.IpmStats()
    st = ctx.lib.tsvm_ipm(ctx.handle, _ptr(Z), ldz, _ptr(y), n, k, float(C), ctypes.byref(o),
                          _ptr(alpha), _ptr(xi), _ptr(sv), ctypes.byref(ym), ctypes.byref(stats))
    _lib.check(st, "tsvm_ipm", allow=(_lib.WARN_ILL_CONDITIONED, _lib.WARN_MAX_ITER,
                                       _lib.ERR_NOT_SPD))
    s = _fields(stats)
    s["status_code"] = st
    if want_xi:
        s["s"] = sv
    return alpha, xi, ym.value, s


def ipm_batched(ctx, Zs, ys, k: int, Cs, kernel: int = _lib.KERNEL_RBF, **opts):
    """Solve len(Zs) duals together (tsvm_ipm_batched).  Zs: CUDA float32 tensors n_i x ldz (one
    ldz for all), ys: CUDA float32 labels, Cs: penalties.  Returns (alphas, stats list, info)."""
    import torch
    count = len(Zs)
    ldz = Zs[0].shape[1]
    if any(Z.shape[1] != ldz for Z in Zs):
        raise ValueError("all problems need the same ldz")
    alphas = [torch.empty(Z.shape[0], dtype=torch.float64, device=Z.device) for Z in Zs]
    probs = (_lib.IpmProblem * count)()
    for i, (Z, y, C, a) in enumerate(zip(Zs, ys, Cs, alphas)):
        probs[i].Z, probs[i].y, probs[i].n = _ptr(Z), _ptr(y), Z.shape[0]
        probs[i].C, probs[i].alpha_out, probs[i].xi_out = float(C), _ptr(a), None
    o = _lib.default_options(kernel=kernel, **opts)
    stats = (_lib.IpmStats * count)()
    info = _lib.BatchInfo()
    st = ctx.lib.tsvm_ipm_batched(ctx.handle, probs, count, k, ldz, ctypes.byref(o), stats,
                                  ctypes.byref(info))
    _lib.check(st, "tsvm_ipm_batched", allow=(_lib.ERR_NOT_SPD,))
    return alphas, [_fields(s) for s in stats], _fields(info)


def hypergrad(ctx, X, y, Xv, yv, gamma: float, C: float, k: int, alpha, xi, s, ymult: float,
              b: float, precision: str = "fp32", want_dxv: bool = False):
    """tsvm_hypergrad on CUDA tensors (the factor is recomputed with `precision`): returns
    (result dict, dL/dXv tensor or None)."""
    import torch
    n, d = X.shape
    nv = Xv.shape[0]
    dxv = torch.empty((nv, d), dtype=torch.float32, device=X.device) if want_dxv else None
    r = _lib.HypergradResult()
    st = ctx.lib.tsvm_hypergrad(ctx.handle, _ptr(X), _ptr(y), n, d, _ptr(Xv), _ptr(yv), nv,
                                float(gamma), float(C), k, PRECISIONS[precision], _ptr(alpha),
                                _ptr(xi), _ptr(s), float(ymult), float(b), ctypes.byref(r),
                                _ptr(dxv))
    _lib.check(st, "tsvm_hypergrad")
    return _fields(r), dxv


def bias(ctx, Z, y, alpha, k: int, C: float):
    n, ldz = Z.shape
    b, bs = ctypes.c_double(), ctypes.c_double()
    nsv, nfree = ctypes.c_int32(), ctypes.c_int32()
    st = ctx.lib.tsvm_bias(ctx.handle, _ptr(Z), ldz, _ptr(y), _ptr(alpha), n, k, float(C),
                           ctypes.byref(b), ctypes.byref(bs), ctypes.byref(nsv), ctypes.byref(nfree))
    _lib.check(st, "tsvm_bias")
    return b.value, bs.value, nsv.value, nfree.value


@dataclass
class Model:
    kernel: int
    alpha: np.ndarray
    b: float
    C: float
    gamma: float
    status: int
    factor_info: dict = field(default_factory=dict)
    ipm_stats: dict = field(default_factory=dict)


def train(ctx, X: np.ndarray, y: np.ndarray, kernel: int = _lib.KERNEL_RBF, gamma: float = 0.0,
          C: float = 1.0, k: int = 50, precision: str = "fp32", **opts) -> Model:
    """End-to-end training from host arrays through tsvm_train (one C call)."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    n, d = X.shape
    alpha = np.empty(n, dtype=np.float64)
    b = ctypes.c_double()
    finfo, istats = _lib.FactorInfo(), _lib.IpmStats()
    opts.setdefault("precision", _lib.PREC_FP32 if precision == "fp32" else _lib.PREC_BF16)
    o = _lib.default_options(kernel=kernel, **opts)
    st = ctx.lib.tsvm_train(ctx.handle, X.ctypes.data, y.ctypes.data, n, d, kernel, float(gamma),
                            float(C), k, PRECISIONS[precision], ctypes.byref(o),
                            alpha.ctypes.data, ctypes.byref(b), ctypes.byref(finfo),
                            ctypes.byref(istats))
    _lib.check(st, "tsvm_train", allow=(_lib.WARN_ILL_CONDITIONED, _lib.WARN_MAX_ITER,
                                         _lib.ERR_NOT_SPD))
    return Model(kernel=kernel, alpha=alpha, b=b.value, C=C, gamma=gamma, status=st,
                 factor_info=_fields(finfo), ipm_stats=_fields(istats))


def write_model(path: str, model: Model, X: np.ndarray, labels: np.ndarray, pos: int, neg: int,
                threads: int = 0):
    """The reference's model text through tsvm_write_model: LIBSVM rbf (T:384-406) or LIBLINEAR
    (T:340-349).  Returns (number of SVs, number of free SVs)."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    labels = np.ascontiguousarray(labels, dtype=np.float32)
    alpha = np.ascontiguousarray(model.alpha, dtype=np.float64)
    n, d = X.shape
    nsv, nfree = ctypes.c_int64(), ctypes.c_int64()
    st = _lib.load().tsvm_write_model(path.encode(), model.kernel, X.ctypes.data, labels.ctypes.data,
                                      alpha.ctypes.data, n, d, float(model.C), float(model.gamma),
                                      float(model.b), pos, neg, threads, ctypes.byref(nsv),
                                      ctypes.byref(nfree))
    _lib.check(st, "tsvm_write_model")
    return nsv.value, nfree.value


def read_libsvm(path: str, scale256: bool = False, threads: int = 0):
    """(labels float32, X float32 n x d dense) through tsvm_read_libsvm (tensorsvm-train.cu:
    1162-1278 semantics, parallel parse).  A malformed line raises TsvmError with .line set."""
    lib = _lib.load()
    L, M = ctypes.c_void_p(), ctypes.c_void_p()
    n, d, nnz, bad = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    st = lib.tsvm_read_libsvm(path.encode(), int(scale256), threads, ctypes.byref(L),
                              ctypes.byref(M), ctypes.byref(n), ctypes.byref(d), ctypes.byref(nnz),
                              ctypes.byref(bad))
    if st != _lib.OK:
        err = _lib.TsvmError(st, f"tsvm_read_libsvm({path}) line {bad.value}")
        err.line = bad.value
        raise err
    try:
        labels = np.ctypeslib.as_array(ctypes.cast(L, ctypes.POINTER(ctypes.c_float)),
                                       shape=(n.value,)).copy() if n.value else np.zeros(0, np.float32)
        X = np.ctypeslib.as_array(ctypes.cast(M, ctypes.POINTER(ctypes.c_float)),
                                  shape=(n.value, d.value)).copy() if n.value * d.value \
            else np.zeros((n.value, d.value), np.float32)
    finally:
        lib.tsvm_free(L)
        lib.tsvm_free(M)
    return labels, X


@dataclass
class ModelFile:
    kernel: int
    pos: int
    neg: int
    rho: float
    gamma: float
    sv: np.ndarray          # RBF: nsv x d; LINEAR: w (d)
    coef: np.ndarray        # RBF: nsv


def read_model(path: str) -> ModelFile:
    """A model file (either format tsvm_write_model writes) through tsvm_read_model."""
    lib = _lib.load()
    mv = _lib.ModelView()
    pos, neg = ctypes.c_int32(), ctypes.c_int32()
    _lib.check(lib.tsvm_read_model(path.encode(), ctypes.byref(mv), ctypes.byref(pos),
                                   ctypes.byref(neg)), "tsvm_read_model")
    try:
        rows = mv.nsv if mv.kernel == _lib.KERNEL_RBF else 1
        sv = np.ctypeslib.as_array(ctypes.cast(mv.sv, ctypes.POINTER(ctypes.c_float)),
                                   shape=(rows, mv.d)).copy()
        coef = (np.ctypeslib.as_array(ctypes.cast(mv.coef, ctypes.POINTER(ctypes.c_double)),
                                      shape=(mv.nsv,)).copy()
                if mv.kernel == _lib.KERNEL_RBF and mv.nsv else np.zeros(0))
    finally:
        lib.tsvm_free_model(ctypes.byref(mv))
    return ModelFile(kernel=mv.kernel, pos=pos.value, neg=neg.value, rho=mv.rho, gamma=mv.gamma,
                     sv=sv if mv.kernel == _lib.KERNEL_RBF else sv[0], coef=coef)


def predict(ctx, model: ModelFile, X: np.ndarray) -> np.ndarray:
    """Decision values (float64) of host rows X through tsvm_predict; rows and SVs are padded to
    a common width."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    m, dx = X.shape
    sv = np.atleast_2d(model.sv)
    d = max(dx, sv.shape[1])
    if dx < d:
        X = np.ascontiguousarray(np.pad(X, ((0, 0), (0, d - dx))))
    if sv.shape[1] < d:
        sv = np.pad(sv, ((0, 0), (0, d - sv.shape[1])))
    sv = np.ascontiguousarray(sv, dtype=np.float32)
    coef = np.ascontiguousarray(model.coef, dtype=np.float64)
    mv = _lib.ModelView(kernel=model.kernel, d=d, nsv=sv.shape[0] if model.kernel == _lib.KERNEL_RBF else 0,
                        sv=sv.ctypes.data, coef=coef.ctypes.data if coef.size else None,
                        rho=model.rho, gamma=model.gamma)
    f = np.empty(m, dtype=np.float64)
    _lib.check(ctx.lib.tsvm_predict(ctx.handle, ctypes.byref(mv), X.ctypes.data, m, f.ctypes.data),
               "tsvm_predict")
    return f


def decision_values(ctx, kernel: int, sv, coef, rho: float, gamma: float, X):
    """tsvm_decision_values on CUDA tensors (sv nsv x d or w, coef float64, X m x d)."""
    import torch
    m, d = X.shape
    f = torch.empty(m, dtype=torch.float64, device=X.device)
    mv = _lib.ModelView(kernel=kernel, d=d, nsv=sv.shape[0] if kernel == _lib.KERNEL_RBF else 0,
                        sv=_ptr(sv), coef=_ptr(coef) if coef is not None else None, rho=float(rho),
                        gamma=float(gamma))
    _lib.check(ctx.lib.tsvm_decision_values(ctx.handle, ctypes.byref(mv), _ptr(X), m, _ptr(f)),
               "tsvm_decision_values")
    return f


def kernel_residual(ctx, X, y, gamma: float, Z, k: int):
    """(||K~||_F, ||K~ - Z Z^T||_F) in FP64 through tsvm_kernel_residual (CUDA tensors)."""
    n, d = X.shape
    a, b = ctypes.c_double(), ctypes.c_double()
    _lib.check(ctx.lib.tsvm_kernel_residual(ctx.handle, _ptr(X), _ptr(y), n, d, float(gamma),
                                            _ptr(Z), Z.shape[1], k, ctypes.byref(a),
                                            ctypes.byref(b)), "tsvm_kernel_residual")
    return a.value, b.value
