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

PRECISIONS = {"fp32": _lib.PREC_FP32, "bf16": _lib.PREC_BF16, "fp16": _lib.PREC_FP16}


def _ptr(t) -> int:
    return int(t.data_ptr()) if t is not None else 0


def _fields(struct) -> dict:
    return {name: getattr(struct, name) for name, _ in struct._fields_}


def factor(ctx, X, y, gamma: float, k: int, precision: str = "fp32", Q=None, ldz: int | None = None):
    """Z (n x ldz float32 CUDA tensor, ldz = round_up(k, 64) by default) with Z Z^T ~= Y K Y."""
    import torch
    n, d = X.shape
    kp = ((k + 63) // 64) * 64
    ldz = ldz or kp
    Z = torch.empty((n, ldz), dtype=torch.float32, device=X.device)
    info = _lib.FactorInfo()
    sketch = _lib.SKETCH_USER if Q is not None else _lib.SKETCH_GLIBC
    st = ctx.lib.tsvm_factor(ctx.handle, _ptr(X), _ptr(y), n, d, float(gamma), k,
                             PRECISIONS[precision], sketch, _ptr(Q), _ptr(Z), ldz,
                             ctypes.byref(info))
    _lib.check(st, "tsvm_factor")
    return Z, _fields(info)


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


def write_model(path: str, model: Model, X: np.ndarray, labels: np.ndarray, pos: int, neg: int):
    """The reference's model text: LIBSVM rbf (T:384-406) or LIBLINEAR (T:340-349)."""
    alpha, C = model.alpha, model.C
    sv = np.nonzero(alpha > 1e-6)[0]
    free = sv[alpha[sv] < C - 1e-6]
    with open(path, "w") as f:
        if model.kernel == _lib.KERNEL_RBF:
            f.write("svm_type c_svc\nkernel_type rbf\n")
            f.write("gamma %.7f\n" % model.gamma)
            f.write("nr_class 2\ntotal_sv %d\n" % len(sv))
            f.write("rho %f\n" % (-model.b))
            f.write("label %d %d\n" % (pos, neg))
            f.write("nr_sv %d %d\nSV\n" % (len(free), len(sv) - len(free)))
            for j in sv:
                parts = ["%7f " % (float(labels[j]) * float(alpha[j]))]
                for c in np.nonzero(X[j])[0]:
                    parts.append("%d:%7f " % (c + 1, float(X[j, c])))
                f.write("".join(parts) + "\n")
        else:
            d = X.shape[1]
            w = (alpha[sv] * labels[sv].astype(np.float64)) @ X[sv].astype(np.float64)
            f.write("solver_type L2R_L1LOSS_SVC_DUAL\nnr_class 2\n")
            f.write("label %d %d\nnr_feature %d\nbias %d\nw\n" % (pos, neg, d, 1))
            for v in w:
                f.write("%.16f \n" % v)
            f.write("%.16f\n" % model.b)


def read_libsvm(path: str):
    """Dense float32 instances and labels, 1-based indices (tensorsvm-train.cu:1162-1278)."""
    labels, rows, max_index, min_index = [], [], 0, 1
    with open(path) as f:
        for line in f:
            toks = line.split()
            if not toks:
                continue
            labels.append(float(toks[0]))
            feats = [(int(t.split(":")[0]), float(t.split(":")[1])) for t in toks[1:]]
            for i, _ in feats:
                min_index = min(min_index, i)
                max_index = max(max_index, i)
            rows.append(feats)
    nf = max_index - min_index + 1 if min_index == 0 else max_index
    X = np.zeros((len(rows), nf), dtype=np.float32)
    for r, feats in enumerate(rows):
        for i, v in feats:
            X[r, i - min_index] = v
    return np.asarray(labels, dtype=np.float32), X
