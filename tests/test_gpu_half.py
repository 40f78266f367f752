"""The half product of the projection pass: R = Y (K o H) Y A over the J blocks from the diagonal
on, H_ij = 1 (j > i), 1/2 (j == i), 0 (j < i), and the projection A^T (Y K Y) A rebuilt from it as
A^T R + R^T A + s u u^T.  Checked against FP64 (oracle) and against the full tensor-core product
of the same precision and split."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as orc
from tensorsvm_b200 import _lib

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
P = ctypes.c_void_p


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _half(ctx, X, y, g, A, prec, split):
    n, kp = A.shape
    R = torch.empty((n, kp), dtype=torch.float32, device="cuda")
    sym = torch.empty(kp + 1, dtype=torch.float64, device="cuda")
    Xd, yd, Ad = dev(X), dev(y), dev(A)
    _lib.check(ctx.lib.tsvm_test_kermatmul_half(ctx.handle, Xd.data_ptr(), yd.data_ptr(), n,
                                                X.shape[1], g, Ad.data_ptr(), kp, R.data_ptr(),
                                                sym.data_ptr(), prec, split), "kermatmul_half")
    return R.cpu().numpy().astype(np.float64), sym.cpu().numpy()


def _full(ctx, X, y, g, A, prec, split):
    n, kp = A.shape
    W = torch.empty((n, kp), dtype=torch.float32, device="cuda")
    Xd, yd, Ad = dev(X), dev(y), dev(A)
    _lib.check(ctx.lib.tsvm_test_kermatmul(ctx.handle, Xd.data_ptr(), yd.data_ptr(), n,
                                           X.shape[1], g, Ad.data_ptr(), kp, W.data_ptr(), prec,
                                           split), "kermatmul_tc")
    return W.cpu().numpy().astype(np.float64)


def _case(n, d, kp, flat, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, d)).astype(np.float32)
    y = np.where(rng.random(n) < 0.5, 1.0, -1.0).astype(np.float32)
    A = rng.standard_normal((n, kp)).astype(np.float32)
    # flat: entries in about [0.9, 1], so the kernel-mean shift is taken off
    g = 0.1 / (2.0 * d) if flat else 0.05
    return X, y, A, g


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


# n: one row block, ragged row blocks, a partial last round of CTAs (n > 148 * 128 rows);
# kp up to 448 (two column slabs); d across the Gram widths 64 / 128 / 192
@pytest.mark.parametrize("n,d,kp", [(3001, 18, 64), (1000, 18, 448), (1500, 28, 256), (900, 54, 448),
                                    (128, 5, 128), (129, 3, 64), (19001, 18, 64)])
@pytest.mark.parametrize("flat", [False, True])
# tolerances of the 16-bit kernel block's rounding (the operand split does not remove it; it
# averages out in the factor), as for the full product
@pytest.mark.parametrize("prec,split,tol", [(_lib.PREC_FP16, 2, 2e-3), (_lib.PREC_FP16_FAST, 0, 2e-3),
                                            (_lib.PREC_BF16, 2, 1.5e-2)])
def test_half_projection(ctx, n, d, kp, flat, prec, split, tol):
    X, y, A, g = _case(n, d, kp, flat, 31 * n + kp + flat)
    R, sym = _half(ctx, X, y, g, A, prec, split)
    A64 = A.astype(np.float64)
    Ch = A64.T @ R
    Ch = Ch + Ch.T + sym[0] * np.outer(sym[1:], sym[1:])
    ref = A64.T @ orc.kermatmul(X, y, g, A)
    assert _rel(Ch, ref) < tol, _rel(Ch, ref)
    # about as accurate as the full product of the same form
    W = _full(ctx, X, y, g, A, prec, split)
    Cf = A64.T @ W
    Cf = 0.5 * (Cf + Cf.T)
    assert _rel(Ch, ref) < 3.0 * _rel(Cf, ref) + 1e-7, (_rel(Ch, ref), _rel(Cf, ref))
    # u = A^T y over the operand the tensor cores saw; no shift for the peaked kernels (d >= 18
    # at gamma 0.05; with d = 3 or 5 that kernel is flat too)
    assert np.allclose(sym[1:], A64.T @ y.astype(np.float64), rtol=1e-3, atol=1e-3 * np.sqrt(n))
    if flat:
        assert 0.5 < sym[0] < 1.0
    elif d >= 18:
        assert sym[0] == 0.0


@pytest.mark.parametrize("n,d,kp", [(700, 18, 64), (300, 54, 128), (129, 3, 64)])
def test_half_product_rows(ctx, n, d, kp):
    """R itself, row by row: the masked, shifted kernel block (diagonal halved) times A."""
    for flat in (False, True):
        X, y, A, g = _case(n, d, kp, flat, 7 * n + kp)
        R, sym = _half(ctx, X, y, g, A, _lib.PREC_FP16, 2)
        K = orc.rbf_block(X, X, y, y, g)   # Y K Y
        yy = np.outer(y, y).astype(np.float64)
        H = np.triu(np.ones((n, n)), 1) + 0.5 * np.eye(n)
        ref = ((K - sym[0] * yy) * H) @ A.astype(np.float64)
        assert _rel(R, ref) < 2e-3, (flat, _rel(R, ref))
