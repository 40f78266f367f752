"""The kernel-block product above 256 columns in one launch (32-row J units, W in up to 416
TMEM columns), against the FP64 oracle and against the column-slab form (two launches of at
most 256 columns, each recomputing the kernel block) on the same inputs."""
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


def _product(ctx, X, y, g, A, kw, prec, split):
    """W = (Y K Y) A; kw = 0 lets the library assume every column of A may be nonzero (kp = 448
    then runs as two slabs), kw > 0 that only the first kw are (one launch up to 416)."""
    n, kp = A.shape
    W = torch.full((n, kp), float("nan"), dtype=torch.float32, device="cuda")
    Xd, yd, Ad = dev(X), dev(y), dev(A)
    _lib.check(ctx.lib.tsvm_test_kermatmul_cols(ctx.handle, P(Xd.data_ptr()), P(yd.data_ptr()), n,
                                                X.shape[1], g, P(Ad.data_ptr()), kp, kw,
                                                P(W.data_ptr()), prec, split), "kermatmul_cols")
    return W.cpu().numpy().astype(np.float64)


def _half(ctx, X, y, g, A, kw, prec, split):
    n, kp = A.shape
    R = torch.full((n, kp), float("nan"), dtype=torch.float32, device="cuda")
    sym = torch.empty(kp + 1, dtype=torch.float64, device="cuda")
    Xd, yd, Ad = dev(X), dev(y), dev(A)
    _lib.check(ctx.lib.tsvm_test_kermatmul_half_cols(ctx.handle, P(Xd.data_ptr()),
                                                     P(yd.data_ptr()), n, X.shape[1], g,
                                                     P(Ad.data_ptr()), kp, kw, P(R.data_ptr()),
                                                     P(sym.data_ptr()), prec, split),
               "kermatmul_half_cols")
    return R.cpu().numpy().astype(np.float64), sym.cpu().numpy()


def _case(n, d, kp, kw, seed, flat=False):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, d)).astype(np.float32)
    y = np.where(rng.random(n) < 0.5, 1.0, -1.0).astype(np.float32)
    A = rng.standard_normal((n, kp)).astype(np.float32)
    A[:, kw:] = 0.0
    g = 0.1 / (2.0 * d) if flat else 0.05
    return X, y, A, g


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


# (n, d, kp, kw), kp = 448 so that kw = 0 selects the slab form: the config-3 shape's 400
# columns at Gram widths 64 and 192, 320 and the largest one-launch width 416 (Gram width 128), a
# ragged width (300 -> 304 MMA columns), one MMA of 208 columns, a partial last round of CTAs
# (n > 148 * 128)
WIDE = [(1000, 18, 448, 400), (900, 54, 448, 400), (700, 40, 448, 320), (517, 12, 448, 300),
        (640, 30, 448, 416), (300, 7, 448, 200), (19001, 18, 448, 400)]


@pytest.mark.parametrize("n,d,kp,kw", WIDE)
@pytest.mark.parametrize("prec,split,tol", [(_lib.PREC_FP16, 0, 2e-3), (_lib.PREC_FP16, 1, 2e-3),
                                            (_lib.PREC_FP16, 2, 2e-3), (_lib.PREC_BF16, 0, 1.5e-2),
                                            (_lib.PREC_BF16, 1, 1.5e-2)])
def test_one_launch_matches_oracle_and_slabs(ctx, n, d, kp, kw, prec, split, tol):
    X, y, A, g = _case(n, d, kp, kw, 13 * n + kp + kw + split)
    W1 = _product(ctx, X, y, g, A, kw, prec, split)
    assert np.all(W1[:, kw:] == 0.0)        # columns past kw written, as zeros
    ref = orc.kermatmul(X, y, g, A)
    assert _rel(W1, ref) < tol, _rel(W1, ref)
    # the slab form contracts the same 16-bit operands in the same J order; with a split the two
    # forms add the hi and lo products to the FP32 accumulator in another order
    W2 = _product(ctx, X, y, g, A, 0, prec, split)
    assert _rel(W1, W2) < (2e-6 if split == 0 else 2e-5), _rel(W1, W2)


@pytest.mark.parametrize("n,d,kp,kw", [(1000, 18, 448, 400), (900, 54, 448, 400),
                                       (640, 54, 448, 384), (19001, 18, 448, 400)])
@pytest.mark.parametrize("flat", [False, True])
@pytest.mark.parametrize("prec,split,tol", [(_lib.PREC_FP16, 2, 2e-3), (_lib.PREC_FP16_FAST, 0, 2e-3),
                                            (_lib.PREC_BF16, 2, 1.5e-2)])
def test_one_launch_half_projection(ctx, n, d, kp, kw, flat, prec, split, tol):
    """The projection pass's half product (from the diagonal on) in one launch: the units that
    cross the diagonal carry the 1 / 0.5 / 0 weights."""
    X, y, A, g = _case(n, d, kp, kw, 17 * n + kp + flat, flat)
    R1, sym1 = _half(ctx, X, y, g, A, kw, prec, split)
    assert np.all(R1[:, kw:] == 0.0)
    A64 = A.astype(np.float64)
    Ch = A64.T @ R1
    Ch = Ch + Ch.T + sym1[0] * np.outer(sym1[1:], sym1[1:])
    ref = A64.T @ orc.kermatmul(X, y, g, A)
    assert _rel(Ch, ref) < tol, _rel(Ch, ref)
    R2, sym2 = _half(ctx, X, y, g, A, 0, prec, split)
    assert _rel(R1, R2) < (2e-6 if split == 0 else 2e-5), _rel(R1, R2)
    assert np.array_equal(sym1, sym2)
