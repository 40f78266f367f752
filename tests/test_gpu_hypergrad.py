"""tsvm_hypergrad on the GPU: against the FP64 restatement (oracle.hypergrad) on the same
solution, and, wrapped in a torch.autograd.Function (here only, in the test harness), against
central finite differences of the GPU pipeline (factor -> IPM -> bias -> validation loss) with
the bias' free-SV set held at the base point."""
import numpy as np
import pytest

from oracle import oracle as orc
from tensorsvm_b200 import _lib, api, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

N, NV, K, D = 2000, 500, 64, 28


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def data():
    X, y = synth.tanh_teacher(N, D, seed=5)
    Xv, yv = synth.tanh_teacher(NV, D, seed=55)
    return X, y, Xv, yv


def train(ctx, X, y, gamma, C, prec="fp32"):
    Z, _ = api.factor(ctx, X, y, gamma, K, prec)
    alpha, xi, ym, st = api.ipm(ctx, Z, y, K, C, want_xi=True, tol=1e-9,
                                precision=_lib.PREC_FP32 if prec == "fp32" else _lib.PREC_BF16)
    b, _, _, _ = api.bias(ctx, Z, y, alpha, K, C)
    return Z, alpha, (xi, st["s"]), ym, b


def loss_fixed_free_set(ctx, X, y, Xv, yv, gamma, C, F):
    """Validation loss of the GPU-trained model, bias averaged over the given free set F."""
    Z, alpha, _, _, _ = train(ctx, X, y, gamma, C)
    Zk = Z[:, :K].double()
    a, yy = alpha, y.double()
    bF = torch.stack([yy[j] - yy[j] * (a * (Zk @ Zk[j])).sum() for j in F]).mean()
    d2 = torch.cdist(X.double(), Xv.double()) ** 2
    f = torch.exp(-gamma * d2).T @ (a * yy) + bF
    h = torch.clamp(1.0 - yv.double() * f, min=0.0)
    return float((h * h).sum() / Xv.shape[0])


class SvmValidationLoss(torch.autograd.Function):
    """loss(log gamma, log C) of the trained SVM; backward from tsvm_hypergrad."""

    @staticmethod
    def forward(fctx, log_gamma, log_C, ctx, X, y, Xv, yv):
        gamma, C = float(torch.exp(log_gamma)), float(torch.exp(log_C))
        Z, alpha, xi, ym, b = train(ctx, X, y, gamma, C)
        res, _ = api.hypergrad(ctx, X, y, Xv, yv, gamma, C, K, alpha, xi[0], xi[1], ym, b)
        fctx.save_for_backward(torch.tensor([res["dloss_dlog_gamma"], res["dloss_dlog_C"]],
                                            dtype=torch.float64))
        fctx.alpha, fctx.C = alpha, C
        return torch.tensor(res["loss"], dtype=torch.float64)

    @staticmethod
    def backward(fctx, grad):
        (g,) = fctx.saved_tensors
        return grad * g[0], grad * g[1], None, None, None, None, None


def test_hypergrad_matches_fp64_restatement(ctx, data):
    X, y, Xv, yv = data
    gamma, C = 0.03, 16.0
    Xd, yd, Xvd, yvd = dev(X), dev(y), dev(Xv), dev(yv)
    Z, alpha, xi, ym, b = train(ctx, Xd, yd, gamma, C)
    res, dxv = api.hypergrad(ctx, Xd, yd, Xvd, yvd, gamma, C, K, alpha, xi[0], xi[1], ym, b,
                             want_dxv=True)
    L, dg, dc, dxv_o = orc.hypergrad(X, y, Xv, yv, gamma, C, K, alpha.cpu().numpy(),
                                     xi[0].cpu().numpy(), xi[1].cpu().numpy(), b)
    assert abs(res["loss"] - L) <= 1e-5 * max(1.0, L)
    assert abs(res["dloss_dlog_C"] - dc) <= 1e-3 * max(abs(dc), 1e-3 * L), (res, dc)
    assert abs(res["dloss_dlog_gamma"] - dg) <= 1e-3 * max(abs(dg), 1e-3 * L), (res, dg)
    err = np.linalg.norm(dxv.cpu().numpy() - dxv_o) / np.linalg.norm(dxv_o)
    assert err < 1e-4, err
    assert 0 < res["n_free_bias"] <= 50


def test_hypergrad_fp16_factor_matches_fp64_restatement(ctx, data):
    # the tensor-core factor rounds its second-pass basis to FP16 in place; the range-finder
    # derivative needs the basis before rounding (B = W R), which R^-1 would otherwise amplify
    X, y, Xv, yv = data
    gamma, C = 0.03, 16.0
    Xd, yd, Xvd, yvd = dev(X), dev(y), dev(Xv), dev(yv)
    Z, alpha, xi, ym, b = train(ctx, Xd, yd, gamma, C, "fp16")
    res, _ = api.hypergrad(ctx, Xd, yd, Xvd, yvd, gamma, C, K, alpha, xi[0], xi[1], ym, b,
                           precision="fp16")
    L, dg, dc, _ = orc.hypergrad(X, y, Xv, yv, gamma, C, K, alpha.cpu().numpy(),
                                 xi[0].cpu().numpy(), xi[1].cpu().numpy(), b)
    assert abs(res["loss"] - L) <= 1e-4 * max(1.0, L)
    # the oracle differentiates its own FP64 factor: the FP16 factor's rounding shows up here
    assert abs(res["dloss_dlog_C"] - dc) <= 3e-2 * max(abs(dc), 1e-3 * L), (res, dc)
    assert abs(res["dloss_dlog_gamma"] - dg) <= 3e-2 * max(abs(dg), 1e-3 * L), (res, dg)


def test_hypergrad_autograd_matches_central_differences(ctx, data):
    X, y, Xv, yv = data
    Xd, yd, Xvd, yvd = dev(X), dev(y), dev(Xv), dev(yv)
    lg = torch.tensor(np.log(0.03), dtype=torch.float64, requires_grad=True)
    lc = torch.tensor(np.log(16.0), dtype=torch.float64, requires_grad=True)
    loss = SvmValidationLoss.apply(lg, lc, ctx, Xd, yd, Xvd, yvd)
    loss.backward()
    # free set of the base solution
    _, alpha, _, _, _ = train(ctx, Xd, yd, 0.03, 16.0)
    a = alpha.cpu().numpy()
    F = [i for i in range(N) if 1e-6 < a[i] < 16.0 - 1e-6][:50]
    # step 1e-4 in log space: at 1e-3 the central difference of this loss carries a ~6%
    # truncation error (measured with the FP64 pipeline: 98.9 at 1e-3, 105.1 at 1e-4, adjoint
    # 104.9), from support vectors changing status inside the interval
    h = 1e-4
    L = lambda g, c: loss_fixed_free_set(ctx, Xd, yd, Xvd, yvd, g, c, F)
    fd_g = (L(0.03 * np.exp(h), 16.0) - L(0.03 * np.exp(-h), 16.0)) / (2 * h)
    fd_c = (L(0.03, 16.0 * np.exp(h)) - L(0.03, 16.0 * np.exp(-h))) / (2 * h)
    scale = 1e-3 * float(loss.detach())
    assert abs(float(lc.grad) - fd_c) <= 2e-2 * max(abs(fd_c), scale), (float(lc.grad), fd_c)
    assert abs(float(lg.grad) - fd_g) <= 2e-2 * max(abs(fd_g), scale), (float(lg.grad), fd_g)


@pytest.mark.parametrize("na,nb,nu,deriv", [(2000, 2000, 1, False), (3001, 1777, 5, True),
                                            (500, 4000, 29, False), (1000, 1000, 1, True)])
def test_kernel_vector_products_tc_and_simt(ctx, na, nb, nu, deriv):
    """The hypergradient's kernel-vector products, SIMT and tensor-core forms, against FP64:
    out = sum_j w_ij K(a_i, b_j) U_j, w = 1 or -||a_i - b_j||^2 (dK/dgamma), rectangular row
    sets included."""
    import ctypes
    rng = np.random.default_rng(na + nb + nu)
    A = rng.standard_normal((na, D)).astype(np.float32)
    B = rng.standard_normal((nb, D)).astype(np.float32) + 0.3
    U = rng.standard_normal((nb, nu))
    gamma = 0.03
    d2 = ((A.astype(np.float64)[:, None, :] - B.astype(np.float64)[None, :, :]) ** 2).sum(-1)
    Kab = np.exp(-gamma * d2)
    ref = ((-d2 * Kab) if deriv else Kab) @ U
    Ad, Bd, Ud = dev(A), dev(B), dev(U)
    for tc, tol in ((0, 1e-5), (1, 2e-5)):
        out = torch.empty((na, nu), dtype=torch.float64, device="cuda")
        _lib.check(ctx.lib.tsvm_test_kprod(ctx.handle, ctypes.c_void_p(Ad.data_ptr()), na,
                                           ctypes.c_void_p(Bd.data_ptr()), nb, D, gamma,
                                           ctypes.c_void_p(Ud.data_ptr()), nu,
                                           ctypes.c_void_p(out.data_ptr()), int(deriv), tc),
                   "kprod")
        err = np.linalg.norm(out.cpu().numpy() - ref) / np.linalg.norm(ref)
        assert err < tol, (tc, err)


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_hypergrad_reuses_kept_factor(ctx, data, prec):
    """With tsvm_set_factor_keep the backward reuses the forward's factor (sketch, R, unrounded
    basis, Z) instead of recomputing it, with the same result as the recomputing call."""
    X, y, Xv, yv = data
    gamma, C = 0.03, 16.0
    Xd, yd, Xvd, yvd = dev(X), dev(y), dev(Xv), dev(yv)
    with _lib.Context(0) as c2:
        c2.set_factor_keep(True)
        Z, alpha, xi, ym, b = train(c2, Xd, yd, gamma, C, prec)
        kept, _ = api.hypergrad(c2, Xd, yd, Xvd, yvd, gamma, C, K, alpha, xi[0], xi[1], ym, b,
                                precision=prec)
    with _lib.Context(0) as c3:   # no kept factor: recomputed
        fresh, _ = api.hypergrad(c3, Xd, yd, Xvd, yvd, gamma, C, K, alpha, xi[0], xi[1], ym, b,
                                 precision=prec)
    assert kept["factor_reused"] == 1 and fresh["factor_reused"] == 0
    for key in ("loss", "dloss_dlog_gamma", "dloss_dlog_C"):
        assert abs(kept[key] - fresh[key]) <= 1e-10 * max(1.0, abs(fresh[key])), key
