"""Kernel-level parity on the GPU (through the C ABI test hooks) against the CPU oracle."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as orc
from tensorsvm_b200 import _lib, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def P(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("count", [1, 31, 2048, 2049, 3_000_001])
def test_rand_stream_bit_exact(ctx, count):
    out = torch.empty(count, dtype=torch.int32, device="cuda")
    _lib.check(ctx.lib.tsvm_test_rand_stream(ctx.handle, count, P(out)), "rand")
    got = out.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, orc.glibc_rand(count))


@pytest.mark.parametrize("n,k", [(8192, 32), (1000, 50), (3, 1), (65536, 256)])
def test_sketch_matches_reference_stream(ctx, n, k):
    cnt = n * k
    out = torch.empty(cnt, dtype=torch.float32, device="cuda")
    _lib.check(ctx.lib.tsvm_test_sketch(ctx.handle, cnt, P(out)), "sketch")
    got = out.cpu().numpy()
    ref = orc.polar_sketch(n, k).ravel()
    # same accept/reject pattern and order; values differ only where log() rounds differently
    # (a 1-ulp log difference grows to a few ulp through the division, sqrt and product)
    assert np.array_equal(np.sign(got), np.sign(ref))
    ulp = np.abs(got.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
    assert ulp.max() <= 4
    assert np.mean(ulp != 0) < 5e-3


@pytest.mark.parametrize("k", [1, 32, 33, 50, 64, 97, 129, 256, 400, 864])
def test_cholesky_and_solve(ctx, k):
    rng = np.random.default_rng(k)
    A = rng.standard_normal((k, k + 5))
    M = A @ A.T + np.eye(k)
    L = dev(M.copy())
    info = ctypes.c_int32(-1)
    _lib.check(ctx.lib.tsvm_test_chol(ctx.handle, P(L), k, ctypes.byref(info)), "chol")
    assert info.value == 0
    Lh = np.tril(L.cpu().numpy())
    assert np.allclose(Lh, np.linalg.cholesky(M), rtol=1e-10, atol=1e-10)
    B = rng.standard_normal((2, k))
    Bd = dev(B.copy())
    _lib.check(ctx.lib.tsvm_test_potrs(ctx.handle, P(L), k, P(Bd), 2, k), "potrs")
    assert np.allclose(Bd.cpu().numpy(), np.linalg.solve(M, B.T).T, rtol=1e-8, atol=1e-10)


@pytest.mark.parametrize("n,bad", [(40, 17), (100, 70), (100, 0), (65, 64), (160, 32), (200, 150),
                                   (256, 255), (300, 290)])
def test_cholesky_reports_indefinite(ctx, n, bad):
    # the first failing pivot's 1-based column, in the first panel and in later ones (n <= 256:
    # the cluster kernel, a failure in any of its CTAs; 300: the one-CTA kernel)
    M = np.eye(n)
    M[bad, bad] = -1.0
    L = dev(M)
    info = ctypes.c_int32(0)
    _lib.check(ctx.lib.tsvm_test_chol(ctx.handle, P(L), n, ctypes.byref(info)), "chol")
    assert info.value == bad + 1


# k <= 128: the one-CTA packed solver; above: the cooperative-grid one
@pytest.mark.parametrize("k", [2, 7, 32, 127, 128, 130, 256])
def test_jacobi_eigensolver(ctx, k):
    rng = np.random.default_rng(100 + k)
    A = rng.standard_normal((k, k))
    S = (A + A.T) / 2
    S[0, :] *= 1e3  # spread of scales, and one negative direction kept in the spectrum
    S = (S + S.T) / 2
    w = torch.empty(k, dtype=torch.float64, device="cuda")
    V = torch.empty((k, k), dtype=torch.float64, device="cuda")
    sweeps = ctypes.c_int32(0)
    Sd = dev(S.copy())
    _lib.check(ctx.lib.tsvm_test_eig(ctx.handle, P(Sd), k, P(w), P(V), ctypes.byref(sweeps)), "eig")
    wh, Vh = w.cpu().numpy(), V.cpu().numpy()
    assert 0 < sweeps.value < 40
    assert np.allclose(np.sort(wh), np.linalg.eigvalsh(S), rtol=1e-10, atol=1e-9 * np.abs(S).max())
    assert np.linalg.norm(Vh @ np.diag(wh) @ Vh.T - S) / np.linalg.norm(S) < 1e-12
    assert np.linalg.norm(Vh.T @ Vh - np.eye(k)) < 1e-11


@pytest.mark.parametrize("k,count", [(128, 64), (64, 9), (33, 5), (130, 3)])
def test_jacobi_eigensolver_batched(ctx, k, count):
    """The batched factor's eigensolver (one CTA per problem in one launch up to k = 128, the
    grid eigensolver one problem after the other above) against numpy, problem by problem."""
    rng = np.random.default_rng(300 + k + count)
    S = rng.standard_normal((count, k, k))
    S = (S + np.transpose(S, (0, 2, 1))) / 2
    S *= np.logspace(0, 3, count)[:, None, None]   # problems of different scales
    w = torch.empty((count, k), dtype=torch.float64, device="cuda")
    V = torch.empty((count, k, k), dtype=torch.float64, device="cuda")
    sweeps = ctypes.c_int32(0)
    _lib.check(ctx.lib.tsvm_test_eig_batched(ctx.handle, P(dev(S.copy())), k, count, P(w), P(V),
                                             ctypes.byref(sweeps)), "eig_batched")
    assert 0 < sweeps.value < 40
    for b in range(count):
        wh, Vh = w[b].cpu().numpy(), V[b].cpu().numpy()
        sc = np.abs(S[b]).max()
        assert np.allclose(np.sort(wh), np.linalg.eigvalsh(S[b]), rtol=1e-10, atol=1e-9 * sc)
        assert np.linalg.norm(Vh @ np.diag(wh) @ Vh.T - S[b]) / np.linalg.norm(S[b]) < 1e-12
        assert np.linalg.norm(Vh.T @ Vh - np.eye(k)) < 1e-11


def test_grid_barrier_wait_runs_out_and_context_stays_usable(ctx):
    # the cooperative eigensolver's grid barrier with an arrival that never comes: every block
    # gives up after its bounded poll count, the error flag reads back as a status, and the same
    # context then runs a barrier that completes and a solve
    released = ctypes.c_int32(-1)
    st = ctx.lib.tsvm_test_grid_barrier(ctx.handle, 8, 9, 1 << 14, ctypes.byref(released))
    assert st == _lib.ERR_TIMEOUT and released.value == 0
    st = ctx.lib.tsvm_test_grid_barrier(ctx.handle, 8, 8, 1 << 14, ctypes.byref(released))
    assert st == _lib.OK and released.value == 8
    S = np.diag(np.arange(1.0, 9.0))
    w = torch.empty(8, dtype=torch.float64, device="cuda")
    V = torch.empty((8, 8), dtype=torch.float64, device="cuda")
    sweeps = ctypes.c_int32(0)
    _lib.check(ctx.lib.tsvm_test_eig(ctx.handle, P(dev(S)), 8, P(w), P(V), ctypes.byref(sweeps)),
               "eig")
    assert np.allclose(np.sort(w.cpu().numpy()), np.arange(1.0, 9.0))


# symmetric and general, narrow and wide (k = 400: seven 64-column tiles, the last ragged), ld > k
@pytest.mark.parametrize("sym,ka,kb", [(True, 70, 70), (False, 70, 33), (True, 256, 256),
                                       (False, 256, 256), (True, 400, 400), (False, 130, 200),
                                       (True, 128, 128), (False, 127, 300), (True, 129, 129)])
def test_gram_fp64_exact_products(ctx, sym, ka, kb):
    rng = np.random.default_rng(7 + ka)
    n = 10007
    lda, ldb = ka + 2, kb + 3
    A = rng.standard_normal((n, lda)).astype(np.float32)
    B = A if sym else rng.standard_normal((n, ldb)).astype(np.float32)
    s = rng.random(n) + 0.5
    G = torch.empty((ka, kb), dtype=torch.float64, device="cuda")
    Ad, Bd, sd = dev(A), dev(B), dev(s)
    _lib.check(ctx.lib.tsvm_test_gram(ctx.handle, P(Ad), lda, P(Bd), B.shape[1], n, ka, kb,
                                      int(sym), P(sd), P(G)), "gram")
    ref = (A[:, :ka].astype(np.float64) * s[:, None]).T @ B[:, :kb].astype(np.float64)
    assert np.allclose(G.cpu().numpy(), ref, rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("n,d,kp", [(3001, 18, 64), (1024, 54, 128), (517, 28, 256), (700, 5, 448)])
def test_kermatmul_fp32(ctx, n, d, kp):
    rng = np.random.default_rng(n)
    X = rng.standard_normal((n, d)).astype(np.float32)
    y = np.where(rng.random(n) < 0.5, 1.0, -1.0).astype(np.float32)
    A = rng.standard_normal((n, kp)).astype(np.float32)
    W = torch.empty((n, kp), dtype=torch.float32, device="cuda")
    g = 0.05
    Xd, yd, Ad = dev(X), dev(y), dev(A)   # keep the device copies alive across the call
    _lib.check(ctx.lib.tsvm_test_kermatmul(ctx.handle, P(Xd), P(yd), n, d, g, P(Ad), kp,
                                           P(W), _lib.PREC_FP32, 0), "kermatmul")
    ref = orc.kermatmul(X, y, g, A)
    err = np.linalg.norm(W.cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err < 2e-6, err


@pytest.mark.parametrize("prec,tol", [(_lib.PREC_FP16, 2e-3), (_lib.PREC_BF16, 1.5e-2)])
@pytest.mark.parametrize("n,d,kp", [(3001, 18, 64), (517, 12, 256), (1000, 18, 448), (300, 3, 128),
                                    # Gram K 128 and 192 (d > 19), with column slabs
                                    (1500, 28, 256), (700, 40, 128), (900, 54, 448), (600, 62, 64)])
def test_kermatmul_tensor_core(ctx, n, d, kp, prec, tol):
    rng = np.random.default_rng(n + kp)
    X = rng.standard_normal((n, d)).astype(np.float32)
    y = np.where(rng.random(n) < 0.5, 1.0, -1.0).astype(np.float32)
    A = rng.standard_normal((n, kp)).astype(np.float32)
    W = torch.empty((n, kp), dtype=torch.float32, device="cuda")
    g = 0.05
    Xd, yd, Ad = dev(X), dev(y), dev(A)
    _lib.check(ctx.lib.tsvm_test_kermatmul(ctx.handle, P(Xd), P(yd), n, d, g, P(Ad), kp,
                                           P(W), prec, 0), "kermatmul_tc")
    ref = orc.kermatmul(X, y, g, A)
    err = np.linalg.norm(W.cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err < tol, err


def test_kermatmul_tensor_core_distance_precision(ctx):
    # the split-FP16 Gram must resolve close pairs: K near 1 for near-duplicate rows
    rng = np.random.default_rng(5)
    n, d, kp = 1024, 18, 64
    base = rng.standard_normal((n // 2, d)).astype(np.float32) * 3.0
    X = np.concatenate([base, base + 1e-3 * rng.standard_normal(base.shape).astype(np.float32)])
    y = np.ones(n, dtype=np.float32)
    A = np.zeros((n, kp), dtype=np.float32)
    A[np.arange(n), np.arange(n) % kp] = 1.0
    W = torch.empty((n, kp), dtype=torch.float32, device="cuda")
    Xd, yd, Ad = dev(X), dev(y), dev(A)
    _lib.check(ctx.lib.tsvm_test_kermatmul(ctx.handle, P(Xd), P(yd), n, d, 0.5, P(Ad), kp, P(W),
                                           _lib.PREC_FP16, 0), "kermatmul_tc")
    ref = orc.kermatmul(X, y, 0.5, A)
    assert np.max(np.abs(W.cpu().numpy() - ref)) < 2e-3 * np.max(np.abs(ref))


@pytest.mark.parametrize("npoly", ["0", "2", "6", "8"])
def test_kermatmul_tensor_core_exp_split(ctx, npoly, monkeypatch):
    # every MUFU / polynomial split of the exponentials gives the same product
    monkeypatch.setenv("TSVM_TC_POLY", npoly)
    rng = np.random.default_rng(11)
    n, d, kp = 2000, 18, 128
    X = rng.standard_normal((n, d)).astype(np.float32)
    y = np.where(rng.random(n) < 0.5, 1.0, -1.0).astype(np.float32)
    A = rng.standard_normal((n, kp)).astype(np.float32)
    W = torch.empty((n, kp), dtype=torch.float32, device="cuda")
    Xd, yd, Ad = dev(X), dev(y), dev(A)
    _lib.check(ctx.lib.tsvm_test_kermatmul(ctx.handle, P(Xd), P(yd), n, d, 0.05, P(Ad), kp, P(W),
                                           _lib.PREC_FP16, 0), "kermatmul_tc")
    ref = orc.kermatmul(X, y, 0.05, A)
    assert np.linalg.norm(W.cpu().numpy() - ref) / np.linalg.norm(ref) < 2e-3


def _kermatmul(ctx, X, y, g, A, prec, split):
    n, kp = A.shape
    W = torch.empty((n, kp), dtype=torch.float32, device="cuda")
    Xd, yd, Ad = dev(X), dev(y), dev(A)
    _lib.check(ctx.lib.tsvm_test_kermatmul(ctx.handle, P(Xd), P(yd), n, X.shape[1], g, P(Ad), kp,
                                           P(W), prec, split), "kermatmul_tc")
    return W.cpu().numpy()


@pytest.mark.parametrize("n,d,kp", [(3001, 18, 64), (1000, 18, 448), (1500, 28, 256),
                                    (900, 54, 448)])
@pytest.mark.parametrize("prec,tol_split,tol_one", [(_lib.PREC_FP16, 2e-5, 2e-4),
                                                    (_lib.PREC_BF16, 2e-4, 2e-3)])
def test_kermatmul_kernel_block_split(ctx, n, d, kp, prec, tol_split, tol_one):
    """The kernel block as hi + lo (the range-finder pass): with an operand that the 16-bit type
    holds exactly, only the kernel block's rounding is left, and the split removes it."""
    rng = np.random.default_rng(7 * n + kp)
    X = rng.standard_normal((n, d)).astype(np.float32)
    y = np.where(rng.random(n) < 0.5, 1.0, -1.0).astype(np.float32)
    A = rng.standard_normal((n, kp)).astype(np.float16 if prec == _lib.PREC_FP16 else np.float32)
    if prec == _lib.PREC_BF16:   # round to bf16 on the host
        A = (A.view(np.uint32) & np.uint32(0xFFFF0000)).view(np.float32)
    A = A.astype(np.float32)
    ref = orc.kermatmul(X, y, 0.05, A)
    e_split = np.linalg.norm(_kermatmul(ctx, X, y, 0.05, A, prec, 1) - ref) / np.linalg.norm(ref)
    e_one = np.linalg.norm(_kermatmul(ctx, X, y, 0.05, A, prec, 0) - ref) / np.linalg.norm(ref)
    assert e_split < tol_split, (e_split, e_one)
    assert e_one > 4 * e_split


@pytest.mark.parametrize("n,kp", [(2048, 64), (3001, 256), (1000, 448)])
@pytest.mark.parametrize("prec,tol_split", [(_lib.PREC_FP16, 5e-6), (_lib.PREC_BF16, 2e-5)])
def test_kermatmul_operand_split(ctx, n, kp, prec, tol_split):
    """The operand as hi + lo (the projection pass): on points in well-separated groups of exact
    duplicates the kernel block is exactly 0 or 1, so only the operand's rounding is left, and
    the split removes it (the one-product form keeps a 16-bit rounding of A).  What remains is
    the FP32 accumulation over ~n/8 unit terms per group, ~sqrt(n) 2^-24 relative (measured
    2.3e-6 at n = 2048 and 3.2e-6 at n = 3001 for FP16, against 1.9e-4 and 2.0e-4 unsplit)."""
    rng = np.random.default_rng(n + 3 * kp)
    d = 18
    # squared distances between centres ~2300 (exp2 of the scaled distance underflows the
    # 16-bit types), within a group the Gram product leaves |S| << 2^-12, so exp2 rounds to 1
    centres = 8.0 * rng.standard_normal((8, d)).astype(np.float32)
    X = centres[rng.integers(0, 8, n)]
    y = np.where(rng.random(n) < 0.5, 1.0, -1.0).astype(np.float32)
    A = rng.standard_normal((n, kp)).astype(np.float32)
    ref = orc.kermatmul(X, y, 0.05, A)
    e_split = np.linalg.norm(_kermatmul(ctx, X, y, 0.05, A, prec, 2) - ref) / np.linalg.norm(ref)
    e_one = np.linalg.norm(_kermatmul(ctx, X, y, 0.05, A, prec, 0) - ref) / np.linalg.norm(ref)
    assert e_split < tol_split, (e_split, e_one)
    assert e_one > 10 * e_split


@pytest.mark.parametrize("spacing", [1, 700, 1025])
def test_bias_first_free_svs_spread_over_many_rounds(ctx, spacing):
    """tsvm_bias with free SVs spread over many 1024-row rounds of its index scan (the 50th
    beyond 34,000 rows at spacing 700 and 1025), against the oracle's bias (T:355-376)."""
    from tensorsvm_b200 import api
    rng = np.random.default_rng(100 + spacing)
    n, k, C = 60 * spacing + 500, 40, 4.0
    Zh = rng.standard_normal((n, k)).astype(np.float32)
    yh = np.where(rng.random(n) < 0.5, 1.0, -1.0).astype(np.float32)
    ah = np.where(rng.random(n) < 0.5, C, 0.0)
    free = np.arange(3, n, spacing)[:70]
    ah[free] = rng.uniform(0.1, C - 0.1, len(free))
    b_ref, bstd_ref = orc.bias_rbf(Zh, yh, ah, C)
    b, bstd, nsv, nfree = api.bias(ctx, dev(Zh), dev(yh), dev(ah), k, C)
    sv, fr = orc.sv_sets(ah, C)
    assert (nsv, nfree) == (len(sv), len(fr))
    assert abs(b - b_ref) <= 1e-9 * max(1.0, abs(b_ref))
    assert abs(bstd - bstd_ref) <= 1e-9 * max(1.0, abs(bstd_ref))


@pytest.mark.parametrize("seed,count", [(0, 1), (1, 7), (12345, 4096), (2 ** 40 + 3, 1_000_001)])
def test_philox_sketch_matches_oracle(ctx, seed, count):
    """TSVM_SKETCH_PHILOX against the oracle's FP64 restatement: the same Philox words (the
    uniforms agree exactly), FP32 logf / sqrtf / sincospif within a few ulp."""
    out = torch.empty(max(count, 4), dtype=torch.float32, device="cuda")
    _lib.check(ctx.lib.tsvm_test_sketch_philox(ctx.handle, seed, count, P(out)), "philox")
    got = out.cpu().numpy()[:count].astype(np.float64)
    ref = orc.philox_sketch(seed, count)
    assert np.max(np.abs(got - ref)) < 2e-5 * max(1.0, np.max(np.abs(ref)))
    out2 = torch.empty_like(out)
    _lib.check(ctx.lib.tsvm_test_sketch_philox(ctx.handle, seed, count, P(out2)), "philox")
    assert torch.equal(out[:count], out2[:count])


def test_factor_with_philox_sketch_matches_oracle(ctx):
    from tensorsvm_b200 import api
    X, y = synth.two_gaussians(3000, 18, seed=9)
    g, k = 0.05, 48
    Z, _ = api.factor(ctx, dev(X), dev(y), g, k, "fp32", philox_seed=99)
    Q = orc.philox_sketch(99, 3000 * k).reshape(3000, k).astype(np.float32)
    f = orc.lra(X, y, g, k, Q=Q.astype(np.float64))
    Zh = Z.cpu().numpy()[:, :k].astype(np.float64)
    G, Gr = Zh @ Zh.T, f.U @ f.U.T
    assert np.linalg.norm(G - Gr) / np.linalg.norm(Gr) < 1e-4
    Z2, _ = api.factor(ctx, dev(X), dev(y), g, k, "fp32", philox_seed=100)
    assert not torch.equal(Z, Z2)
