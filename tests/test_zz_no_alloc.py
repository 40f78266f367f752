"""The allocation-free bias entry point (tsvm_bias_noalloc) against the context-based one.

tsvm_bias_noalloc serves callers that must not let the library allocate device memory; its
scratch is a fixed static device array shared by every call.  This file is collected last so a
run that stops at the first failure has already run everything else; it also passes alone in
a fresh process.
"""
import ctypes

import numpy as np
import pytest

from tensorsvm_b200 import _lib, api, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_bias_noalloc_matches_context_bias_twice(ctx):
    X, y = synth.two_gaussians(3000, 18, seed=21, noise=0.05)
    g, C, k = 0.05, 8.0, 48
    Xd, yd = torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda()
    Z, _ = api.factor(ctx, Xd, yd, g, k, "fp32")
    alpha, _, _, _ = api.ipm(ctx, Z, yd, k, C)
    b, bstd, nsv, nfree = api.bias(ctx, Z, yd, alpha, k, C)
    assert nfree > 0
    out = torch.full((4,), -1.0, dtype=torch.float64, device="cuda")
    n, ldz = Z.shape
    for call in range(2):
        out.fill_(-1.0)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        st = ctx.lib.tsvm_bias_noalloc(Z.data_ptr(), ldz, yd.data_ptr(), alpha.data_ptr(), n, k, C,
                                       out.data_ptr(), None)
        assert st == _lib.OK
        torch.cuda.synchronize()
        if call == 1:  # the second call allocates nothing at all
            assert torch.cuda.mem_get_info()[0] == free_before
        got = out.cpu().numpy()
        assert abs(got[0] - b) <= 1e-9 * max(1.0, abs(b))
        assert abs(got[1] - bstd) <= 1e-9 * max(1.0, abs(bstd))
        assert (int(got[2]), int(got[3])) == (nsv, nfree)


def test_bias_noalloc_rejects_k_beyond_capacity(ctx):
    Z = torch.zeros((64, 1028), dtype=torch.float32, device="cuda")
    y = torch.ones(64, dtype=torch.float32, device="cuda")
    a = torch.zeros(64, dtype=torch.float64, device="cuda")
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    st = ctx.lib.tsvm_bias_noalloc(Z.data_ptr(), 1028, y.data_ptr(), a.data_ptr(), 64, 1025, 1.0,
                                   out.data_ptr(), None)
    assert st == _lib.ERR_INVALID_ARGUMENT


def _noalloc(ctx, Z, y, alpha, k, C, stream=None):
    out = torch.full((4,), -1.0, dtype=torch.float64, device="cuda")
    n, ldz = Z.shape
    st = ctx.lib.tsvm_bias_noalloc(Z.data_ptr(), ldz, y.data_ptr(), alpha.data_ptr(), n, k, C,
                                   out.data_ptr(), stream)
    assert st == _lib.OK
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("spacing", [1, 37, 700, 1025])
def test_bias_noalloc_sparse_free_svs_against_oracle(ctx, spacing):
    """Free SVs spread over many 1024-row rounds of the index scan (spacing 700 and 1025 put
    the 50th free SV beyond 34,000 rows), between bounded SVs and non-SVs, checked against
    the oracle's restatement of the reference's bias rule (T:355-376)."""
    from oracle import oracle as orc
    rng = np.random.default_rng(spacing)
    n, k, C = 60 * spacing + 500, 40, 4.0
    Zh = rng.standard_normal((n, 48)).astype(np.float32)
    yh = np.where(rng.random(n) < 0.5, 1.0, -1.0).astype(np.float32)
    ah = np.where(rng.random(n) < 0.5, C, 0.0)       # bounded SVs and non-SVs
    free = np.arange(3, n, spacing)[:70]
    ah[free] = rng.uniform(0.1, C - 0.1, len(free))  # free SVs, more than 50 of them
    b, bstd = orc.bias_rbf(Zh[:, :k], yh, ah, C)
    sv, fr = orc.sv_sets(ah, C)
    got = _noalloc(ctx, torch.from_numpy(Zh).cuda(), torch.from_numpy(yh).cuda(),
                   torch.from_numpy(ah).cuda(), k, C)
    assert (int(got[2]), int(got[3])) == (len(sv), len(fr))
    assert abs(got[0] - b) <= 1e-9 * max(1.0, abs(b))
    assert abs(got[1] - bstd) <= 1e-9 * max(1.0, abs(bstd))


def test_bias_noalloc_no_free_sv_gives_nan(ctx):
    """With every SV at the bound the reference's mean over free SVs is 0/0 (T:372): NaN."""
    n, k, C = 5000, 16, 2.0
    Zh = np.ones((n, k), np.float32)
    yh = np.ones(n, np.float32)
    ah = np.where(np.arange(n) % 3 == 0, C, 0.0)
    got = _noalloc(ctx, torch.from_numpy(Zh).cuda(), torch.from_numpy(yh).cuda(),
                   torch.from_numpy(ah).cuda(), k, C)
    assert np.isnan(got[0]) and np.isnan(got[1])
    assert (int(got[2]), int(got[3])) == (int((ah > 1e-6).sum()), 0)


def test_bias_noalloc_on_a_side_stream(ctx):
    """The call is asynchronous on the caller's stream."""
    from oracle import oracle as orc
    rng = np.random.default_rng(5)
    n, k, C = 4096, 32, 1.0
    Zh = rng.standard_normal((n, k)).astype(np.float32)
    yh = np.where(rng.random(n) < 0.5, 1.0, -1.0).astype(np.float32)
    ah = rng.uniform(0.0, C, n)
    b, _ = orc.bias_rbf(Zh, yh, ah, C)
    Zd, yd, ad = (torch.from_numpy(v).cuda() for v in (Zh, yh, ah))
    s = torch.cuda.Stream()
    out = torch.full((4,), -1.0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = ctx.lib.tsvm_bias_noalloc(Zd.data_ptr(), k, yd.data_ptr(), ad.data_ptr(), n, k, C,
                                   out.data_ptr(), ctypes.c_void_p(s.cuda_stream))
    assert st == _lib.OK
    s.synchronize()
    assert abs(out[0].item() - b) <= 1e-9 * max(1.0, abs(b))
