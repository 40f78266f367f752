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
