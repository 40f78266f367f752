import os
import re
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 box)")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx():
    if not has_gpu():
        pytest.skip("no CUDA device")
    from tensorsvm_b200 import _lib
    c = _lib.Context(0)
    yield c
    c.close()


def ref_fixture(name):
    """(sv_index, coef, rho, header) of a compacted reference model."""
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    hdr = str(z["header"])
    rho = float(re.search(r"rho (\S+)", hdr).group(1))
    return z["sv_index"], z["coef"], rho, hdr


def ref_log(name):
    """[(iter, mu, normdx, normdy, cond, pobj, dobj)] from a reference log."""
    out = []
    pat = re.compile(r"iter (\d+), mu=(\S+), normdx=(\S+), normdy=(\S+) max/min\(D\)=(\S+) "
                     r"pobj=(\S+) dobj=(\S+)")
    with open(os.path.join(GOLDEN, name + ".log")) as f:
        for ln in f:
            m = pat.search(ln)
            if m:
                out.append(tuple(float(v) for v in m.groups()))
    return out


def jaccard(a, b) -> float:
    a, b = set(map(int, a)), set(map(int, b))
    return len(a & b) / max(1, len(a | b))
