"""Host-side logic and the C ABI boundary, without a GPU: the library loads and exports every
declared symbol, the CLI parses/rejects input like the reference, I/O formats round-trip."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, has_gpu
from oracle import oracle as orc
from tensorsvm_b200 import _lib, api, synth


def declared_functions(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tsvm_\w+)\s*\(", text)))


@pytest.mark.parametrize("header", ["tensorsvm.h", "tensorsvm_testing.h"])
def test_library_exports_every_declared_symbol(header):
    lib = _lib.load()
    names = declared_functions(header)
    assert names, header
    for name in names:
        assert hasattr(lib, name), name
    expected = _lib.EXPORTS if header == "tensorsvm.h" else _lib.TEST_EXPORTS
    assert set(names) == set(expected)


def test_status_strings():
    lib = _lib.load()
    assert lib.tsvm_status_string(_lib.ERR_NOT_SPD).decode().startswith("capacitance")
    assert lib.tsvm_status_string(999).decode() == "unknown status"


def test_default_options_are_the_reference_constants():
    o = _lib.default_options()
    assert o.max_iter == 100 and o.tol == 1e-7 and o.kernel == _lib.KERNEL_RBF


def test_cli_usage_without_arguments():
    p = subprocess.run([_lib.CLI_PATH], capture_output=True, text=True)
    assert p.returncode == 1 and "Usage: tensorsvm-train" in p.stdout


def test_cli_rejects_unknown_kernel(tmp_path):
    p = subprocess.run([_lib.CLI_PATH, "-t", "1", "x"], capture_output=True, text=True)
    assert p.returncode == 1 and "unimplemented -t 1" in p.stdout


@pytest.mark.parametrize("line", ["1 1:0.5 1:0.7\n", "1 a:0.5\n", "x 1:0.5\n", "1 2:zz\n"])
def test_cli_rejects_malformed_libsvm(tmp_path, line):
    f = tmp_path / "bad.train"
    f.write_text("1 1:0.1 2:0.2\n-1 1:0.3\n" + line)
    p = subprocess.run([_lib.CLI_PATH, str(f)], capture_output=True, text=True)
    assert p.returncode == 1
    assert "Wrong input format" in p.stdout or "Empty line" in p.stdout


def test_cli_single_class_is_an_error(tmp_path):
    f = tmp_path / "one.train"
    f.write_text("1 1:0.1\n1 1:0.3\n")
    p = subprocess.run([_lib.CLI_PATH, str(f)], capture_output=True, text=True)
    assert p.returncode == 1 and "single class" in p.stderr


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_cli_reports_missing_device(tmp_path):
    X, y = synth.two_gaussians(64, 3, seed=1)
    f = tmp_path / "t.train"
    synth.write_libsvm(str(f), X, y)
    p = subprocess.run([_lib.CLI_PATH, "-t", "2", "-k", "4", str(f)], capture_output=True, text=True)
    assert p.returncode == 1 and "no CUDA device" in p.stderr


def test_libsvm_round_trip(tmp_path):
    X, y, *_ = synth.make("c1", n=300)
    X[5, 3] = 0.0
    f = tmp_path / "r.train"
    synth.write_libsvm(str(f), X, y)
    lab, X2 = api.read_libsvm(str(f))
    assert np.array_equal(X2, X) and np.array_equal(lab, y)
    lab3, X3 = orc.read_libsvm(str(f))
    assert np.array_equal(X3, X)


def test_model_writer_matches_reference_format(tmp_path):
    X, y, *_ = synth.make("c1", n=200)
    rng = np.random.default_rng(0)
    alpha = np.where(rng.random(200) < 0.5, 0.0, rng.random(200) * 32)
    alpha[:3] = 32.0
    m = api.Model(kernel=_lib.KERNEL_RBF, alpha=alpha, b=0.0123, C=32.0, gamma=0.01, status=0)
    path = tmp_path / "m.model"
    api.write_model(str(path), m, X, y, 1, -1)
    ref_text = orc.format_model_rbf(alpha, y, X, 32.0, 0.01, 0.0123, 1, -1)
    assert path.read_text() == ref_text
    lin = api.Model(kernel=_lib.KERNEL_LINEAR, alpha=alpha, b=0.5, C=32.0, gamma=0.0, status=0)
    api.write_model(str(path), lin, X, y, 1, -1)
    # w summed over the SVs in index order, as writemodel's loop (T:330-335) does
    w = np.zeros(X.shape[1])
    for j in np.nonzero(alpha > 1e-6)[0]:
        w += alpha[j] * float(y[j]) * X[j].astype(np.float64)
    assert path.read_text() == orc.format_model_linear(w, 0.5, X.shape[1], 1, -1)


def test_label_remap_first_label_is_positive():
    y, pos, neg = orc.remap_labels(np.array([-1, 1, -1, 1], dtype=np.float32))
    assert (pos, neg) == (-1, 1) and list(y) == [1, -1, 1, -1]
