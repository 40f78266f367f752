"""Host I/O of the library (no GPU): the parallel LIBSVM reader against the oracle's restatement
of libsvmread (tensorsvm-train.cu:1162-1278), its error lines, and the model writer and reader
(writemodel, tensorsvm-train.cu:273-417) against the oracle's formatter."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as orc
from tensorsvm_b200 import _lib, api, synth


def write_lines(path, lines):
    path.write_text("".join(ln + "\n" for ln in lines))
    return str(path)


@pytest.mark.parametrize("threads", [1, 3, 8, 64])
def test_reader_matches_oracle_any_thread_count(tmp_path, threads):
    X, y, *_ = synth.make("c3", n=2000)       # one-hot columns: many omitted zeros
    f = tmp_path / "c3.train"
    synth.write_libsvm(str(f), X, y)
    lab, X2 = api.read_libsvm(str(f), threads=threads)
    lab_o, X_o = orc.read_libsvm(str(f))
    assert np.array_equal(lab, lab_o) and np.array_equal(X2, X_o)
    assert np.array_equal(X2, X)


def test_reader_values_are_strtod_rounded_to_float(tmp_path):
    # every value is the correctly rounded double of its decimal text (what strtod gives),
    # then rounded to float: the fast path for plain decimals and the general path agree
    rng = np.random.default_rng(12)
    toks = ["1e22", "1e23", "9007199254740993", "123456789012345678901", "-0", "+5", "4.9e-324",
            "1.7976931348623157e308", "00012.50", "1.5E+05", "-2.5e-22", "7e-23", "1e0",
            "0.000000000000000000000001", "3.4028235e38", "1.1754944e-38", "0.1", "-0.3"]
    for _ in range(3000):
        x = rng.uniform(-1, 1) * 10.0 ** rng.integers(-40, 40)
        toks.append(rng.choice(["%.9g", "%.17g", "%.6e", "%.3f", "%.25g"]) % x)
    lines = ["1 " + " ".join(f"{j + 1}:{t}" for j, t in enumerate(toks[i:i + 7]))
             for i in range(0, len(toks) - 6, 7)]
    p = write_lines(tmp_path / "v.train", lines)
    _, X = api.read_libsvm(p, threads=3)
    with np.errstate(over="ignore"):   # beyond float range: inf, as the C cast gives
        want = np.array([[np.float32(float(t)) for t in toks[i:i + 7]]
                         for i in range(0, len(toks) - 6, 7)], dtype=np.float32)
    assert X.shape == want.shape
    assert np.array_equal(X.view(np.uint32), want.view(np.uint32))


def test_reader_index_rules_and_scale256(tmp_path):
    # 0-based indices give max index + 1 columns; '+1' labels; tabs and CRLF; scale256
    p = write_lines(tmp_path / "z.train", ["+1 0:1.5\t3:2", "-1 1:-4 2:8e-1\r", "1"])
    lab, X = api.read_libsvm(p)
    assert list(lab) == [1, -1, 1] and X.shape == (3, 4)
    assert np.array_equal(X, np.array([[1.5, 0, 0, 2], [0, -4, 0.8, 0], [0, 0, 0, 0]],
                                      dtype=np.float32))
    lab2, X2 = api.read_libsvm(p, scale256=True)
    assert np.array_equal(X2, X / np.float32(256))
    lab_o, X_o = orc.read_libsvm(p, scale256=True)
    assert np.array_equal(X2, X_o)


@pytest.mark.parametrize("bad,line", [("1 2:1 2:3", 2), ("1 3:1 x:2", 2), ("", 2), ("1 1:abc", 2),
                                      ("one 1:1", 2), ("1 4", 2)])
def test_reader_reports_first_malformed_line(tmp_path, bad, line):
    p = write_lines(tmp_path / "bad.train", ["1 1:1 2:2", bad, "-1 1:3"] + ["1 1:1"] * 500)
    with pytest.raises(_lib.TsvmError) as e:
        api.read_libsvm(p, threads=4)
    assert e.value.line == line and e.value.status == _lib.ERR_IO


def test_reader_missing_file(tmp_path):
    with pytest.raises(_lib.TsvmError) as e:
        api.read_libsvm(str(tmp_path / "none.train"))
    assert e.value.status == _lib.ERR_IO and e.value.line == 0


@pytest.mark.parametrize("threads", [1, 5])
def test_writer_rbf_byte_identical_and_reader_round_trip(tmp_path, threads):
    X, y, *_ = synth.make("c3", n=3000)
    rng = np.random.default_rng(1)
    alpha = np.where(rng.random(3000) < 0.6, 0.0, rng.random(3000) * 32)
    alpha[:5] = 32.0
    m = api.Model(kernel=_lib.KERNEL_RBF, alpha=alpha, b=-0.25, C=32.0, gamma=0.02, status=0)
    path = tmp_path / "m.model"
    nsv, nfree = api.write_model(str(path), m, X, y, 7, 3, threads=threads)
    assert path.read_text() == orc.format_model_rbf(alpha, y, X, 32.0, 0.02, -0.25, 7, 3)
    sv = np.nonzero(alpha > 1e-6)[0]
    assert nsv == len(sv) and nfree == int(np.sum(alpha[sv] < 32.0 - 1e-6))
    mf = api.read_model(str(path))
    assert (mf.kernel, mf.pos, mf.neg) == (_lib.KERNEL_RBF, 7, 3)
    assert mf.rho == 0.25 and mf.gamma == 0.02
    # the file keeps %7f digits: values round-trip to 6 decimals
    assert np.max(np.abs(mf.coef - alpha[sv] * y[sv])) <= 5e-7
    assert mf.sv.shape[0] == len(sv)
    assert np.max(np.abs(mf.sv - X[sv][:, :mf.sv.shape[1]])) <= 5e-7 + 6e-8   # + float32 storage
    parsed = orc.parse_model(path.read_text())
    assert np.array_equal(mf.coef, parsed["coef"])


def test_writer_linear_and_reader(tmp_path):
    X, y, *_ = synth.make("c1", n=500)
    alpha = np.linspace(0, 2, 500)
    m = api.Model(kernel=_lib.KERNEL_LINEAR, alpha=alpha, b=0.75, C=1.0, gamma=0.0, status=0)
    path = tmp_path / "lin.model"
    api.write_model(str(path), m, X, y, 1, -1)
    mf = api.read_model(str(path))
    w = np.zeros(X.shape[1])
    for j in np.nonzero(alpha > 1e-6)[0]:
        w += alpha[j] * float(y[j]) * X[j].astype(np.float64)
    assert mf.kernel == _lib.KERNEL_LINEAR and mf.rho == -0.75
    assert np.allclose(mf.sv, w.astype(np.float32), rtol=1e-6, atol=0)
