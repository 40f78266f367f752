"""Seeded synthetic training sets standing in for the SUSY/covtype-shaped data the reference
trainer is run on (the datasets themselves are not available; none of their records are used).

Every generator is deterministic for a given seed (numpy PCG64) and returns float32 features
(row-major n x d) and float32 labels in {+1, -1}.

* ``two_gaussians``   config 1/2: class means +-0.5 u (u a random unit vector), unit covariance,
                      balanced labels, optional label noise.
* ``mixed_onehot``    config 3: 10 uniform[0,1] features + one-hot groups of 4 and 40 columns,
                      labels = sign of a random RBF function (median-centred), optional flips.
* ``tanh_teacher``    config 4/5: N(0,1) features, labels from a random two-layer tanh network.
"""
from __future__ import annotations

import numpy as np


def two_gaussians(n: int, d: int = 18, seed: int = 1, noise: float = 0.0, mix_seed: int = 1000):
    u = np.random.Generator(np.random.PCG64(mix_seed)).standard_normal(d)
    u /= np.linalg.norm(u)
    rng = np.random.Generator(np.random.PCG64(seed))
    y = np.ones(n, dtype=np.float32)
    y[n // 2:] = -1.0
    rng.shuffle(y)
    X = rng.standard_normal((n, d)).astype(np.float32)
    X += (0.5 * y[:, None] * u[None, :]).astype(np.float32)
    if noise > 0:
        flip = rng.random(n) < noise
        y[flip] = -y[flip]
    return X, y


def mixed_onehot(n: int, seed: int = 3, noise: float = 0.05, n_centres: int = 64,
                 fgamma: float = 0.5):
    rng = np.random.Generator(np.random.PCG64(seed))
    d = 54
    X = np.zeros((n, d), dtype=np.float32)
    X[:, :10] = rng.random((n, 10), dtype=np.float32)
    X[np.arange(n), 10 + rng.integers(0, 4, n)] = 1.0
    X[np.arange(n), 14 + rng.integers(0, 40, n)] = 1.0
    centres = X[rng.integers(0, n, n_centres)].astype(np.float64)
    w = rng.standard_normal(n_centres)
    f = np.empty(n)
    for i in range(0, n, 65536):
        blk = X[i:i + 65536].astype(np.float64)
        d2 = (blk * blk).sum(1)[:, None] + (centres * centres).sum(1)[None, :] - 2 * blk @ centres.T
        f[i:i + 65536] = np.exp(-fgamma * d2) @ w
    y = np.where(f > np.median(f), 1.0, -1.0).astype(np.float32)
    flip = rng.random(n) < noise
    y[flip] = -y[flip]
    return X, y


def tanh_teacher(n: int, d: int = 28, seed: int = 5, hidden: int = 32, teacher_seed: int = 4242):
    trng = np.random.Generator(np.random.PCG64(teacher_seed))
    W1 = trng.standard_normal((d, hidden)) / np.sqrt(d)
    b1 = 0.1 * trng.standard_normal(hidden)
    w2 = trng.standard_normal(hidden) / np.sqrt(hidden)
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, d)).astype(np.float32)
    f = np.tanh(X.astype(np.float64) @ W1 + b1) @ w2
    y = np.where(f > 0.0, 1.0, -1.0).astype(np.float32)
    if (y > 0).all() or (y < 0).all():
        y[0] = -y[0]
    return X, y


def batch_sizes(count: int = 64, lo: int = 2000, hi: int = 200000, seed: int = 44):
    """Problem sizes log-uniform in [lo, hi] for the batched (C, gamma) grid."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(np.int64)


def grid_problems(count: int = 64, lo: int = 2000, hi: int = 200000, seed: int = 44, d: int = 28):
    """The batched workload: `count` tanh-teacher problems of log-uniform sizes on the 8 x 8
    grid C in 2^{-2, 0, ..., 12}, gamma in 2^{-9, ..., -2} (row-major over (C, gamma)).
    Returns a list of (X, y, gamma, C)."""
    sizes = batch_sizes(count, lo, hi, seed)
    Cs = [2.0 ** e for e in range(-2, 13, 2)]
    gammas = [2.0 ** e for e in range(-9, -1)]
    out = []
    for i in range(count):
        X, y = tanh_teacher(int(sizes[i]), d=d, seed=1000 + i)
        out.append((X, y, gammas[i % 8], Cs[(i // 8) % 8]))
    return out


def write_libsvm(path: str, X: np.ndarray, y: np.ndarray) -> None:
    """LIBSVM text, values as %.9g so float32 round-trips exactly; zero features omitted."""
    with open(path, "w") as f:
        for i in range(X.shape[0]):
            row = X[i]
            nz = np.nonzero(row)[0]
            feats = " ".join("%d:%.9g" % (c + 1, float(row[c])) for c in nz)
            f.write("%d %s\n" % (int(y[i]), feats))


CONFIGS = {
    # name: (generator, kwargs, gamma, C, k)
    "c1": (two_gaussians, dict(n=8192, d=18, seed=1), 0.01, 32.0, 32),
    "c1_test": (two_gaussians, dict(n=2048, d=18, seed=101), 0.01, 32.0, 32),
    "c2": (two_gaussians, dict(n=1_000_000, d=18, seed=2, noise=0.10), 0.05, 32.0, 256),
    "c2_test": (two_gaussians, dict(n=20_000, d=18, seed=102, noise=0.10), 0.05, 32.0, 256),
    "c3": (mixed_onehot, dict(n=500_000, seed=3, noise=0.05), 0.02, 32.0, 400),
    "c5": (tanh_teacher, dict(n=200_000, d=28, seed=5), 0.03, 16.0, 256),
    "c5_val": (tanh_teacher, dict(n=50_000, d=28, seed=55), 0.03, 16.0, 256),
}


def make(name: str, n: int | None = None):
    """(X, y, gamma, C, k) for a named config; ``n`` overrides the row count (same generator)."""
    gen, kw, gamma, C, k = CONFIGS[name]
    kw = dict(kw)
    if n is not None:
        kw["n"] = n
    X, y = gen(**kw)
    return X, y, gamma, C, k
