"""Turn the reference's model files (from make_ref_goldens.sh) into compact fixtures.

A model file lists every support vector's coefficient and its features as %7f.  The features
are regenerated exactly from the seeded generator, so a fixture keeps only the header, the
row index of each SV in the training set (matched by its printed features) and the printed
coefficient.  usage: python tests/golden/compact_goldens.py RUN_DIR
"""
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as orc  # noqa: E402
from tensorsvm_b200 import synth  # noqa: E402

DATASETS = {
    "ref_c1_rbf": lambda: synth.make("c1")[:2],
    "ref_m32k_rbf": lambda: synth.two_gaussians(32768, 18, seed=7, noise=0.10),
}


def compact(run_dir: str, name: str) -> None:
    X, y = DATASETS[name]()
    with open(os.path.join(run_dir, name + ".model")) as f:
        text = f.read()
    model = orc.parse_model(text)
    d = X.shape[1]
    S = np.zeros((len(model["sv"]), d))
    for r, feats in enumerate(model["sv"]):
        for c, v in feats.items():
            S[r, c - 1] = v
    Xr = np.round(X.astype(np.float64), 6)
    lookup = {tuple(row): i for i, row in enumerate(Xr)}
    idx = np.array([lookup[tuple(np.round(s, 6))] for s in S], dtype=np.int32)
    header = text.split("SV\n")[0]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), sv_index=idx,
                        coef=model["coef"].astype(np.float64), header=np.array(header))


if __name__ == "__main__":
    run = sys.argv[1]
    for name in DATASETS:
        compact(run, name)
    for f in os.listdir(run):
        if f.endswith(".log") or f.endswith(".model.head") or f == "ref_c1_lin.model" \
                or f in ("walltimes.txt", "host.txt"):
            shutil.copy(os.path.join(run, f), os.path.join(HERE, f))
    print("fixtures written to", HERE)
