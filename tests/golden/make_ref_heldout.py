"""Decision values of the reference build's own model for the benchmark workload on held-out
points, kept as a fixture for the full-size parity test.

The reference trainer (oracle/_ref/tensorsvm-train-ref, built by oracle/build_ref.sh; its LRA
runs on cuBLAS, so this needs a GPU) is run on synth "c2" (n = 1M, d = 18, gamma 0.05, C 32,
k 256, seed 2) written as a LIBSVM file.  Its model file is parsed and
f(x) = sum_i coef_i exp(-gamma ||sv_i - x||^2) - rho (the ThunderSVM rule) is evaluated in FP64
(torch on the GPU, in chunks; no code of this package) on the 20,000 points of synth "c2_test".

usage: python tests/golden/make_ref_heldout.py OUT_DIR
writes OUT_DIR/ref_c2_1000000_heldout.npz (f as float64, the model's label order, its SV counts)
and OUT_DIR/ref_c2_1000000_heldout.log (the reference's log).
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402
from tensorsvm_b200 import synth  # noqa: E402


def main(out: str) -> None:
    import torch
    os.makedirs(out, exist_ok=True)
    X, y, g, C, k = synth.make("c2")
    tmp = tempfile.mkdtemp()
    train = os.path.join(tmp, "c2.train")
    model_path = os.path.join(tmp, "c2.model")
    synth.write_libsvm(train, X, y)
    del X, y
    ref = os.path.join(ROOT, "oracle", "_ref", "tensorsvm-train-ref")
    p = subprocess.run([ref, "-k", str(k), "-c", str(C), "-g", str(g), "-t", "2", train,
                        model_path], capture_output=True, text=True, timeout=1800)
    with open(os.path.join(out, "ref_c2_1000000_heldout.log"), "w") as f:
        f.write(p.stdout + p.stderr)
    if p.returncode != 0:
        raise SystemExit(f"reference exited {p.returncode}")
    with open(model_path) as f:
        model = orc.parse_model(f.read())
    d = 18
    S = np.zeros((len(model["sv"]), d))
    for r, feats in enumerate(model["sv"]):
        for c, v in feats.items():
            S[r, c - 1] = v
    Xt, _, *_ = synth.make("c2_test")
    St = torch.from_numpy(S).cuda()
    coef = torch.from_numpy(model["coef"]).cuda()
    sn = (St * St).sum(1)
    f = np.empty(Xt.shape[0])
    for i in range(0, Xt.shape[0], 256):
        xb = torch.from_numpy(np.asarray(Xt[i:i + 256], np.float64)).cuda()
        d2 = (xb * xb).sum(1)[:, None] + sn[None, :] - 2.0 * xb @ St.T
        f[i:i + 256] = (torch.exp(-model["gamma"] * d2) @ coef).cpu().numpy() - model["rho"]
    hdr = model["header"]
    np.savez_compressed(os.path.join(out, "ref_c2_1000000_heldout.npz"), f=f,
                        labels=np.array([float(v) for v in hdr["label"]]),
                        total_sv=int(hdr["total_sv"][0]),
                        nr_sv=np.array([int(v) for v in hdr["nr_sv"]]), rho=model["rho"])
    print("held-out decision values:", f.shape, "max |f|", np.max(np.abs(f)))


if __name__ == "__main__":
    main(sys.argv[1])
