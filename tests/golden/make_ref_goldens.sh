#!/usr/bin/env bash
# Run the reference trainer (oracle/_ref/tensorsvm-train-ref, built by oracle/build_ref.sh from
# robbwu/tensorsvm's tensorsvm-train.cu) on seeded synthetic data and keep its model files and
# logs.  Needs a GPU (the reference's LRA runs on cuBLAS/cuSOLVER).  The committed fixtures in
# tests/golden/ref_*.model and ref_*.log were produced by this script on a B200.
#
# usage: tests/golden/make_ref_goldens.sh OUTDIR [--timing]
set -euo pipefail
ROOT="$(cd "$(dirname "${BASH_SOURCE[0]}")/../.." && pwd)"
OUT="${1:?output directory}"
TIMING="${2:-}"
REF="$ROOT/oracle/_ref/tensorsvm-train-ref"
mkdir -p "$OUT"
cd "$ROOT"
echo "host cores: $(nproc)  OPENBLAS_NUM_THREADS=${OPENBLAS_NUM_THREADS:-unset}" > "$OUT/host.txt"

python3 - "$OUT" <<'PY'
import sys
from tensorsvm_b200 import synth
out = sys.argv[1]
X, y, *_ = synth.make("c1");            synth.write_libsvm(f"{out}/c1.train", X, y)
X, y = synth.two_gaussians(32768, 18, seed=7, noise=0.10); synth.write_libsvm(f"{out}/m32k.train", X, y)
PY

run() {  # name args...
  local name="$1"; shift
  local t0 t1
  t0=$(date +%s.%N)
  timeout 1200 "$REF" "$@" > "$OUT/$name.log" 2>&1
  t1=$(date +%s.%N)
  echo "$name wall_s $(python3 -c "print($t1-$t0)")" >> "$OUT/walltimes.txt"
}
run ref_c1_rbf   -k 32 -c 32 -g 0.01 -t 2 "$OUT/c1.train" "$OUT/ref_c1_rbf.model"
run ref_c1_lin   -k 32 -c 1 -t 0 "$OUT/c1.train" "$OUT/ref_c1_lin.model"
run ref_m32k_rbf -k 64 -c 32 -g 0.05 -t 2 "$OUT/m32k.train" "$OUT/ref_m32k_rbf.model"

if [ "$TIMING" = "--timing" ]; then
  python3 - "$OUT" <<'PY'
import sys
from tensorsvm_b200 import synth
out = sys.argv[1]
for n in (131072, 1000000):
    X, y, *_ = synth.make("c2", n=n)
    synth.write_libsvm(f"{out}/c2_{n}.train", X, y)
PY
  run ref_c2_131072 -k 256 -c 32 -g 0.05 -t 2 "$OUT/c2_131072.train" "$OUT/ref_c2_131072.model"
  run ref_c2_1000000 -k 256 -c 32 -g 0.05 -t 2 "$OUT/c2_1000000.train" "$OUT/ref_c2_1000000.model"
  rm -f "$OUT"/c2_*.train
  for m in "$OUT"/ref_c2_*.model; do   # keep only the header lines of the large models
    head -n 9 "$m" > "$m.head" && rm -f "$m"
  done
fi
rm -f "$OUT"/*.train
ls -la "$OUT"
