#!/usr/bin/env bash
# Compile the reference trainer (robbwu/tensorsvm, tensorsvm-train.cu) from its own single
# source file, in place, into oracle/_ref/tensorsvm-train-ref.  Test infrastructure only:
# the binary is the reference arm of bench.py and the generator of tests/golden fixtures.
#
# Flags follow the reference's Makefile:11 (-O2 -m64 -DCUDA, compute_70 PTX that the driver
# JIT-compiles for sm_100).  MKL is not in the image; oracle/mklshim/mkl.h maps the twelve
# CBLAS/LAPACKE calls onto the scipy-bundled OpenBLAS 0.3.30.  NVBLAS (Makefile:13) is not
# linked: the reference calls cblas_* directly, which NVBLAS does not intercept.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
# The reference checkout is looked for beside the repository (../reference), unless
# TSVM_REFERENCE_SRC names the source file.
SRC="${TSVM_REFERENCE_SRC:-$HERE/../../reference/tensorsvm-train.cu}"
OUT="$HERE/_ref"
if [ ! -f "$SRC" ]; then
  echo "build_ref: reference source not found at $SRC; keeping existing $OUT" >&2
  exit 0
fi
OPENBLAS_DIR="$(python3 -c 'import os, scipy; print(os.path.join(os.path.dirname(scipy.__file__), os.pardir, "scipy.libs"))')"
OPENBLAS_DIR="$(cd "$OPENBLAS_DIR" && pwd)"
OPENBLAS_SO="$(ls "$OPENBLAS_DIR"/libscipy_openblas-*.so | head -1)"
mkdir -p "$OUT"
nvcc -O2 -m64 -DCUDA -w \
  -gencode=arch=compute_70,code=compute_70 \
  -I"$HERE/mklshim" \
  "$SRC" -o "$OUT/tensorsvm-train-ref" \
  -Xlinker "$OPENBLAS_SO" -Xlinker -rpath -Xlinker "$OPENBLAS_DIR" \
  -lpthread -lm -ldl -lcudart -lcublas -lcusolver
echo "build_ref: built $OUT/tensorsvm-train-ref"
