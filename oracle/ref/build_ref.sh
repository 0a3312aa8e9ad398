#!/bin/bash
# Builds the reference GPU correction from the reference checkout's own
# source (src/ExtreM_cuda.cu, unmodified) into oracle/_ref/ref_gpu, with the
# stub headers next to this script.  Test infrastructure only; needs the
# reference checkout given as the first argument -- the GPU box uses the built
# binary, which travels with the repository.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:?usage: build_ref.sh <reference checkout>}"
OUT="$HERE/../_ref"
mkdir -p "$OUT"
test -f "$REF/src/ExtreM_cuda.cu"
/usr/local/cuda/bin/nvcc -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -w \
  -I "$HERE/stubs" -I "$REF/src" -o "$OUT/ref_gpu" "$HERE/ref_harness.cu"
echo "$OUT/ref_gpu"
