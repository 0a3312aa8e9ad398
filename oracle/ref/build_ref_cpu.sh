#!/bin/bash
# Builds the reference's CPU correction (src/ExtreM.cpp + main.cpp of the
# reference checkout given as the first argument) into oracle/_ref/ref_cpu, the
# same program with zero-filled allocations into oracle/_ref/ref_cpu_zero,
# and its merge-tree functions behind a file interface into
# oracle/_ref/ref_mergetree.
# Test infrastructure only: it records the behaviour of the reference's CPU
# path on 2-D fields (census_cpu.py).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:?usage: build_ref_cpu.sh <reference checkout>}"
OUT="$HERE/../_ref"
mkdir -p "$OUT"
test -f "$REF/src/ExtreM.cpp"
FLAGS=(-O2 -std=c++17 -fopenmp -w -I "$HERE/stubs" -I "$REF" -I "$REF/include" -I "$REF/include/api" -I "$REF/src")
g++ "${FLAGS[@]}" -o "$OUT/ref_cpu" "$HERE/ref_cpu_harness.cpp"
g++ "${FLAGS[@]}" -o "$OUT/ref_cpu_zero" "$HERE/ref_cpu_harness.cpp" "$HERE/zero_alloc.cpp"
g++ "${FLAGS[@]}" -o "$OUT/ref_mergetree" "$HERE/ref_mergetree_harness.cpp"
echo "$OUT/ref_cpu $OUT/ref_cpu_zero $OUT/ref_mergetree"
