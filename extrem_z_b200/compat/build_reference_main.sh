#!/bin/bash
# Compiles the reference's own driver main.cpp, unmodified and against its own
# unmodified header include/api/ExtreM.h, and links it against this
# repository's libExtreMz.so (the reference host API over the GPU library).
# The program lands in extrem_z_b200/compat/_build/extrem_main; the GPU tests
# run it and compare its fixed.bin with the library's own correction.
#   build_reference_main.sh <reference checkout>
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:?usage: build_reference_main.sh <reference checkout>}"
PKG="$(cd "$HERE/.." && pwd)"
OUT="$HERE/_build"
mkdir -p "$OUT"
test -f "$REF/main.cpp" && test -f "$REF/include/api/ExtreM.h"
test -f "$PKG/libExtreMz.so"
g++ -std=c++17 -O2 -fopenmp -w -I "$REF/include/api" "$REF/main.cpp" \
  -L "$PKG" -lExtreMz -Wl,-rpath,'$ORIGIN/../..' -o "$OUT/extrem_main"
echo "$OUT/extrem_main"
