#!/usr/bin/env bash
# Builds the reference xFluid pressure solvers (variational and normal),
# unmodified, from their own sources
# into oracle/_ref/libxfref.so, together with oracle/ref_harness.cpp (the test
# harness that binds it).  TEST INFRASTRUCTURE ONLY.
#
#   XFLUID_REF  root of the reference checkout (default: a checkout named
#               `reference` beside this repository)
#
# g++ needs <climits>/<cmath> force-included: variationalpressure/util.h uses
# UINT_MAX and the math functions without including their headers (the
# reference targets MSVC).  FP contraction is off so the x86-64 build rounds
# every multiply and add separately, as the reference's own build does.
# OpenMP is on, as in the reference's project (its applyPressure loop is an
# omp parallel for); the loop's iterations are independent, so results do not
# depend on the thread count.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${XFLUID_REF:-$HERE/../../reference}"
SRC="$REF/xFluid/xFluid"
OUT="$HERE/_ref"
if [ ! -f "$SRC/variationalpressure/variational_pressuresolver.cpp" ]; then
  echo "build_ref: reference sources not found under $SRC" >&2
  exit 2
fi
mkdir -p "$OUT"
# The system g++ (not $CXX): the library must share the process's libstdc++.
CXX="${XFREF_CXX:-/usr/bin/g++}"
"$CXX" -std=c++17 -O2 -fPIC -shared -ffp-contract=off -fno-fast-math -fopenmp -w \
  -include climits -include cmath \
  -I"$SRC" -I"$SRC/variationalpressure" \
  "$SRC/variationalpressure/variational_pressuresolver.cpp" \
  "$SRC/pressuresolver.cpp" \
  "$SRC/xfluidutil.cpp" \
  "$HERE/ref_harness.cpp" \
  -o "$OUT/libxfref.so.tmp"
mv -f "$OUT/libxfref.so.tmp" "$OUT/libxfref.so"
echo "build_ref: $OUT/libxfref.so"
