#!/usr/bin/env bash
# Builds xFluid's FluidSimulator from the reference sources into
# oracle/_ref/libxfsim.so, with oracle/sim_harness.cpp (the test harness that
# steps it).  TEST INFRASTRUCTURE ONLY.
#
#   XFLUID_REF  root of the reference checkout (default: a checkout named
#               `reference` beside this repository)
#
# Every source compiles as it lies in the reference except FluidSimulator.cpp,
# which is compiled from a copy in a temporary directory with one call
# rewritten: FluidSimulator.cpp:179 passes a temporary GridIndex3d to
# _addParticle(GridIndex3d&), which MSVC accepts and g++ rejects; the copy
# binds it to a named local first (same value, same particles).  The copy is
# deleted after the build and nothing is written into this repository but the
# library.  main.cpp (the reference's demo driver) is not compiled.
#
# A second library, oracle/_ref/libxfsim_dropin.so, builds the same simulator
# with this project's solver swapped in: the temporary copy of FluidSimulator.h
# also declares its pressure-solver member (FluidSimulator.h:215) as
# xfp::VariationalPressureSolver (include/xfp_solver.hpp) instead of xFluid's
# VariationalPressureSolver; FluidSimulator.cpp is the same copy as above.  It
# is stepped by oracle/sim_dropin_harness.cpp and links xfluid_b200/libxfp.so
# (built first; skipped with a note when it is absent).
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${XFLUID_REF:-$HERE/../../reference}"
SRC="$REF/xFluid/xFluid"
OUT="$HERE/_ref"
if [ ! -f "$SRC/FluidSimulator.cpp" ]; then
  echo "build_sim: reference sources not found under $SRC" >&2
  exit 2
fi
mkdir -p "$OUT"
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT
sed 's/_addParticle(GridIndex3d(i, j, k));/{ GridIndex3d g_(i, j, k); _addParticle(g_); }/' \
  "$SRC/FluidSimulator.cpp" > "$TMP/FluidSimulator.cpp"
if cmp -s "$SRC/FluidSimulator.cpp" "$TMP/FluidSimulator.cpp"; then
  echo "build_sim: expected call not found in FluidSimulator.cpp" >&2
  exit 3
fi
CXX="${XFREF_CXX:-/usr/bin/g++}"
SRCS=()
for f in "$SRC"/*.cpp "$SRC"/variationalpressure/*.cpp; do
  case "$(basename "$f")" in
    main.cpp|FluidSimulator.cpp) ;;
    *) SRCS+=("$f") ;;
  esac
done
"$CXX" -std=c++17 -O2 -fPIC -shared -ffp-contract=off -fno-fast-math -w \
  -include climits -include cmath -include cstring \
  -I"$SRC" -I"$SRC/variationalpressure" \
  "$TMP/FluidSimulator.cpp" "${SRCS[@]}" "$HERE/sim_harness.cpp" \
  -o "$OUT/libxfsim.so.tmp"
mv -f "$OUT/libxfsim.so.tmp" "$OUT/libxfsim.so"
echo "build_sim: $OUT/libxfsim.so"

REPO="$(cd "$HERE/.." && pwd)"
if [ ! -f "$REPO/xfluid_b200/libxfp.so" ]; then
  echo "build_sim: xfluid_b200/libxfp.so not built; skipping the drop-in simulator" >&2
  exit 0
fi
sed 's/^\([[:space:]]*\)VariationalPressureSolver _pressureSolver;/\1xfp::VariationalPressureSolver _pressureSolver;/' \
  "$SRC/FluidSimulator.h" > "$TMP/FluidSimulator.h"
if cmp -s "$SRC/FluidSimulator.h" "$TMP/FluidSimulator.h"; then
  echo "build_sim: expected member declaration not found in FluidSimulator.h" >&2
  exit 4
fi
# the class's header, after the reference's own includes
sed -i 's|^#include "fluidsource.h"|#include "fluidsource.h"\n#include "xfp_solver.hpp"|' "$TMP/FluidSimulator.h"
grep -q 'xfp_solver.hpp' "$TMP/FluidSimulator.h" || { echo "build_sim: include point not found" >&2; exit 5; }
"$CXX" -std=c++17 -O2 -fPIC -shared -ffp-contract=off -fno-fast-math -w \
  -include climits -include cmath -include cstring \
  -I"$TMP" -I"$SRC" -I"$SRC/variationalpressure" -I"$REPO/include" \
  "$TMP/FluidSimulator.cpp" "${SRCS[@]}" "$HERE/sim_dropin_harness.cpp" \
  -L"$REPO/xfluid_b200" -lxfp -Wl,-rpath,'$ORIGIN/../../xfluid_b200' -Wl,-Bsymbolic \
  -o "$OUT/libxfsim_dropin.so.tmp"
mv -f "$OUT/libxfsim_dropin.so.tmp" "$OUT/libxfsim_dropin.so"
echo "build_sim: $OUT/libxfsim_dropin.so"
