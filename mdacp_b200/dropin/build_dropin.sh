#!/usr/bin/env bash
# Builds the MDACP drop-in: the reference's unchanged application layer
# (main, ProjectManager, the Benchmark/Collision/Langevin/... projects,
# configuration makers, Parameter, mout, Communicator, SimulationInfo,
# ParaInfo, MDRect -- compiled from the reference's own source files where
# they lie) linked against this directory's Variables / MeshList / PairList /
# ForceCalculator / observers / MDUnit / MDManager, which run the timestep on
# the GPU through libmdacp_b200.so.  CUTOFF_LENGTH is the reference's
# compile-time constant (include/mdconfig.h:31); one binary per cut-off:
#   mdacp_b200/dropin/_build/mdacp_rc25   mdacp_b200/dropin/_build/mdacp_rc30
# Usage: mdacp_b200/dropin/build_dropin.sh REFERENCE_ROOT   (or MDACP_REFERENCE=REFERENCE_ROOT)
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
PKG="$(cd "$HERE/.." && pwd)"
REPO="$(cd "$PKG/.." && pwd)"
REF="${1:-${MDACP_REFERENCE:-}}"
OUT="$HERE/_build"
if [ ! -f "$REF/src/main.cc" ]; then
  echo "build_dropin: reference sources not found at $REF" >&2
  exit 2
fi
[ -f "$PKG/libmdacp_b200.so" ] || make -C "$PKG/csrc"
mkdir -p "$OUT"
# the application layer of the reference, unchanged
APP=(main.cc projectmanager.cc benchmark.cc collision.cc langevin.cc confmaker.cc configtemp.cc
     phaseflow.cc rankine.cc burst.cc cavitation.cc parameter.cc mpistream.cc communicator.cc
     mdconfig.cc simulationinfo.cc parainfo.cc mdrect.cc)
SRCS=()
for f in "${APP[@]}"; do SRCS+=("$REF/src/$f"); done
for f in "$HERE"/src/*.cc; do SRCS+=("$f"); done
PSTL="$(dirname "$(echo '#include <algorithm>' | g++ -x c++ -std=c++17 -M - | tr ' ' '\n' | grep 'pstl/glue_algorithm_defs.h' | head -1)")"

build_one() {
  local tag="$1" rc="$2"
  local inc="$OUT/inc_rc$tag"
  mkdir -p "$inc"
  sed -E "s/^const double CUTOFF_LENGTH = [0-9.]+;/const double CUTOFF_LENGTH = $rc;/" \
    "$REF/include/mdconfig.h" > "$inc/mdconfig.h"
  grep -q "^const double CUTOFF_LENGTH = $rc;" "$inc/mdconfig.h"
  # "-I-": the drop-in headers (variables.h, meshlist.h, ...) shadow the
  # reference's even for includes from the reference's own include directory.
  g++ -O2 -fopenmp -std=c++17 -w -I- -I"$inc" -I"$HERE/include" -I"$REPO/include" -I"$REF/include" \
    -I"$PSTL" "${SRCS[@]}" -L"$PKG" -lmdacp_b200 -Wl,-rpath,'$ORIGIN/../..' \
    -o "$OUT/mdacp_rc$tag.tmp" 2> >(grep -v "obsolete option '-I-'" >&2)
  mv "$OUT/mdacp_rc$tag.tmp" "$OUT/mdacp_rc$tag"
}
pids=()
build_one 25 2.5 & pids+=($!)
build_one 30 3.0 & pids+=($!)
rc=0
for p in "${pids[@]}"; do wait "$p" || rc=1; done
[ "$rc" = 0 ] || { echo "build_dropin: build failed" >&2; exit 1; }
ls -l "$OUT"/mdacp_rc*
