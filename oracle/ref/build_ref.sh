#!/usr/bin/env bash
# Builds the reference MDACP CPU code (kohnakagawa/mdacp) from its own source
# files, where they lie, into oracle/_ref/ as a test oracle and timed CPU
# baseline.  Nothing is copied into the repository: the only generated input
# is oracle/_ref/inc_rcXX/mdconfig.h, the reference header with its
# compile-time CUTOFF_LENGTH (include/mdconfig.h:31) set to the cut-off the
# workload needs, which is how the reference is configured for another rc.
#
# Outputs (git-ignored; the tests and bench.py run the built binaries):
#   oracle/_ref/mdacp_rc25_plain  oracle/_ref/mdacp_rc30_plain   (-ffp-contract=off, SSE2: bit-exact oracle)
#   oracle/_ref/mdacp_rc25_avx2   oracle/_ref/mdacp_rc30_avx2    (-DAVX2 -mavx2 -mfma: timed CPU baseline)
#
# Usage: oracle/ref/build_ref.sh REFERENCE_ROOT   (or MDACP_REFERENCE=REFERENCE_ROOT)
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REPO="$(cd "$HERE/../.." && pwd)"
REF="${1:-${MDACP_REFERENCE:-}}"
OUT="$REPO/oracle/_ref"
if [ ! -f "$REF/src/mdmanager.cc" ]; then
  echo "build_ref: reference sources not found at $REF" >&2
  exit 2
fi
mkdir -p "$OUT"
# Every reference translation unit except the CUDA device query (the CPU
# build excludes it the same way, CMakeLists.txt:64-67).
SRCS=()
for f in "$REF"/src/*.cc; do
  case "$(basename "$f")" in
    device_info.cc) ;;
    *) SRCS+=("$f") ;;
  esac
done
SRCS+=("$HERE/ref_harness.cc")

# libstdc++'s parallel-algorithm headers include their siblings with quotes;
# with "-I-" their directory has to be named explicitly.
PSTL="$(dirname "$(echo '#include <algorithm>' | g++ -x c++ -std=c++17 -M - | tr ' ' '\n' | grep 'pstl/glue_algorithm_defs.h' | head -1)")"

build_one() {
  local tag="$1" rc="$2" flavour="$3"
  local inc="$OUT/inc_rc$tag"
  mkdir -p "$inc"
  sed -E "s/^const double CUTOFF_LENGTH = [0-9.]+;/const double CUTOFF_LENGTH = $rc;/" \
    "$REF/include/mdconfig.h" > "$inc/mdconfig.h"
  grep -q "^const double CUTOFF_LENGTH = $rc;" "$inc/mdconfig.h"
  local flags=(-O3 -fopenmp -std=c++17 -w)
  if [ "$flavour" = avx2 ]; then
    flags+=(-DAVX2 -mavx2 -mfma)
  else
    flags+=(-ffp-contract=off)
  fi
  # "-I-" stops the quote-include search in the including file's own
  # directory, so the generated mdconfig.h shadows the reference's copy.
  g++ "${flags[@]}" -I- -I"$inc" -I"$HERE" -I"$REF/include" -I"$PSTL" "${SRCS[@]}" \
    -o "$OUT/mdacp_rc${tag}_${flavour}.tmp" 2> >(grep -v "obsolete option '-I-'" >&2)
  mv "$OUT/mdacp_rc${tag}_${flavour}.tmp" "$OUT/mdacp_rc${tag}_${flavour}"
}

pids=()
build_one 25 2.5 plain & pids+=($!)
build_one 30 3.0 plain & pids+=($!)
build_one 25 2.5 avx2 & pids+=($!)
build_one 30 3.0 avx2 & pids+=($!)
rc=0
for p in "${pids[@]}"; do wait "$p" || rc=1; done
[ "$rc" = 0 ] || { echo "build_ref: a reference build failed" >&2; exit 1; }
ls -l "$OUT"/mdacp_rc*
