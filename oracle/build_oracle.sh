#!/usr/bin/env bash
# Oracle test infrastructure (not product code): builds the plain-C
# restatement into oracle/liblmoracle.so. No FP contraction, so every float
# operation rounds separately as in the reference's float SSE build.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
CC_BIN="${LMORACLE_CC:-/usr/bin/gcc}"
"$CC_BIN" -std=c99 -O2 -fPIC -shared -ffp-contract=off -fno-fast-math -fexcess-precision=standard \
  -o "$HERE/liblmoracle.so" "$HERE/lmoracle.c" "$HERE/lmoracle_pt.c" -lm
echo "built $HERE/liblmoracle.so"
