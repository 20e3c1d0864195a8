#!/usr/bin/env bash
# Oracle test infrastructure (not product code).
#
# Builds the product's lightmetrica plugin (lightmetrica_b200/plugin/
# plugin.gpu.cpp) the way the reference builds its plugins
# (plugin/plugin.embree/CMakeLists.txt: the plugin source plus the
# reference's plugin.common.cpp, LM_USE_SINGLE_PRECISION), against the
# reference headers where they lie and this directory's stand-ins, linked to
# the float reference build (oracle/_ref/liblmref_f.so, the "application")
# and to liblmgpu.so. Output: oracle/_ref/plugin.gpu.so. -Bsymbolic keeps the
# plugin's own plugin registry (plugin.common.cpp) inside the plugin.
#
# Usage: oracle/build_plugin.sh [REFERENCE_ROOT]   (default: $LM_REFERENCE_ROOT)
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
ROOT="$(dirname "$HERE")"
REF="${1:-${LM_REFERENCE_ROOT:-}}"
if [ -z "$REF" ]; then
  echo "no reference tree: pass REFERENCE_ROOT or set LM_REFERENCE_ROOT" >&2
  exit 2
fi
OUT="$HERE/_ref"
if [ ! -d "$REF/src/liblightmetrica" ] || [ ! -f "$OUT/liblmref_f.so" ] || [ ! -f "$ROOT/lightmetrica_b200/_lib/liblmgpu.so" ]; then
  echo "reference tree, oracle/_ref/liblmref_f.so or liblmgpu.so missing; skipping plugin.gpu.so" >&2
  exit 0
fi
CXX="${LMREF_CXX:-/usr/bin/g++}"
FLAGS=(-std=c++14 -O2 -msse4.2 -mno-fma -fPIC -w -fno-gnu-unique
       -include cstdint -include stdexcept -include cstring -include cmath
       -I"$HERE/shim" -I"$REF/include" -I"$REF/src/liblightmetrica" -I"$REF/pch" -I"$ROOT/include"
       -DLM_USE_SINGLE_PRECISION -DLM_PLUGIN_EXPORTS -DNDEBUG)
mkdir -p "$OUT/obj_plugin"
"$CXX" "${FLAGS[@]}" -c "$ROOT/lightmetrica_b200/plugin/plugin.gpu.cpp" -o "$OUT/obj_plugin/plugin.gpu.o"
"$CXX" "${FLAGS[@]}" -c "$REF/src/liblightmetrica/plugin.common.cpp" -o "$OUT/obj_plugin/plugin.common.o"
"$CXX" -shared -Wl,-Bsymbolic -o "$OUT/plugin.gpu.so" "$OUT/obj_plugin/plugin.gpu.o" "$OUT/obj_plugin/plugin.common.o" \
    -L"$OUT" -l:liblmref_f.so -L"$ROOT/lightmetrica_b200/_lib" -l:liblmgpu.so \
    -Wl,-rpath,'$ORIGIN' -Wl,-rpath,'$ORIGIN/../../lightmetrica_b200/_lib' -lpthread
echo "built $OUT/plugin.gpu.so"
