#!/usr/bin/env bash
# Oracle test infrastructure (not product code).
#
# Compiles the reference's own hot-path sources, unmodified and where they lie
# in the reference tree, together with this directory's stand-ins
# (shim/, ref_stubs.cpp) and C harness (ref_harness.cpp, ref_render.cpp) into
#   oracle/_ref/liblmref_f.so   (Math::Float = float,  LM_USE_SINGLE_PRECISION)
#   oracle/_ref/liblmref_d.so   (Math::Float = double, LM_USE_DOUBLE_PRECISION)
# Flags follow the reference's CMakeLists.txt:300-313 for GCC (-msse4.2,
# -mno-fma) and its default Release build type (CMakeLists.txt:55-56, NDEBUG);
# the QBVH source needs -fno-strict-aliasing on GCC 13, without it
# it returns no hits. Nothing is written outside oracle/_ref.
#
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]   (default: $LM_REFERENCE_ROOT)
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${LM_REFERENCE_ROOT:-}}"
if [ -z "$REF" ]; then
  echo "no reference tree: pass REFERENCE_ROOT or set LM_REFERENCE_ROOT" >&2
  exit 2
fi
OUT="$HERE/_ref"
if [ ! -d "$REF/src/liblightmetrica" ]; then
  echo "reference tree not found at $REF; skipping oracle/_ref build" >&2
  exit 0
fi
mkdir -p "$OUT"
SRC="$REF/src/liblightmetrica"
CORE="scene.cpp scene.bvh.cpp scene.naive.cpp object.cpp align.cpp"
RENDER="pathtrace.cpp pathtrace.direct.cpp pathtrace.mis.cpp renderutils.cpp diffuse.cpp mirror.cpp \
        light.area.cpp light.env.const.cpp emittershape.sphere.cpp perspectivecamera.cpp \
        randomsampler.cpp standardmtrand.cpp sched.mt.cpp constanttexture.cpp hdrfilm.cpp bitmap.cpp"
# The system g++ (the one whose libgomp is installed); override with LMREF_CXX.
CXX="${LMREF_CXX:-/usr/bin/g++}"
# -fno-gnu-unique: the float and double builds are loaded into one process, and
# template statics (component registration) must stay per library.
COMMON=(-std=c++14 -O2 -msse4.2 -mno-fma -fPIC -fopenmp -w -fno-gnu-unique
        -include cstdint -include stdexcept -include cstring -include cmath
        -I"$HERE/shim" -I"$REF/include" -I"$SRC" -I"$REF/pch" -DLM_EXPORTS -DNDEBUG)

build_one() {  # $1 = f|d
  local tag="$1" prec objdir
  if [ "$tag" = f ]; then prec=-DLM_USE_SINGLE_PRECISION; else prec=-DLM_USE_DOUBLE_PRECISION; fi
  objdir="$OUT/obj_$tag"
  mkdir -p "$objdir"
  local objs=() pids=()
  for s in $CORE $RENDER; do
    "$CXX" "${COMMON[@]}" $prec -c "$SRC/$s" -o "$objdir/${s%.cpp}.o" & pids+=($!)
    objs+=("$objdir/${s%.cpp}.o")
  done
  if [ "$tag" = f ]; then
    "$CXX" "${COMMON[@]}" $prec -fno-strict-aliasing -c "$SRC/scene.qbvh.cpp" -o "$objdir/scene.qbvh.o" & pids+=($!)
    objs+=("$objdir/scene.qbvh.o")
  fi
  "$CXX" "${COMMON[@]}" $prec -c "$REF/plugin/plugin.diffusemirror/diffusemirror.cpp" -o "$objdir/diffusemirror.o" -DLM_PLUGIN_EXPORTS & pids+=($!)
  objs+=("$objdir/diffusemirror.o")
  for h in ref_stubs ref_harness ref_render; do
    "$CXX" "${COMMON[@]}" $prec -c "$HERE/$h.cpp" -o "$objdir/$h.o" & pids+=($!)
    objs+=("$objdir/$h.o")
  done
  for p in "${pids[@]}"; do wait "$p"; done
  "$CXX" -shared -fopenmp -o "$OUT/liblmref_$tag.so" "${objs[@]}" -lpthread
  echo "built $OUT/liblmref_$tag.so"
}

build_one f
build_one d
