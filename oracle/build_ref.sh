#!/usr/bin/env bash
# Compiles the reference's own sources (jcapriot/lifted src/, unmodified,
# read where they lie) against the Highway stand-in in oracle/hwy_shim, plus
# the C entry points in oracle/ref_capi.cpp, into oracle/_ref/.
#
# The result is a checker and the timed CPU baseline, never part of the GPU
# library.  Outputs (git-ignored, but they travel with the tree):
#   oracle/_ref/liblifted_ref_scalar.so   one lane   (bit-stable checker)
#   oracle/_ref/liblifted_ref_avx2.so     32-byte vectors, x86-64-v3
#   oracle/_ref/liblifted_ref_avx512.so   64-byte vectors, x86-64-v4
#
# Usage: oracle/build_ref.sh [reference_root]
# The reference checkout is the argument, else $LIFTED_REFERENCE, else a
# checkout named "reference" beside this repository.  Skips quietly (exit 0)
# when the reference tree is absent.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${LIFTED_REFERENCE:-$HERE/../../reference}}"
SRC="$REF/src"
OUT="$HERE/_ref"
if [ ! -f "$SRC/lifted.hpp" ]; then
  echo "build_ref: reference sources not found at $SRC; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
CXX="${CXX:-g++}"
# Same language mode and defines as the reference's meson build
# (meson.build:8-9,24-27; src/meson.build:31).
COMMON=(-std=c++20 -O3 -fPIC -DLIFTED_PTHREADS -DNDEBUG
        -I "$HERE/hwy_shim" -I "$SRC" -w)
REF_TUS=(lifted-float.cpp lifted-double.cpp lifted-sep-float.cpp lifted-sep-double.cpp)

# objects outside the tree (only the linked libraries sit in oracle/_ref)
OBJ="${LIFTED_BUILD_DIR:-${TMPDIR:-/tmp}/lifted_b200_build}/ref"
build_variant() {
  local name="$1" bytes="$2" arch="$3"
  local dir="$OBJ/obj_$name"
  mkdir -p "$dir"
  local objs=()
  local pids=()
  for tu in "${REF_TUS[@]}"; do
    local o="$dir/${tu%.cpp}.o"
    objs+=("$o")
    if [ ! -f "$o" ] || [ "$SRC/$tu" -nt "$o" ] || [ "$HERE/hwy_shim/hwy/highway.h" -nt "$o" ]; then
      "$CXX" "${COMMON[@]}" -fno-rtti $arch -DSHIM_VEC_BYTES="$bytes" -c "$SRC/$tu" -o "$o" &
      pids+=($!)
    fi
  done
  local wo="$dir/ref_capi.o"
  objs+=("$wo")
  if [ ! -f "$wo" ] || [ "$HERE/ref_capi.cpp" -nt "$wo" ] || [ "$HERE/hwy_shim/hwy/highway.h" -nt "$wo" ]; then
    "$CXX" "${COMMON[@]}" $arch -DSHIM_VEC_BYTES="$bytes" -c "$HERE/ref_capi.cpp" -o "$wo" &
    pids+=($!)
  fi
  for p in "${pids[@]}"; do wait "$p"; done
  "$CXX" -shared -o "$OUT/liblifted_ref_$name.so" "${objs[@]}" -lpthread
}

build_variant scalar 0 "-march=x86-64-v3" &
P1=$!
build_variant avx2 32 "-march=x86-64-v3" &
P2=$!
build_variant avx512 64 "-march=x86-64-v4" &
P3=$!
wait $P1 $P2 $P3
echo "build_ref: built $(ls "$OUT"/*.so | wc -l) libraries in $OUT"
