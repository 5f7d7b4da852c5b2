#!/usr/bin/env bash
# Builds the CPU oracle (a plain-C restatement of the reference algorithm,
# test infrastructure only) into oracle/_build/liblifted_oracle.so.
# -ffp-contract=off: the only fused multiply-adds are the explicit fma()
# calls that restate the reference's MulAdd/NegMulAdd.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
mkdir -p "$HERE/_build"
OUT="$HERE/_build/liblifted_oracle.so"
if [ -f "$OUT" ] && [ "$OUT" -nt "$HERE/lifted_oracle.c" ] && [ "$OUT" -nt "$HERE/lifted_oracle_impl.h" ] \
   && [ "$OUT" -nt "$HERE/lifted_oracle.h" ] && [ "$OUT" -nt "$HERE/../lifted_b200/csrc/wavelet_catalogue.inc" ]; then
  exit 0
fi
${CC:-gcc} -std=c11 -O2 -march=x86-64-v3 -ffp-contract=off -fPIC -shared -Wall -Wno-unused-function \
  -o "$OUT" "$HERE/lifted_oracle.c" -lm
