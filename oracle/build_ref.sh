#!/usr/bin/env bash
# Builds oracle/_ref/libddref.so: oracle/ref_shim.cpp compiled against the reference
# solver's headers where they lie (REF_DIR/src, default /root/reference/src). The
# reference's own build system is not used and none of its sources are copied.
# Test infrastructure only (the checker), never linked by the product.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF_DIR="${REF_DIR:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF_DIR/src/dd.h" ]; then
  echo "build_ref: $REF_DIR/src/dd.h not found; reference oracle not built" >&2
  exit 3
fi
mkdir -p "$OUT"
g++ -O3 -std=c++17 -march=x86-64-v3 -pthread -fPIC -shared -I"$REF_DIR/src" \
  -o "$OUT/libddref.so.tmp" "$HERE/ref_shim.cpp"
mv "$OUT/libddref.so.tmp" "$OUT/libddref.so"
echo "built $OUT/libddref.so"
