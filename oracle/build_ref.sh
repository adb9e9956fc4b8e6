#!/usr/bin/env bash
# Builds oracle/_ref/libddref.so: oracle/ref_shim.cpp compiled against the reference
# solver's headers where they lie (REF_DIR/src, default /root/reference/src). The
# reference's own build system is not used and none of its sources are copied.
# Test infrastructure only (the checker), never linked by the product.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF_DIR="${REF_DIR:-/root/reference}"
OUT="$HERE/_ref"
if [ "${1:-}" = "--where" ]; then  # prints the reference tree this recipe reads
  echo "$REF_DIR"
  exit 0
fi
if [ ! -f "$REF_DIR/src/dd.h" ]; then
  echo "build_ref: $REF_DIR/src/dd.h not found; reference oracle not built" >&2
  exit 3
fi
mkdir -p "$OUT"
g++ -O3 -std=c++17 -march=x86-64-v3 -pthread -fPIC -shared -I"$REF_DIR/src" \
  -o "$OUT/libddref.so.tmp" "$HERE/ref_shim.cpp"
mv "$OUT/libddref.so.tmp" "$OUT/libddref.so"
echo "built $OUT/libddref.so"
# The same with the reference's 12-byte signature entries (-DDD_TT_SIG, src/dd.h:74-85).
g++ -O3 -std=c++17 -march=x86-64-v3 -pthread -fPIC -shared -DDD_TT_SIG -I"$REF_DIR/src" \
  -o "$OUT/libddref_sig.so.tmp" "$HERE/ref_shim.cpp"
mv "$OUT/libddref_sig.so.tmp" "$OUT/libddref_sig.so"
echo "built $OUT/libddref_sig.so"
g++ -O3 -std=c++17 -march=x86-64-v3 -pthread -DWITH_REF -I"$REF_DIR/src" \
  -o "$OUT/cpu_window.tmp" "$HERE/cpu_window.cpp"
mv "$OUT/cpu_window.tmp" "$OUT/cpu_window"
echo "built $OUT/cpu_window"
# The reference's own GPU batch driver (gpu/gpu_main.cu), for sm_100a: a timing baseline
# of its wavefront kernel on the same GPU (run with WAVE=1 and CHECK=0).
if command -v nvcc > /dev/null && [ -f "$REF_DIR/gpu/gpu_main.cu" ]; then
  nvcc -O3 -std=c++17 -gencode arch=compute_100a,code=sm_100a -I"$REF_DIR/src" \
    -o "$OUT/dd_gpu_ref.tmp" "$REF_DIR/gpu/gpu_main.cu"
  mv "$OUT/dd_gpu_ref.tmp" "$OUT/dd_gpu_ref"
  echo "built $OUT/dd_gpu_ref"
fi
