#!/usr/bin/env bash
# Builds oracle/_ref/libtrav_dropin.so: oracle/dropin_harness.cpp (the
# reference's own GPU callers, compiled from its headers where they lie)
# linked against parallel-task1_b200/libtrav_b200.so in place of the
# reference's bellman_ford.cu / bfs.cu.  The reference root is the first
# argument or $REF_ROOT; without either, the existing build is kept.  Output
# goes only to oracle/_ref/ (git-ignored, shipped with the working tree).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF_ROOT="${1:-${REF_ROOT:-}}"
CUDA_HOME="${CUDA_HOME:-/usr/local/cuda}"
PKG="$(cd "$HERE/../parallel-task1_b200" && pwd)"
OUT="$HERE/_ref"
if [ -z "$REF_ROOT" ] || [ ! -d "$REF_ROOT/algorithm" ]; then
  echo "build_dropin: no reference sources given (argument or REF_ROOT); keeping existing $OUT" >&2
  exit 0
fi
if [ ! -f "$PKG/libtrav_b200.so" ]; then
  echo "build_dropin: $PKG/libtrav_b200.so is not built yet" >&2
  exit 1
fi
mkdir -p "$OUT"
# Same reference compile switches as build_ref.sh; the reference's
# architectures.h already defines __USE_GPU__, so the GPU members are
# compiled and their wrapper calls bind to libtrav_b200.so.
g++ -O2 -w -std=c++11 -fopenmp -fpermissive -fPIC -shared \
    -include cstdint -include algorithm -include cfloat \
    -I"$REF_ROOT" -I"$CUDA_HOME/include" \
    "$HERE/dropin_harness.cpp" -o "$OUT/libtrav_dropin.so.tmp" \
    -L"$PKG" -ltrav_b200 -Wl,-rpath,"\$ORIGIN/../../parallel-task1_b200" \
    -L"$CUDA_HOME/lib64" -lcudart
mv "$OUT/libtrav_dropin.so.tmp" "$OUT/libtrav_dropin.so"
echo "build_dropin: wrote $OUT/libtrav_dropin.so"
