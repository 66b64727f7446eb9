#!/usr/bin/env bash
# Builds oracle/_ref/libtrav_ref.so: oracle/ref_harness.cpp compiled against the
# reference library's headers where they lie.  The reference root is the first
# argument or $REF_ROOT; without either, the existing oracle/_ref is kept.
# Nothing is copied from the reference; the output goes only to oracle/_ref/
# (git-ignored, but shipped with the working tree so the CPU baseline can run
# where the reference sources are absent).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF_ROOT="${1:-${REF_ROOT:-}}"
CUDA_HOME="${CUDA_HOME:-/usr/local/cuda}"
OUT="$HERE/_ref"
if [ -z "$REF_ROOT" ] || [ ! -d "$REF_ROOT/algorithm" ]; then
  echo "build_ref: no reference sources given (argument or REF_ROOT); keeping existing $OUT" >&2
  exit 0
fi
mkdir -p "$OUT"
# The reference headers need <cstdint>, <algorithm> and <cfloat> injected and
# -fpermissive for pre-C++11 constructs; -I CUDA only for header lookups
# (no CUDA library is linked: the GPU methods are never instantiated).
g++ -O3 -w -std=c++11 -fopenmp -fpermissive -fPIC -shared \
    -include cstdint -include algorithm -include cfloat \
    -I"$REF_ROOT" -I"$CUDA_HOME/include" \
    "$HERE/ref_harness.cpp" -o "$OUT/libtrav_ref.so.tmp"
mv "$OUT/libtrav_ref.so.tmp" "$OUT/libtrav_ref.so"
echo "build_ref: wrote $OUT/libtrav_ref.so"
