#!/usr/bin/env bash
# Builds oracle/_ref/libtrav_refgpu.so: the reference's own GPU path
# (algorithm/sssp/gpu/bellman_ford.cu and algorithm/bfs/gpu/bfs.cu, compiled
# unchanged from where they lie for sm_100a) with oracle/refgpu_harness.cpp,
# which drives its wrappers on a resident edge list.  The reference root is the
# first argument or $REF_ROOT; without either, the existing build is kept.
# Output goes only to oracle/_ref/ (git-ignored, shipped with the working tree).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF_ROOT="${1:-${REF_ROOT:-}}"
CUDA_HOME="${CUDA_HOME:-/usr/local/cuda}"
OUT="$HERE/_ref"
if [ -z "$REF_ROOT" ] || [ ! -d "$REF_ROOT/algorithm" ]; then
  echo "build_refgpu: no reference sources given (argument or REF_ROOT); keeping existing $OUT" >&2
  exit 0
fi
mkdir -p "$OUT/obj"
NVCC="$CUDA_HOME/bin/nvcc"
# The reference's .cu files use the `register` storage class, which C++17
# removed: compile them as C++14.  -w silences their old-style warnings.
# -Bsymbolic binds the harness to these objects even in a process that also
# loaded libtrav_b200.so, which exports the same wrapper symbols.
for f in algorithm/sssp/gpu/bellman_ford.cu algorithm/bfs/gpu/bfs.cu; do
  "$NVCC" -gencode arch=compute_100a,code=sm_100a -O3 -std=c++14 -w -Xcompiler -fPIC \
      -I"$REF_ROOT" -c "$REF_ROOT/$f" -o "$OUT/obj/$(basename "$f").o"
done
"$NVCC" -gencode arch=compute_100a,code=sm_100a -O2 -std=c++14 -Xcompiler -fPIC,-fopenmp -shared \
    "$HERE/refgpu_harness.cpp" "$OUT/obj/bellman_ford.cu.o" "$OUT/obj/bfs.cu.o" \
    -o "$OUT/libtrav_refgpu.so.tmp" -lgomp -lcudart -Xlinker -Bsymbolic
mv "$OUT/libtrav_refgpu.so.tmp" "$OUT/libtrav_refgpu.so"
echo "build_refgpu: wrote $OUT/libtrav_refgpu.so"
