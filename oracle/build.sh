#!/usr/bin/env bash
# Builds the CPU oracle (test infrastructure): oracle/liborc.so from
# trav_oracle.c, then oracle/_ref/ from the reference sources when their root
# is given as the first argument or in $REF_ROOT (see build_ref.sh).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
gcc -O2 -std=c11 -fopenmp -fPIC -shared -ffp-contract=off \
    "$HERE/trav_oracle.c" -o "$HERE/liborc.so.tmp" -lm
mv "$HERE/liborc.so.tmp" "$HERE/liborc.so"
"$HERE/build_ref.sh" "$@"
