#!/bin/sh
# Builds the CPU oracle (the restatement in bq_oracle.c) into oracle/_build/.
# Test infrastructure only.
set -e
here="$(cd "$(dirname "$0")" && pwd)"
mkdir -p "$here/_build"
gcc -O2 -std=c11 -fPIC -shared -ffp-contract=off -fno-fast-math -Wall -Wno-misleading-indentation \
    -o "$here/_build/liboracle.so" "$here/bq_oracle.c" -lm
