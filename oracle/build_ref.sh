#!/bin/sh
# Compiles the reference library's own code paths, directly from the
# unmodified reference sources, into oracle/_ref/.
#   sh oracle/build_ref.sh <reference source tree>   (or REF=<tree> sh ...)
# Without a tree (or where it has no cuBQL/ directory) the existing
# oracle/_ref is kept.  Test / baseline infrastructure only; nothing from the
# reference is copied into this repository.
#   libref_cpu.so  cpuBuilder + host findClosest/findKNN/triangles (g++)
#   libref_gpu.so  gpuBuilder, radixBuilder, rebinRadixBuilder and the
#                  per-thread query device functions, for sm_100a (nvcc)
# Both are built with FMA contraction as each compiler does by default for
# that code: g++ on x86-64 (no -mfma) emits none, nvcc contracts.
set -e
REF="${1:-${REF:-}}"
if [ -z "$REF" ]; then
  echo "no reference source tree given; keeping existing oracle/_ref" >&2
  exit 0
fi
here="$(cd "$(dirname "$0")" && pwd)"
if [ ! -d "$REF/cuBQL" ]; then
  echo "reference sources not found at $REF; keeping existing oracle/_ref" >&2
  exit 0
fi
mkdir -p "$here/_ref"
g++ -std=c++17 -O2 -fPIC -shared -I"$REF" -w -o "$here/_ref/libref_cpu.so" "$here/ref_cpu.cpp" -lpthread
/usr/local/cuda/bin/nvcc -std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC -shared \
    -I"$REF" -w -o "$here/_ref/libref_gpu.so" "$here/ref_gpu.cu"
# drop-in check: the reference's types and query kernel over libbq trees
/usr/local/cuda/bin/nvcc -std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC -shared \
    -I"$REF" -I"$here/../include" -w -o "$here/_ref/libref_shim.so" "$here/ref_shim.cu" \
    -L"$here/../cubql_b200" -lbq -Xlinker -rpath -Xlinker '$ORIGIN/../../cubql_b200'
