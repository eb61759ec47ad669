#!/usr/bin/env bash
# Compiles the reference's own sources, where they lie, into oracle/_ref/ (git-ignored;
# travels to the GPU box with the other built files). Test infrastructure only.
#
#   oracle/_ref/solution      the reference's original CUDA solution (src/solve.cu + src/main.cpp),
#                             built for sm_100a: a GPU cross-check at points it can initialise
#   oracle/_ref/harness_b200  the reference's unmodified harness src/main.cpp linked against this
#                             repository's fherma_init/run/free (libfherma_negacyclic.so): the drop-in
#
# Equivalent of the reference's CMake target (src/CMakeLists.txt: add_executable(solution main.cpp
# solve.cu), -O3, C++17) without running its build system.
set -euo pipefail
REFERENCE="${REFERENCE:-/root/reference}"
HERE="$(cd "$(dirname "$0")" && pwd)"
REPO="$(dirname "$HERE")"
OUT="$HERE/_ref"
if [ ! -f "$REFERENCE/src/solve.cu" ]; then
    echo "reference sources not present; keeping any prebuilt oracle/_ref" >&2
    exit 0
fi
mkdir -p "$OUT"
nvcc -O3 -std=c++17 -gencode arch=compute_100a,code=sm_100a -I"$REFERENCE/src" \
    "$REFERENCE/src/solve.cu" "$REFERENCE/src/main.cpp" -o "$OUT/solution"
PKG="$REPO/fherma-polynomial-cuda_b200"
cp "$PKG/libnegacyclic.so" "$PKG/libfherma_negacyclic.so" "$OUT/"
g++ -O2 -std=c++17 -include "$REFERENCE/src/fherma.h" -DFHERMA_TYPES_DEFINED -I"$REFERENCE/src" \
    "$REFERENCE/src/main.cpp" -o "$OUT/harness_b200" -L"$OUT" -lfherma_negacyclic -Wl,-rpath,'$ORIGIN'
echo "built $OUT/solution and $OUT/harness_b200"
