#!/usr/bin/env bash
# Compiles the reference's own sources, where they lie, into oracle/_ref/ (git-ignored;
# travels to the GPU box with the other built files). Test and comparison infrastructure only.
#
#   REFERENCE=<checkout of the reference project> oracle/build_ref.sh
#
#   oracle/_ref/solution             the reference's original CUDA solution (src/solve.cu + src/main.cpp)
#   oracle/_ref/ordered_streaming    its best ranked entry (candidates/ordered-streaming/solve.cu + main.cpp)
#   oracle/_ref/caller_fused_strips  its fastest measured entry (candidates/caller-fused-strips/solve.cu + main.cpp)
#   oracle/_ref/harness_b200         the reference's unmodified harness src/main.cpp linked against this
#                                    repository's fherma_init/run/free (the package's libfherma_negacyclic.so,
#                                    found through its rpath): the drop-in
#
# The three reference solutions are built for sm_100a, each as its own CMakeLists.txt builds it
# (add_executable(solution main.cpp solve.cu), -O3, C++17, Threads, and the CUDA driver library
# for caller-fused-strips), without running CMake.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REPO="$(dirname "$HERE")"
OUT="$HERE/_ref"
if [ -z "${REFERENCE:-}" ]; then
    echo "REFERENCE is not set; keeping any prebuilt oracle/_ref" >&2
    exit 0
fi
if [ ! -f "$REFERENCE/src/solve.cu" ]; then
    echo "no reference sources under REFERENCE=$REFERENCE; keeping any prebuilt oracle/_ref" >&2
    exit 0
fi
mkdir -p "$OUT"
ARCH="-gencode arch=compute_100a,code=sm_100a"
nvcc -O3 -std=c++17 $ARCH -I"$REFERENCE/src" "$REFERENCE/src/solve.cu" "$REFERENCE/src/main.cpp" -o "$OUT/solution" &
CAND="$REFERENCE/candidates/ordered-streaming"
nvcc -O3 -std=c++17 $ARCH -I"$CAND" "$CAND/solve.cu" "$CAND/main.cpp" -o "$OUT/ordered_streaming" -lpthread &
CAND="$REFERENCE/candidates/caller-fused-strips"
nvcc -O3 -std=c++17 $ARCH -I"$CAND" "$CAND/solve.cu" "$CAND/main.cpp" -o "$OUT/caller_fused_strips" -lpthread -lcuda &
PKG="$REPO/fherma-polynomial-cuda_b200"
rm -f "$OUT/libnegacyclic.so" "$OUT/libfherma_negacyclic.so"  # older builds copied the library here
g++ -O2 -std=c++17 -include "$REFERENCE/src/fherma.h" -DFHERMA_TYPES_DEFINED -I"$REFERENCE/src" \
    "$REFERENCE/src/main.cpp" -o "$OUT/harness_b200" -L"$PKG" -lfherma_negacyclic \
    -Wl,-rpath,'$ORIGIN/../../fherma-polynomial-cuda_b200'
wait
echo "built $OUT/{solution,ordered_streaming,caller_fused_strips,harness_b200}"
