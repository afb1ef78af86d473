#!/usr/bin/env bash
# Compiles the reference's own CUDA sources, in place under the reference
# checkout, into oracle/_ref/refdriver (test infrastructure; git-ignored).
#
# The reference's CMake build (sm_35, find_package(MPI REQUIRED)) is bypassed:
# nvcc is called directly for sm_100a with -rdc=true (the reference relies on
# separable compilation for int_log2, src/dequeue.cu:4), with two
# project-written shims on the include path (a single-rank mpi.h and a
# libmorton interleave, both under oracle/ref_shims/) and CUDA's own CUB
# (CCCL 2.8) in place of the empty cub submodule. Flags otherwise mirror a
# release build of the reference (-O3 -DNDEBUG, --expt-relaxed-constexpr).
#
# Usage: oracle/build_ref.sh [reference_root]
#   The reference checkout is the argument, else $SHAPEX_REFERENCE_ROOT; there
#   is no built-in default. Without either, a prebuilt refdriver is kept.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${SHAPEX_REFERENCE_ROOT:-}}"
OUT="$HERE/_ref"
if [ -z "$REF" ]; then
    echo "no reference checkout given (argument or SHAPEX_REFERENCE_ROOT); keeping any prebuilt $OUT" >&2
    exit 0
fi
SRC="$REF/src"
if [ ! -d "$SRC" ]; then
    echo "reference sources not found at $SRC; keeping any prebuilt $OUT" >&2
    exit 0
fi
mkdir -p "$OUT/obj"
NVCC="${NVCC:-nvcc}"
FLAGS=(-std=c++17 -O3 -DNDEBUG -gencode arch=compute_100a,code=sm_100a --expt-relaxed-constexpr -rdc=true
       -I"$HERE/ref_shims" -I"$SRC" -ccbin /usr/bin/g++)
objs=()
for f in MortonUtils RadixTree Octree dequeue CudaCommon; do
    "$NVCC" "${FLAGS[@]}" -c "$SRC/$f.cu" -o "$OUT/obj/$f.o"
    objs+=("$OUT/obj/$f.o")
done
"$NVCC" "${FLAGS[@]}" -c "$HERE/ref_driver.cu" -o "$OUT/obj/ref_driver.o"
objs+=("$OUT/obj/ref_driver.o")
"$NVCC" -gencode arch=compute_100a,code=sm_100a -rdc=true -ccbin /usr/bin/g++ "${objs[@]}" \
    -o "$OUT/refdriver" -lcusolver -lcublas
rm -rf "$OUT/obj"
echo "built $OUT/refdriver"
