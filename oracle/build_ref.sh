#!/bin/sh
# TEST INFRASTRUCTURE ONLY.
#
# Compiles the reference (GFTEvolver) from its own sources where they lie,
# with g++ directly (its CMake build is not used), into two binaries:
#   oracle/_ref/ref32  -- the reference as shipped (float storage, -O3 like its Release build)
#   oracle/_ref/ref64  -- the same sources with float -> double (FP64-storage oracle)
# Both replace the reference's main.cpp with oracle/ref_harness.cpp and read
# their configuration from $GFT_REF_WORKDIR (oracle/ref_shim.h).  Outputs go to
# oracle/_ref/ only.
#
# Usage: sh oracle/build_ref.sh [REFERENCE_DIR]   (default /root/reference)
set -eu

HERE=$(cd "$(dirname "$0")" && pwd)
REF=${1:-${GFT_REFERENCE_DIR:-/root/reference}}
OUT="$HERE/_ref"
CXX=${CXX:-g++}

if [ ! -f "$REF/Core/Source/Lattice.cpp" ]; then
    echo "build_ref: reference sources not found under $REF" >&2
    exit 2
fi

MODULES="Core Potentials Gradients WilsonLoops InitialConditions BoundaryConditions Analysers"
INC=""
for m in $MODULES; do INC="$INC -I$REF/$m/Header"; done

mkdir -p "$OUT"
JOBS=$(nproc 2>/dev/null || echo 4)

for v in 32 64; do
    OBJ="$OUT/obj$v"
    mkdir -p "$OBJ"
    EXTRA=""
    if [ "$v" = 64 ]; then EXTRA="-DGFT_REF_FP64"; fi
    : > "$OBJ/cmds.txt"
    for m in $MODULES; do
        for src in "$REF/$m/Source/"*.cpp; do
            b=$(basename "$src" .cpp)
            echo "$CXX -std=c++17 -O3 -ffp-contract=off -w -include $HERE/ref_shim.h -DGFT_REF_MODULE=$m $EXTRA $INC -c $src -o $OBJ/${m}_$b.o" >> "$OBJ/cmds.txt"
        done
    done
    echo "$CXX -std=c++17 -O3 -ffp-contract=off -w -include $HERE/ref_shim.h $EXTRA $INC -c $HERE/ref_harness.cpp -o $OBJ/harness.o" >> "$OBJ/cmds.txt"
    tr '\n' '\0' < "$OBJ/cmds.txt" | xargs -0 -n1 -P "$JOBS" sh -c
    $CXX -o "$OUT/ref$v" "$OBJ"/*.o
done
echo "build_ref: built $OUT/ref32 $OUT/ref64"
