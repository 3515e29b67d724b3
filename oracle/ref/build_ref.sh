#!/bin/sh
# Compiles the reference's self-contained primitives (SFMT engine, Henyey-Greenstein phase, warps,
# smooth dielectric BSDF, thin lens) from their sources in place under the reference checkout,
# together with ref_shim.cpp, into oracle/_ref/libref_prims.so. Test infrastructure only: the
# library pins the oracle's restatements. Flags follow the reference's own optimised build
# (CMakeLists.txt:110-116). Usage: build_ref.sh [reference-root]; without the argument the checkout
# is $SIMPLER_REFERENCE_ROOT, else /root/reference.
set -e
REF=${1:-${SIMPLER_REFERENCE_ROOT:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/../_ref"
mkdir -p "$OUT"
SRC="$REF/renderer/src"
INC="$REF/renderer/include"
if [ ! -d "$SRC" ]; then
    echo "reference sources not found under $REF; skipping oracle/_ref" >&2
    exit 0
fi
g++ -std=c++17 -O3 -march=native -ffast-math -fno-math-errno -fPIC -shared \
    -DUSE_SFMT=1 -DNDEBUG=1 -DUSE_DOUBLE_PRECISION=0 -w \
    -I"$INC" \
    "$SRC/rng_sse.cpp" "$SRC/phase.cpp" "$SRC/warp.cpp" "$SRC/bsdf.cpp" "$SRC/lens.cpp" \
    "$HERE/ref_shim.cpp" -o "$OUT/libref_prims.so"
echo "built $OUT/libref_prims.so"
