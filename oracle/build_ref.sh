#!/usr/bin/env bash
# Builds oracle/_ref/libtvl1_ref.so from the reference's sequential TV-L1
# sources where they lie (src/tvl1/sequential under the reference checkout),
# without copying them.  Test infrastructure: the checker and the CPU baseline.
#
#   REF_ROOT   reference checkout (default /root/reference)
#
# Flags:
#   -include ref_shim/tvl1_decl.hpp   replaces tvl1.hpp (run-time MAX_ITERATIONS,
#                                     public members; see that header)
#   -I ref_shim                       mkl.h stand-in (BLAS-1 loops)
#   -ffp-contract=off                 no fused multiply-add: IEEE single/double
#                                     arithmetic exactly as written
#   -fopenmp                          the reference's own OpenMP pragmas
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF_ROOT="${REF_ROOT:-/root/reference}"
SRC="$REF_ROOT/src/tvl1/sequential"
OUT="$HERE/_ref"
if [ ! -f "$SRC/tvl1.cpp" ]; then
    echo "build_ref: reference sources not found under $SRC; skipping" >&2
    exit 0
fi
mkdir -p "$OUT"
# The system g++ ships libgomp; a $CXX from another prefix may not.
CXX="${ORACLE_CXX:-/usr/bin/g++}"
[ -x "$CXX" ] || CXX=g++
FLAGS=(-std=gnu++17 -O3 -fopenmp -ffp-contract=off -fPIC -w
       -include "$HERE/ref_shim/tvl1_decl.hpp" -I "$HERE/ref_shim" -I "$HERE")
"$CXX" "${FLAGS[@]}" -shared -o "$OUT/libtvl1_ref.so.tmp" \
    "$SRC/tvl1.cpp" "$SRC/mask/mask.cpp" "$SRC/zoom/zoom.cpp" \
    "$SRC/bicubic_interpolation/bicubic_interpolation.cpp" \
    "$HERE/ref_harness.cpp"
mv "$OUT/libtvl1_ref.so.tmp" "$OUT/libtvl1_ref.so"
echo "build_ref: built $OUT/libtvl1_ref.so"
