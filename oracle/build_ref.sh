#!/usr/bin/env bash
# Builds the reference's own code, where it lies in the reference checkout and
# without copying it, into oracle/_ref.  Test infrastructure: the checker and
# the CPU baseline.
#
#   REF_ROOT   reference checkout (default: a directory named "reference"
#              beside the repository's parent directory)
#
# 1. _ref/libtvl1_ref.so: the sequential TV-L1 (src/tvl1/sequential).
#   -include ref_shim/tvl1_decl.hpp   replaces tvl1.hpp (run-time MAX_ITERATIONS,
#                                     public members; see that header)
#   -I ref_shim                       mkl.h stand-in (BLAS-1 loops)
#   -ffp-contract=off                 no fused multiply-add: IEEE single/double
#                                     arithmetic exactly as written
#   -fopenmp                          the reference's own OpenMP pragmas
#
# 2. _ref/libhslk_ref.so and _ref/libhslk_ref_stock.so: the reference's
#    Horn-Schunck kernels (src/hs/cuda/kernels/*.cuh, included by
#    ref_gpu_harness.cu) and Lucas-Kanade sources (src/lk/cuda/lucaskanade.cu,
#    kernels/kernels.cu) for sm_100a.  The first is built with -fmad=false
#    (every product and sum rounded as written, the library's own arithmetic
#    contract); the second with the reference's CMake flags (-O3, nvcc's
#    default contraction into fused multiply-adds).
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF_ROOT="${REF_ROOT:-$HERE/../../reference}"
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

NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
HS="$REF_ROOT/src/hs/cuda"
LK="$REF_ROOT/src/lk/cuda"
if [ ! -x "$NVCC" ] || [ ! -f "$HS/kernels/solverKernel.cuh" ] || [ ! -f "$LK/lucaskanade.cu" ]; then
    echo "build_ref: nvcc or the HS/LK CUDA sources missing; skipping the GPU kernels" >&2
    exit 0
fi
build_gpu() {  # $1 = output name, rest = extra nvcc flags
    local name="$1"; shift
    local tmp="$OUT/.obj_$name"
    mkdir -p "$tmp"
    local common=(-gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -w
                  -Xcompiler -fPIC -ccbin "$CXX" "$@")
    "$NVCC" "${common[@]}" -I "$HS" -I "$LK" -c "$HERE/ref_gpu_harness.cu" -o "$tmp/h.o"
    "$NVCC" "${common[@]}" -c "$LK/lucaskanade.cu" -o "$tmp/lk.o"
    "$NVCC" "${common[@]}" -c "$LK/kernels/kernels.cu" -o "$tmp/k.o"
    "$NVCC" -gencode arch=compute_100a,code=sm_100a -shared -cudart static -ccbin "$CXX" \
        -o "$OUT/$name.tmp" "$tmp/h.o" "$tmp/lk.o" "$tmp/k.o"
    mv "$OUT/$name.tmp" "$OUT/$name"
    rm -f "$tmp/h.o" "$tmp/lk.o" "$tmp/k.o"
    rmdir "$tmp"
    echo "build_ref: built $OUT/$name"
}
build_gpu libhslk_ref.so -fmad=false
build_gpu libhslk_ref_stock.so
