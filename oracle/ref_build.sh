#!/usr/bin/env bash
# Builds the reference apo GPU library from its own sources, exactly as its CMake target
# compiles them (nvcc, --use_fast_math, relocatable device code, extended lambdas), for
# sm_100a, and links it with oracle/ref_driver.cu. Three binaries come out:
#   oracle/_ref/apo_ref_driver       default `apo` target (FP64 Real)
#   oracle/_ref/apo_ref_driver_fp32  `apo-fp32` target (-DAPO_REAL_SIZE=4)
#   oracle/_ref/apo_ref_contrib      the contributing-nearest study (oracle/ref_contrib.cu)
# The only file not taken from the reference is oracle/ref_shim/fmt/*, a logging stub
# for the missing `fmt` submodule. Nothing here is copied into the repository; the
# reference sources are read where they lie. Outputs go to oracle/_ref/ only.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${APO_REFERENCE_ROOT:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -d "$REF/apo/src/gpu" ]; then
    echo "reference sources not found at $REF; skipping the reference build" >&2
    exit 0
fi
mkdir -p "$OUT"
NVCC="${NVCC:-nvcc}"
SOURCES=(
    "$REF/apo/src/gpu/algorithm.cu"
    "$REF/apo/src/gpu/lbvh.cu"
    "$REF/apo/src/gpu/memory.cu"
    "$REF/apo/src/gpu/benchmark.cu"
    "$REF/apo/src/gpu/algorithm.cpp"
    "$REF/apo/src/core/utils.cpp"
    "$HERE/ref_driver.cu"
)
FLAGS=(-std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a -lineinfo --use_fast_math
       -rdc=true --extended-lambda -Xcudafe "--diag_suppress=1215 --diag_suppress=20012 --diag_suppress=20050"
       -I "$REF/apo/include" -I "$REF/apo/extern/cuda_helper" -I "$HERE/ref_shim" -w)
build() {
    local name="$1"; shift
    local obj="$OUT/obj_$name"
    mkdir -p "$obj"
    local objects=()
    for src in "${SOURCES[@]}"; do
        local o="$obj/$(basename "$src").o"
        "$NVCC" "${FLAGS[@]}" "$@" -x cu -dc "$src" -o "$o"
        objects+=("$o")
    done
    "$NVCC" -gencode arch=compute_100a,code=sm_100a -rdc=true "${objects[@]}" -o "$OUT/$name"
    rm -rf "$obj"
}
build apo_ref_driver &
build apo_ref_driver_fp32 -DAPO_REAL_SIZE=4 &
# the contributing-nearest study's labels, through oracle/ref_contrib.cu (its harness source is
# included where it lies; its own headers under app/ are found there too)
CONTRIB_SRC="$REF/app/benchmarks/benchmark_contributing_nearest.cu"
if [ -f "$CONTRIB_SRC" ]; then
    SOURCES[${#SOURCES[@]}-1]="$HERE/ref_contrib.cu"
    build apo_ref_contrib -DAPO_CONTRIB_SOURCE="\"$CONTRIB_SRC\"" -I "$REF/app" &
fi
wait
echo "reference drivers in $OUT"
