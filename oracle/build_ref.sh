#!/usr/bin/env bash
# Builds the reference's own FP32 CUDA solver (unmodified sources, read where
# they lie) into oracle/_ref/ with the reference's numeric flags
# (--use_fast_math -O3, CMakeLists.txt:277-298) retargeted to sm_100a:
#   oracle/_ref/libfvm_ref.so      src/solver.cu + oracle/ref_harness.cu
#   oracle/_ref/kernel_benchmark   src/solver.cu + src/test/kernel_benchmark.cu
#   oracle/_ref/libcmap_ref.so     the colour-table generators and the field
#                                  fragment shader of src/renderer.cpp, compiled
#                                  for the host by oracle/ref_colormap.py
# Test infrastructure only.  The reference checkout is $FVM_REFERENCE when
# set, else a directory named `reference` beside this repository; when
# neither holds the reference sources the script says so and does nothing
# (machines that only run the prebuilt files need no sources).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${FVM_REFERENCE:-$(cd "$HERE/../.." && pwd)/reference}"
OUT="$HERE/_ref"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
if [ ! -f "$REF/src/solver.cu" ]; then
    echo "build_ref: no reference sources at $REF (set FVM_REFERENCE to the checkout), skipping"
    exit 0
fi
mkdir -p "$OUT"
FLAGS="-std=c++17 -O3 --use_fast_math --expt-relaxed-constexpr -gencode arch=compute_100a,code=sm_100a -lineinfo"
if [ ! -f "$OUT/libfvm_ref.so" ] || [ "$HERE/ref_harness.cu" -nt "$OUT/libfvm_ref.so" ]; then
    "$NVCC" $FLAGS -Xcompiler -fPIC -shared -I"$REF/src/include" \
        "$REF/src/solver.cu" "$HERE/ref_harness.cu" -o "$OUT/libfvm_ref.so"
fi
if [ ! -f "$OUT/kernel_benchmark" ]; then
    "$NVCC" $FLAGS -I"$REF/src/include" "$REF/src/test/kernel_benchmark.cu" "$REF/src/solver.cu" \
        -o "$OUT/kernel_benchmark"
fi
# the renderer's colour tables and field shader as a host library (libcmap_ref.so)
if [ ! -f "$OUT/libcmap_ref.so" ] || [ "$HERE/ref_colormap.py" -nt "$OUT/libcmap_ref.so" ]; then
    "${PYTHON:-python3}" "$HERE/ref_colormap.py" "$REF" "$OUT"
fi
echo "build_ref: built $OUT"
