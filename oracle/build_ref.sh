#!/usr/bin/env bash
# Compiles the reference's own CUDA sources (read in place from the reference
# checkout, never copied) plus oracle/ref/ref_harness.cu into
# oracle/_ref/libfdref.so for sm_100a.  Flags follow the reference build
# (CMakeLists.txt: -lineinfo -use_fast_math), with the architecture changed.
# The shims in oracle/ref/shim stand in for Boost.Filesystem, HDF5 and the
# Boost program-options argument table, which are not installed here.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${FD_REFERENCE_DIR:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -d "$REF/FastDoseLib" ]; then
    echo "reference checkout not found at $REF; skipping the reference build" >&2
    exit 0
fi
mkdir -p "$OUT"
SRCS=("$REF"/FastDoseLib/src/*.cu "$REF/IMRTOpt/src/IMRTBeamBundle.cu" "$REF/IMRTOpt/src/IMRTgeom.cu" "$HERE/ref/ref_harness.cu")
newest=0
for f in "${SRCS[@]}" "$HERE"/ref/shim/*.h "$HERE"/ref/shim/*.cuh "$HERE/build_ref.sh"; do
    t=$(stat -c %Y "$f"); [ "$t" -gt "$newest" ] && newest=$t
done
if [ -f "$OUT/libfdref.so" ] && [ "$(stat -c %Y "$OUT/libfdref.so")" -ge "$newest" ]; then
    exit 0
fi
nvcc -O3 -std=c++17 -gencode arch=compute_100a,code=sm_100a -lineinfo -use_fast_math \
    -Xcompiler -fPIC -shared -w \
    -I "$HERE/ref/shim" -I "$REF/FastDoseLib/include" -I "$REF/IMRTOpt/include" \
    "${SRCS[@]}" -o "$OUT/libfdref.so.tmp" -lcudart
mv "$OUT/libfdref.so.tmp" "$OUT/libfdref.so"
echo "built $OUT/libfdref.so"
