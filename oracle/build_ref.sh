#!/usr/bin/env bash
# Compiles the reference's own CUDA sources, read in place from the reference
# checkout (never copied into the repository), plus the harnesses
# oracle/ref/ref_harness.cu (dose path) and oracle/ref/opt_harness.cu
# (optimizer) into oracle/_ref/libfdref.so for sm_100a.  Flags follow the
# reference build (CMakeLists.txt: -lineinfo -use_fast_math), with the
# architecture changed.  TEST INFRASTRUCTURE: golden fixtures and the
# reference-CUDA timings come from this library; the product never links it.
#
# The reference checkout is taken from $FD_REFERENCE_DIR, else the first
# argument, else the folder "reference" beside this repository.
#
# What stands in for absent dependencies:
# - oracle/ref/eigen_stub: the few Eigen types the optimizer's headers name
#   (Eigen is not installed); the reference's headers compile unmodified
#   against it;
# - oracle/ref/shim: Boost.Filesystem (-> std::filesystem), HDF5's C++ names
#   (doseDataSave only), and the program-options argument table (a registry
#   the harness fills).
#
# IMRTOptimize.cu mixes the GPU solver with Eigen-heavy host plumbing, so only
# its include block (lines 1-14) and the two Eigen-free solver bodies --
# BOO_IMRT_L2OneHalf_gpu_QL (lines 16-194) and polish_BOO_IMRT_gpu (lines
# 391-476) -- are compiled, extracted into oracle/_ref/gen/ at build time with
# #line markers.  The extraction checks each range's first and last line and
# stops if the checkout differs.  Every other file compiles whole.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${FD_REFERENCE_DIR:-${1:-$(cd "$HERE/../.." && pwd)/reference}}"
OUT="$HERE/_ref"
if [ ! -d "$REF/FastDoseLib" ] || [ ! -d "$REF/IMRTOpt" ]; then
    echo "reference checkout not found at $REF; skipping the reference build" >&2
    exit 0
fi
mkdir -p "$OUT/gen" "$OUT/obj"

OPT_SRC="$REF/IMRTOpt/src/IMRTOptimize.cu"
GEN="$OUT/gen/IMRTOptimize_solvers.cu"
SRCS=("$REF"/FastDoseLib/src/*.cu
      "$REF/IMRTOpt/src/IMRTBeamBundle.cu" "$REF/IMRTOpt/src/IMRTgeom.cu"
      "$REF/IMRTOpt/src/IMRTDoseMat.cu" "$REF/IMRTOpt/src/IMRTSparseMatEns.cu"
      "$REF/IMRTOpt/src/IMRTOptUtils.cu" "$REF/IMRTOpt/src/IMRTOptimize_var1.cu"
      "$GEN" "$HERE/ref/ref_harness.cu" "$HERE/ref/opt_harness.cu")

newest=0
for f in "$REF"/FastDoseLib/src/*.cu "$REF"/FastDoseLib/include/* "$REF"/IMRTOpt/include/* \
         "$REF"/IMRTOpt/src/*.cu "$HERE"/ref/*.cu "$HERE"/ref/shim/*.h "$HERE"/ref/eigen_stub/Eigen/* \
         "$HERE/build_ref.sh"; do
    [ -f "$f" ] || continue
    t=$(stat -c %Y "$f"); [ "$t" -gt "$newest" ] && newest=$t
done
if [ -f "$OUT/libfdref.so" ] && [ "$(stat -c %Y "$OUT/libfdref.so")" -ge "$newest" ]; then
    exit 0
fi

# ---- extract the solver bodies of IMRTOptimize.cu
expect() {  # expect <line> <prefix>
    local got
    got="$(sed -n "$1p" "$OPT_SRC")"
    case "$got" in
        "$2"*) ;;
        *) echo "build_ref.sh: $OPT_SRC:$1 is '$got', expected '$2...'" >&2; exit 1 ;;
    esac
}
expect 16 "bool IMRT::BOO_IMRT_L2OneHalf_gpu_QL"
expect 194 "}"
expect 391 "bool IMRT::polish_BOO_IMRT_gpu("
expect 476 "}"
{
    echo "#line 1 \"$OPT_SRC\""
    sed -n '1,194p' "$OPT_SRC"
    echo "#line 391 \"$OPT_SRC\""
    sed -n '391,476p' "$OPT_SRC"
} > "$GEN.tmp"
mv "$GEN.tmp" "$GEN"

FLAGS=(-O3 -std=c++17 -gencode arch=compute_100a,code=sm_100a -lineinfo -use_fast_math
       -Xcompiler -fPIC -w --diag-suppress 20012
       -I "$HERE/ref/eigen_stub" -I "$HERE/ref/shim" -I "$REF/FastDoseLib/include" -I "$REF/IMRTOpt/include")
OBJS=()
pids=()
i=0
for s in "${SRCS[@]}"; do
    o="$OUT/obj/$(printf '%02d' $i)_$(basename "$s").o"
    OBJS+=("$o")
    nvcc "${FLAGS[@]}" -c "$s" -o "$o" &
    pids+=($!)
    i=$((i + 1))
    if [ "${#pids[@]}" -ge 8 ]; then wait "${pids[0]}"; pids=("${pids[@]:1}"); fi
done
for p in "${pids[@]}"; do wait "$p"; done
nvcc -shared -gencode arch=compute_100a,code=sm_100a "${OBJS[@]}" -o "$OUT/libfdref.so.tmp" \
    -lcudart -lcusparse -lcublas -Xlinker --no-undefined
mv "$OUT/libfdref.so.tmp" "$OUT/libfdref.so"
echo "built $OUT/libfdref.so"
