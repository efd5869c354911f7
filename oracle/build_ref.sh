#!/bin/sh
# Builds the reference's own CPU implementation (trotter-suzuki-mpi 1.6.2,
# read in place from its source tree, never copied) together with
# oracle/ref_driver.cpp into oracle/_ref/.  Test infrastructure only.
#
#   libtsref.so       -O2 -fopenmp               parity oracle (no FMA contraction
#                                                 without -march, as in a plain build)
#   libtsref_fast.so  -Ofast -march=x86-64-v3     the reference's own optimisation
#                     -fopenmp                    flags (configure.ac:37 uses -Ofast
#                                                 -march=native; x86-64-v3 keeps the
#                                                 binary runnable on another host CPU)
#   libtsref_gpu.so   nvcc -DCUDA -O2, sm_100a    adds the reference's CUDA kernel
#
# Usage: oracle/build_ref.sh [--optional] [reference_root]
#   reference_root defaults to $TS_REFERENCE_ROOT, else /root/reference (where
#   the reference is mounted read-only beside this repository); with
#   --optional a missing source tree is not an error (nothing is built).
set -eu
OPTIONAL=0
if [ "${1:-}" = "--optional" ]; then
    OPTIONAL=1
    shift
fi
REF=${1:-${TS_REFERENCE_ROOT:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
SRC="$REF/src"
if [ ! -f "$SRC/cpukernel.cpp" ]; then
    if [ "$OPTIONAL" = 1 ]; then
        echo "reference sources not found under $SRC: oracle/_ref not rebuilt"
        exit 0
    fi
    echo "reference sources not found under $SRC" >&2
    exit 1
fi
mkdir -p "$OUT"
FILES="$SRC/common.cpp $SRC/cpukernel.cpp $SRC/cpucartesian.cpp $SRC/cpucylindrical.cpp $SRC/model.cpp $SRC/solver.cpp $HERE/ref_driver.cpp"
CXX=${TSREF_CXX:-g++}
$CXX -O2 -fopenmp -fPIC -shared -w -I"$SRC" $FILES -o "$OUT/libtsref.so.tmp"
mv "$OUT/libtsref.so.tmp" "$OUT/libtsref.so"
$CXX -Ofast -march=x86-64-v3 -fopenmp -fPIC -shared -w -I"$SRC" $FILES -o "$OUT/libtsref_fast.so.tmp"
mv "$OUT/libtsref_fast.so.tmp" "$OUT/libtsref_fast.so"
# libtsref_gpu.so: the same sources plus the reference's own CUDA kernel
# (CC2Kernel, src/gpukernel.cu + src/gpucartesian.cu, selected by
# kernel_type "gpu"), -DCUDA as the reference's configure sets it, for sm_100a.
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
if [ -x "$NVCC" ]; then
    "$NVCC" -DCUDA -O2 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC,-fopenmp \
        -shared -w -I"$SRC" $FILES "$SRC/gpukernel.cu" "$SRC/gpucartesian.cu" -lcublas -lgomp \
        -o "$OUT/libtsref_gpu.so.tmp"
    mv "$OUT/libtsref_gpu.so.tmp" "$OUT/libtsref_gpu.so"
    echo "built $OUT/libtsref_gpu.so"
fi
echo "built $OUT/libtsref.so $OUT/libtsref_fast.so"
