#!/bin/sh
# Builds the reference's own Solver (trotter-suzuki-mpi 1.6.2, sources read in
# place, never copied) with its GPU kernel class CC2Kernel implemented by
# cc2kernel_b200.cpp on libtsb200.so, into oracle/_ref/libtsref_b200.so,
# together with oracle/ref_driver.cpp (the tests' ctypes entry point).  The
# reference's src/gpukernel.cu and src/gpucartesian.cu are not compiled:
# kernel_type "gpu" of the unmodified Solver runs the B200 engine.
#
# Usage: build_with_reference.sh [--optional] [reference_root]
#   reference_root defaults to $TS_REFERENCE_ROOT, else /root/reference; with
#   --optional a missing source tree is not an error.  libtsb200.so must be
#   built first (python -m trottersuzuki_b200.build).
set -eu
OPTIONAL=0
if [ "${1:-}" = "--optional" ]; then
    OPTIONAL=1
    shift
fi
REF=${1:-${TS_REFERENCE_ROOT:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
PKG="$HERE/../trottersuzuki_b200"
PKG=$(cd "$PKG" && pwd)
REPO=$(cd "$HERE/../.." && pwd)
OUT="$REPO/oracle/_ref"
SRC="$REF/src"
if [ ! -f "$SRC/solver.cpp" ]; then
    if [ "$OPTIONAL" = 1 ]; then
        echo "reference sources not found under $SRC: libtsref_b200.so not rebuilt"
        exit 0
    fi
    echo "reference sources not found under $SRC" >&2
    exit 1
fi
if [ ! -f "$PKG/libtsb200.so" ]; then
    echo "build libtsb200.so first" >&2
    exit 1
fi
mkdir -p "$OUT"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
FILES="$SRC/common.cpp $SRC/cpukernel.cpp $SRC/cpucartesian.cpp $SRC/cpucylindrical.cpp $SRC/model.cpp $SRC/solver.cpp $REPO/oracle/ref_driver.cpp $HERE/cc2kernel_b200.cpp"
"$NVCC" -DCUDA -O2 -Wno-deprecated-gpu-targets -Xcompiler -fPIC,-fopenmp -shared -w -I"$SRC" -I"$REPO/include" $FILES \
    -L"$PKG" -ltsb200 -Xlinker -rpath,'$ORIGIN/../../trotter-suzuki-mpi_b200/trottersuzuki_b200' -lgomp -o "$OUT/libtsref_b200.so.tmp"
mv "$OUT/libtsref_b200.so.tmp" "$OUT/libtsref_b200.so"
echo "built $OUT/libtsref_b200.so"
