#!/usr/bin/env bash
# Compile the reference DoseCUDA CUDA extension (its own five .cu files,
# unmodified, read in place) for sm_100a into oracle/_ref/.
#
# The result is the reference's CPython module `dose_kernels`, used only as a
# checker: tests/golden/make_golden.py runs it on a B200 to produce golden
# fixtures, and `bench.py --impl reference` times it.  Nothing in the product
# imports it.  The reference's own CMake build is not used; this is the
# equivalent nvcc command line (separable compilation, as its
# DoseCUDA/dose_kernels/CMakeLists.txt requests).
#
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]   (default /root/reference)
set -euo pipefail
REF=${1:-/root/reference}
SRC="$REF/DoseCUDA/dose_kernels"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
if [ ! -d "$SRC" ]; then
    echo "build_ref: reference sources not found at $SRC (skipped)" >&2
    exit 0
fi
mkdir -p "$OUT/obj"
PY=${PYTHON:-python}
PYINC=$($PY -c 'import sysconfig; print(sysconfig.get_paths()["include"])')
NPINC=$($PY -c 'import numpy; print(numpy.get_include())')
SUFFIX=$($PY -c 'import sysconfig; print(sysconfig.get_config_var("EXT_SUFFIX"))')
NVCC=${NVCC:-nvcc}
FLAGS="-std=c++17 -O3 -rdc=true -Xcompiler -fPIC -gencode arch=compute_100a,code=sm_100a -lineinfo"
OBJS=()
for f in CudaClasses TextureClasses IMPTClasses IMRTClasses dosemodule; do
    $NVCC $FLAGS -I"$SRC" -I"$PYINC" -I"$NPINC" -c "$SRC/$f.cu" -o "$OUT/obj/$f.o"
    OBJS+=("$OUT/obj/$f.o")
done
$NVCC -shared -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC \
    "${OBJS[@]}" -o "$OUT/dose_kernels$SUFFIX" -lcudart
rm -rf "$OUT/obj"
echo "build_ref: wrote $OUT/dose_kernels$SUFFIX"
