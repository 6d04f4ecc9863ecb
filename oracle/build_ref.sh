#!/usr/bin/env bash
# Compile the reference DoseCUDA CUDA extension (its own five .cu files,
# unmodified, read in place) for sm_100a into oracle/_ref/.
#
# The results are the reference's CPython module `dose_kernels` and a TERMA
# harness (libref_terma.so, oracle/ref_terma.cu), used only as checkers:
# tests/golden/make_golden.py ran the module on a B200 to produce the golden
# fixtures, the GPU tests compare against both, and `bench.py --impl
# reference` times the module when the pip-installed reference is absent.
# Nothing in the product imports them.  The reference's own CMake build is not used; this is the
# equivalent nvcc command line (separable compilation, as its
# DoseCUDA/dose_kernels/CMakeLists.txt requests).
#
# Usage: oracle/build_ref.sh REFERENCE_ROOT
#        (or DOSECUDA_REFERENCE=REFERENCE_ROOT oracle/build_ref.sh)
set -euo pipefail
REF=${1:-${DOSECUDA_REFERENCE:-}}
if [ -z "$REF" ]; then
    echo "build_ref: give the reference checkout as an argument or in DOSECUDA_REFERENCE" >&2
    exit 2
fi
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
# TERMA harness: the reference's ray-trace and TERMA kernels with their
# intermediate volumes handed back (oracle/ref_terma.cu), linked against the
# same reference objects.
$NVCC $FLAGS -I"$SRC" -c "$HERE/ref_terma.cu" -o "$OUT/obj/ref_terma.o"
$NVCC -shared -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC \
    "$OUT/obj/CudaClasses.o" "$OUT/obj/TextureClasses.o" "$OUT/obj/IMRTClasses.o" "$OUT/obj/ref_terma.o" \
    -o "$OUT/libref_terma.so" -lcudart
rm -rf "$OUT/obj"
echo "build_ref: wrote $OUT/dose_kernels$SUFFIX and $OUT/libref_terma.so"
