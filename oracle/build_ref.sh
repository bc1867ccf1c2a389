#!/bin/bash
# Builds the reference's own FMM (mumairsadiq/exafmm-rd, variant 3dpp) from
# its unmodified sources where they lie, into oracle/_ref/ (git-ignored).
# Test infrastructure only.
#
#   bash oracle/build_ref.sh [--if-present] [/path/to/reference]
#
# The reference checkout is the argument, else $RTFMM_REFERENCE, else the
# read-only mount this recipe was written against.  --if-present exits 0
# without building when the sources are not there (a machine without the
# reference uses a prebuilt oracle/_ref).
#
# Missing third-party pieces and their stand-ins:
#   FFTW3 (not installed)  -> oracle/ref_shim/fftw3.h + fftw_shim.cpp (written here)
#   <cblas.h>              -> oracle/ref_shim/cblas.h (prototypes)
#   CBLAS + LAPACK dgesvd_ -> the OpenBLAS shared library bundled with the
#                             Python environment (opencv_python_headless.libs)
# The reference's type.h includes <cuda.h>/<cuda_runtime.h> for host/device
# qualifiers only, so the CUDA include directory is on the path.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
IF_PRESENT=0
if [ "${1:-}" = "--if-present" ]; then IF_PRESENT=1; shift; fi
REF="${1:-${RTFMM_REFERENCE:-/root/reference}}/3dpp"
OUT="$HERE/_ref"
if [ ! -d "$REF/src" ]; then
  if [ "$IF_PRESENT" = 1 ]; then echo "reference sources not found under $REF; oracle/_ref not rebuilt"; exit 0; fi
  echo "reference sources not found under $REF" >&2; exit 1
fi
BLAS="$(ls "$(python3 -c 'import site; print(site.getsitepackages()[0])')"/opencv_python_headless.libs/libopenblasp-*.so 2>/dev/null | head -1)"
[ -n "$BLAS" ] || { echo "OpenBLAS shared library not found" >&2; exit 1; }
mkdir -p "$OUT"
# the system compiler: its OpenMP runtime is installed (an alternative gcc on
# PATH may lack libgomp)
CXX="${RTFMM_REF_CXX:-/usr/bin/g++}"
FLAGS="-std=gnu++17 -O3 -march=native -fopenmp -w"
INC="-I$HERE/ref_shim -I$REF/include -I/usr/local/cuda/include"
objs=()
for src in "$REF"/src/*.cpp "$HERE"/ref_shim/fftw_shim.cpp "$HERE"/ref/rtfmm_ref_pass.cpp; do
  obj="$OUT/$(basename "$src" .cpp).o"
  $CXX $FLAGS $INC -c "$src" -o "$obj"
  objs+=("$obj")
done
LIBDIR="$(dirname "$BLAS")"
# OpenBLAS was built with gfortran; its runtime sits next to it
EXTRA="$(ls "$LIBDIR"/libgfortran-*.so* "$LIBDIR"/libquadmath-*.so* 2>/dev/null | tr '\n' ' ')"
$CXX $FLAGS -o "$OUT/rtfmm_ref_pass" "${objs[@]}" "$BLAS" $EXTRA -Wl,--disable-new-dtags,-rpath,"$LIBDIR"
rm -f "$OUT"/*.o
echo "built $OUT/rtfmm_ref_pass"
