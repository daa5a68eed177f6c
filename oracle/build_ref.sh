#!/usr/bin/env bash
# Builds oracle/_ref/libhplref.so from rocHPL's own sources, read in place from
# the reference tree (nothing is copied), through the shim in oracle/ref_shim/.
# Only matgen, pivot bookkeeping and the single-process row swap are built:
# the LU itself needs rocBLAS, MPI and HIP cooperative launches, so it is
# not buildable here.  Test infrastructure only.
#
#   oracle/build_ref.sh [REFERENCE_TREE]
#
# REFERENCE_TREE is the rocHPL checkout (the directory holding src/ and
# include/): the first argument, else $HPLB_REFERENCE, else /root/reference,
# where the build container mounts it.  Without it nothing is built.
set -euo pipefail
REF=${1:-${HPLB_REFERENCE:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
if [ ! -d "$REF/src" ]; then
  echo "build_ref: reference tree not found at $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
NVCC=${NVCC:-nvcc}
FLAGS="-O2 -std=c++17 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC -I$HERE/ref_shim -I$REF/include"
$NVCC $FLAGS -shared -o "$OUT/libhplref.so" \
  -x cu "$REF/src/matgen/HPL_pdrandmat_device.cpp" \
  -x cu "$REF/src/matgen/HPL_xjumpm.cpp" \
  -x cu "$REF/src/pgesv/HPL_pipid.cpp" \
  -x cu "$REF/src/pauxil/HPL_dlaswp00N_device.cpp" \
  -x cu "$HERE/ref_shim/ref_entry.cu"
echo "build_ref: wrote $OUT/libhplref.so"
