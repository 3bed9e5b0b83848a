#!/bin/sh
# ORACLE -- builds the reference's packer kernels from the reference sources
# (read where they lie, never copied) into oracle/_ref/libref_pack.so.
# Needs the reference tree (TEMPI_REFERENCE, else the checkout this recipe was
# written against); without it the recipe does nothing and exits 0.  The
# built .so then travels with the repository.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${TEMPI_REFERENCE:-/root/reference}
[ -f "$REF/include/pack_kernels.cuh" ] || { echo "reference sources not found at $REF"; exit 0; }
mkdir -p "$HERE/_ref"
/usr/local/cuda/bin/nvcc -O3 -std=c++14 -gencode arch=compute_100a,code=sm_100a \
  -Xcompiler -fPIC -shared -w -I"$REF/include" -DNDEBUG \
  -o "$HERE/_ref/libref_pack.so" "$HERE/ref_kernels.cu"
echo "built $HERE/_ref/libref_pack.so"
