#!/usr/bin/env bash
# ORACLE TEST INFRASTRUCTURE -- not part of the product.
#
# Compiles the reference's own OpenCL kernel sources as C++ (through
# cl_shim.h, block_size == 1) into oracle/_ref/libbaemm_refcl.so.
#   src/Helmholtz_OpenCL/BoundaryOperatorKernel.cl
#   src/Helmholtz_OpenCL/FarFieldOperatorKernel.cl
#   src/Helmholtz_OpenCL/HerglotzWaveKernel.cl
#   src/Helmholtz_OpenCL/NearFieldOperatorKernel.cl
# Each .cl file is a C++ raw-string literal: its first line `R"(` and last line
# `)"` are stripped and the remainder is streamed to g++ on stdin, so no copy of
# the reference source is written anywhere.  One namespace per k_chunk_size in
# {1,2,4,8,16,32,64} (the #define of StringManipulation.hpp:11).
#
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]   (default /root/reference)
set -euo pipefail
REF="${1:-${BAEMM_REFERENCE:-/root/reference}}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
KDIR="$REF/src/Helmholtz_OpenCL"

for f in BoundaryOperatorKernel FarFieldOperatorKernel HerglotzWaveKernel NearFieldOperatorKernel; do
    if [ ! -f "$KDIR/$f.cl" ]; then
        echo "build_ref.sh: $KDIR/$f.cl not found" >&2
        exit 1
    fi
done
mkdir -p "$OUT"

emit() {
    echo '#include "cl_shim.h"'
    for K in 1 2 4 8 16 32 64; do
        echo "namespace refcl_k$K {"
        echo "#define k_chunk_size $K"
        for pair in bok:BoundaryOperatorKernel ffk:FarFieldOperatorKernel hwk:HerglotzWaveKernel \
                    nfk:NearFieldOperatorKernel; do
            ns="${pair%%:*}"; f="${pair#*:}"
            echo "namespace $ns {"
            echo "#line 2 \"$f.cl\""
            sed '1d;$d' "$KDIR/$f.cl"
            echo "} // namespace $ns"
        done
        echo "#undef k_chunk_size"
        echo "} // namespace refcl_k$K"
    done
    echo '#include "cl_shim_driver.h"'
}

emit | g++ -x c++ -std=c++17 -O3 -march=x86-64-v3 -fopenmp -fPIC -shared \
    -Wno-unknown-pragmas -Wno-unused-value -Wno-unused-variable \
    -I"$HERE" - -o "$OUT/libbaemm_refcl.so.tmp"
mv "$OUT/libbaemm_refcl.so.tmp" "$OUT/libbaemm_refcl.so"
echo "built $OUT/libbaemm_refcl.so"
