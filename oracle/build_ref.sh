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
# Two builds of the same source:
#   libbaemm_refcl.so       strict IEEE (-O3): the parity checker;
#   libbaemm_refcl_fast.so  -ffast-math, the counterpart of the reference's own
#                           -cl-fast-relaxed-math (Helmholtz_OpenCL.hpp:77): the
#                           timed CPU baseline only.
# The reference root used is recorded in oracle/_ref/REFERENCE_ROOT, where the
# tests that read the reference's mesh files find it.
#
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]
#   (default: $BAEMM_REFERENCE, else /root/reference; skipped, exit 0, when the
#   reference tree is absent -- a GPU box uses the prebuilt libraries)
set -euo pipefail
REF="${1:-${BAEMM_REFERENCE:-/root/reference}}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
KDIR="$REF/src/Helmholtz_OpenCL"

if [ ! -d "$KDIR" ]; then
    echo "build_ref.sh: no reference tree at $REF; reference kernels not built" >&2
    exit 0
fi

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

build() {   # build <output name> <extra g++ flags...>
    local name="$1"; shift
    emit | g++ -x c++ -std=c++17 -O3 -march=x86-64-v3 -fopenmp -fPIC -shared "$@" \
        -Wno-unknown-pragmas -Wno-unused-value -Wno-unused-variable \
        -I"$HERE" - -o "$OUT/$name.tmp"
    mv "$OUT/$name.tmp" "$OUT/$name"
    echo "built $OUT/$name"
}
build libbaemm_refcl.so
build libbaemm_refcl_fast.so -ffast-math
printf '%s\n' "$(cd "$REF" && pwd)" > "$OUT/REFERENCE_ROOT"
