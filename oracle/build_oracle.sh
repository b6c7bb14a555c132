#!/usr/bin/env bash
# ORACLE TEST INFRASTRUCTURE -- not part of the product.
# Builds the CPU restatement (baemm_oracle.cpp) into oracle/_build/liboracle.so.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
mkdir -p "$HERE/_build"
g++ -std=c++17 -O3 -march=x86-64-v3 -fopenmp -fcx-limited-range -fPIC -shared \
    "$HERE/baemm_oracle.cpp" -o "$HERE/_build/liboracle.so.tmp"
mv "$HERE/_build/liboracle.so.tmp" "$HERE/_build/liboracle.so"
echo "built $HERE/_build/liboracle.so"
