#!/bin/sh
# Compile the reference's own header-only PME math from the reference tree
# (never copied into this repository) into oracle/_ref/libref_pme.so.
# Test infrastructure: the oracle's restatement is checked against it.
# Usage: oracle/ref_build.sh REFERENCE_ROOT
set -e
here=$(cd "$(dirname "$0")" && pwd)
if [ $# -lt 1 ]; then
    echo "usage: $0 REFERENCE_ROOT (the Atomiverse source tree)" >&2
    exit 2
fi
ref=$1
if [ ! -f "$ref/include/atomiverse/cpu/longrange/pme_spline.h" ]; then
    echo "reference tree not found at $ref; skipping" >&2
    exit 0
fi
mkdir -p "$here/_ref"
g++ -std=c++20 -O2 -ffp-contract=off -fPIC -shared \
    -I "$here/ref_shim" -I "$ref/include" \
    "$here/ref_pme_wrap.cpp" -o "$here/_ref/libref_pme.so"
echo "built $here/_ref/libref_pme.so"
