#!/bin/sh
# Builds the reference's own block-ILU(0) ordering routines (test infrastructure) from the
# reference tree into oracle/_ref/.  Usage: sh oracle/build_ref.sh [reference root]
set -e
REF=${1:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
mkdir -p "$HERE/_ref"
g++ -O2 -std=c++17 -fPIC -shared -w -DREF_CPUIMPL="\"$REF/backend/Common/cpuimpl.h\"" \
    "$HERE/ref_bilu0_shim.cpp" -o "$HERE/_ref/libref_bilu0.so"
