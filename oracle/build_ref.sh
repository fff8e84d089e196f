#!/bin/sh
# Builds the reference's own block-ILU(0) ordering routines (test infrastructure) from the
# reference tree into oracle/_ref/.  Usage: sh oracle/build_ref.sh [reference root]
# (default: $EXASIM_REF)
set -e
REF=${1:-$EXASIM_REF}
[ -n "$REF" ] || { echo "give the reference root as an argument or in EXASIM_REF" >&2; exit 2; }
HERE=$(cd "$(dirname "$0")" && pwd)
mkdir -p "$HERE/_ref"
g++ -O2 -std=c++17 -fPIC -shared -w -DREF_CPUIMPL="\"$REF/backend/Common/cpuimpl.h\"" \
    "$HERE/ref_bilu0_shim.cpp" -o "$HERE/_ref/libref_bilu0.so"
