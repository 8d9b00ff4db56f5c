#!/usr/bin/env bash
# Compile the reference's KISS FFT header (src/fftmpi/src/kissfft.h with
# ffttype.h, double precision) from a reference tree into oracle/_ref/ as a
# checker of the oracle's DFT.  Output only into oracle/_ref/ (git-ignored).
#
# Usage: oracle/build_ref.sh <reference tree>   (or MIMICA_REFERENCE_TREE=<tree>)
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
TREE="${1:-${MIMICA_REFERENCE_TREE:-}}"
if [ -z "$TREE" ]; then
    echo "usage: $0 <reference tree> (or set MIMICA_REFERENCE_TREE)" >&2
    exit 2
fi
REF="$TREE/src/fftmpi/src"
mkdir -p "$HERE/_ref"
g++ -O2 -fPIC -shared -I"$REF" -o "$HERE/_ref/libkissref.so" "$HERE/ref_kiss_shim.cpp"
