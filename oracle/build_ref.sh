#!/usr/bin/env bash
# Compile the reference's KISS FFT header (src/fftmpi/src/kissfft.h with
# ffttype.h, double precision) from the reference tree into oracle/_ref/ as a
# checker of the oracle's DFT.  Output only into oracle/_ref/ (git-ignored).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF=/root/reference/src/fftmpi/src
mkdir -p "$HERE/_ref"
g++ -O2 -fPIC -shared -I"$REF" -o "$HERE/_ref/libkissref.so" "$HERE/ref_kiss_shim.cpp"
