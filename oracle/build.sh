#!/bin/sh
# Builds the CPU checker (test infrastructure): oracle/liboracle.so.
# -ffp-contract=off keeps every a*b+c as two rounded operations, as the
# reference (Julia, no @fastmath) and the device build (-fmad=false) do.
set -e
here=$(cd "$(dirname "$0")" && pwd)
g++ -O2 -std=c++17 -fPIC -shared -fopenmp -ffp-contract=off -fno-fast-math \
    -o "$here/liboracle.so" "$here/cbm_oracle.cpp"
