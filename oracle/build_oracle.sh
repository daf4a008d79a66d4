#!/bin/sh
# Builds the CPU oracle (test infrastructure) into oracle/_build/.
# -ffp-contract=off keeps a*b+c as two roundings, as the Fortran reference
# evaluates it on x86-64 without FMA contraction.
set -e
here=$(cd "$(dirname "$0")" && pwd)
mkdir -p "$here/_build"
gcc -O2 -std=c11 -fPIC -shared -ffp-contract=off -fno-fast-math -fopenmp \
    -o "$here/_build/libsph_oracle.so" "$here/sph_oracle.c" -lm
