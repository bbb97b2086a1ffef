#!/bin/sh
# Builds the CPU FP64 oracle (test infrastructure) into oracle/liblsd_oracle.so.
# -ffp-contract=off: keep every a*b+c as two roundings.
set -e
cd "$(dirname "$0")"
g++ -O3 -march=x86-64-v3 -fopenmp -ffp-contract=off -fPIC -shared -std=c++17 \
    -Wall -Wno-unused-function -o liblsd_oracle.so lsd_oracle.cpp
