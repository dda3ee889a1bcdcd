#!/bin/sh
# Builds the CPU oracle (test infrastructure only) next to its source.
# No multiply-add contraction: the oracle's arithmetic is plain IEEE double.
set -e
cd "$(dirname "$0")"
g++ -O2 -fopenmp -ffp-contract=off -fno-fast-math -fPIC -shared -Wall -o liboracle.so pg_oracle.cpp
