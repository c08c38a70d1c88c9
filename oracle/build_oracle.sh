#!/usr/bin/env bash
# Build recipe for oracle/_build/libcirrus_oracle.so, the CPU restatement of the reference's
# Poisson path (test infrastructure only).  -ffp-contract=off: the oracle spells out every
# fused multiply-add it mirrors with std::fma, so the compiler must not add others.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
mkdir -p "$HERE/_build"
"${CIRRUS_CXX:-g++}" -std=c++17 -O3 -mavx2 -mfma -ffp-contract=off -fopenmp -shared -fPIC -Wall -Wno-unused-function \
  -o "$HERE/_build/libcirrus_oracle.so.tmp" "$HERE/cirrus_oracle.cpp"
mv "$HERE/_build/libcirrus_oracle.so.tmp" "$HERE/_build/libcirrus_oracle.so"
echo "built $HERE/_build/libcirrus_oracle.so"
