#!/usr/bin/env bash
# Builds the CPU restatement (oracle/icp_oracle.c) into oracle/_build/libicp_oracle.so.
# Test infrastructure only: the product never loads this library.
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
mkdir -p "$here/_build"
gcc -std=c11 -O2 -fno-fast-math -ffp-contract=off -fPIC -shared \
    "$here/icp_oracle.c" -lm -o "$here/_build/libicp_oracle.so"
echo "built $here/_build/libicp_oracle.so"
