#!/bin/sh
# Builds the oracle (test infrastructure only): the strict-IEEE CPU
# restatement of the polesitter tick in oracle/ps_oracle.c ->
# oracle/_build/libpsoracle.so.  -mavx2 gives it the AVX2 lane arithmetic of
# the reference's x86 P2P path; -ffp-contract=off and no fast-math keep every
# operation rounded as written.
set -eu
HERE=$(cd "$(dirname "$0")" && pwd)
mkdir -p "$HERE/_build"
gcc -std=c99 -O2 -ffp-contract=off -fno-fast-math -mavx2 -fPIC -shared \
    -fvisibility=hidden -o "$HERE/_build/libpsoracle.so" "$HERE/ps_oracle.c" -lm
echo "built $HERE/_build/libpsoracle.so"
