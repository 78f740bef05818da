#!/bin/sh
# Builds the checker's copy of the reference (test infrastructure only).
#
# Compiles the unmodified single header src/polesitter.h from the reference
# checkout (by include path; nothing is copied) through oracle/ref_wrap.c into
#   oracle/_ref/libpsref.so         the reference's own flags
#                                   (CMakeLists.txt:37-46: -std=c99 -O3
#                                   -ffast-math -march=native) with
#                                   PS_MULTITHREADING; -march=native is pinned
#                                   to the AVX2+FMA ISA that x86 hosts take
#                                   (polesitter.h:182-185) so the binary runs
#                                   on any AVX2 host, this one or a GPU host.
#   oracle/_ref/libpsref_strict.so  same source, strict IEEE (-O2, no
#                                   fast-math, no FMA contraction): used to
#                                   show the fast-math build computes the same
#                                   Morton codes, order, tree and MAC decisions.
# Usage: oracle/build_ref.sh [reference_root]
#   (default: $PS_REFERENCE_ROOT, else the checkout beside this repository)
set -eu
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${1:-${PS_REFERENCE_ROOT:-$HERE/../../reference}}
OUT="$HERE/_ref"
if [ ! -f "$REF/src/polesitter.h" ]; then
  echo "reference header not found under $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
COMMON="-std=c99 -fPIC -shared -fvisibility=hidden -I$REF/src -mavx2 -mfma"
gcc $COMMON -O3 -ffast-math -o "$OUT/libpsref.so" "$HERE/ref_wrap.c" -lpthread -lm
gcc $COMMON -O2 -ffp-contract=off -o "$OUT/libpsref_strict.so" "$HERE/ref_wrap.c" -lpthread -lm
echo "built $OUT/libpsref.so $OUT/libpsref_strict.so"
