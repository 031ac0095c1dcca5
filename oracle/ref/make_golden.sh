#!/bin/sh
# Compiles the reference's generator sources, unchanged, from the read-only
# reference tree (REF, default /root/reference) into oracle/_ref/ and writes
# the golden vectors to tests/golden/reference_generator.txt (BUILD_ONLY=1:
# compile only).
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REPO=$(cd "$HERE/../.." && pwd)
REF=${REF:-/root/reference}
OUT="$REPO/oracle/_ref"
mkdir -p "$OUT" "$REPO/tests/golden"
# The driver includes "../generator/graph_generator.hpp"; give it a sibling
# directory of the reference's generator through a symlink tree in _ref.
rm -rf "$OUT/tree"
mkdir -p "$OUT/tree/driver"
ln -s "$REF/generator" "$OUT/tree/generator"
ln -s "$REF/mpi" "$OUT/tree/mpi"
cp "$HERE/gen_golden.cc" "$OUT/tree/driver/gen_golden.cc"
gcc -O2 -c -I"$HERE/stub" -I"$REF/generator" "$REF/generator/splittable_mrg.c" -o "$OUT/splittable_mrg.o"
g++ -O2 -std=gnu++14 -fopenmp -I"$HERE/stub" -I"$REF/generator" "$OUT/tree/driver/gen_golden.cc" \
    "$OUT/splittable_mrg.o" -o "$OUT/gen_golden"
[ "${BUILD_ONLY:-0}" = 1 ] && exit 0
"$OUT/gen_golden" > "$REPO/tests/golden/reference_generator.txt"
echo "wrote $REPO/tests/golden/reference_generator.txt"
