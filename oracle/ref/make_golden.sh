#!/bin/sh
# Writes tests/golden/reference_generator.txt from the reference's own
# generator (oracle/_ref/gen_golden, built by oracle/ref/Makefile from the
# reference tree; REF in the environment overrides the Makefile's default).
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REPO=$(cd "$HERE/../.." && pwd)
make -s -C "$HERE" all
if [ ! -x "$REPO/oracle/_ref/gen_golden" ]; then
  echo "make_golden.sh: oracle/_ref/gen_golden not built (reference tree absent); nothing written"
  exit 0
fi
mkdir -p "$REPO/tests/golden"
"$REPO/oracle/_ref/gen_golden" > "$REPO/tests/golden/reference_generator.txt"
echo "wrote $REPO/tests/golden/reference_generator.txt"
