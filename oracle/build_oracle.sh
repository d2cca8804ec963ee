#!/bin/sh
# Builds the oracle restatement (test infrastructure) into oracle/_build/.
# Plain -O2 with no -march: no FMA contraction, like the reference built by ref.mk.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
mkdir -p "$HERE/_build"
/usr/bin/gcc -O2 -std=c99 -D_GNU_SOURCE -fPIC -shared -Wall -Wextra -Wno-unused-parameter -Wno-maybe-uninitialized -Wno-alloc-size-larger-than \
    "$HERE/xtoracle.c" "$HERE/lbvh_cpu.c" -o "$HERE/_build/libxtoracle.so" -lm
