#!/bin/sh
# Test infrastructure: build the oracle restatement into oracle/liboracle.so.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
CC=${CC:-gcc}
$CC -O2 -std=c99 -fPIC -shared -o "$HERE/liboracle.so" "$HERE/p3m_oracle.c" "$HERE/dft.c" -lm
echo "built $HERE/liboracle.so"
