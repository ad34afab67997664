#!/bin/sh
# Test infrastructure: compile the reference's own C sources, where they lie,
# into oracle/_ref/ (never copied into this repository):
#   oracle/_ref/p3m            the reference CLI binary (main.c + Makefile:15 OBJECTS)
#   oracle/_ref/libp3mref.so   the same objects + ref_harness.c, for ctypes
# FFTW3 and GSL are absent from this image; the FFTW/GSL API subsets the
# reference calls come from oracle/shim (the oracle's own DFT restatement and
# a published MT19937).  Flags follow the reference Makefile:1-4, plus -fPIC.
# Usage: sh oracle/build_ref.sh <reference_dir>   (or P3M_REFERENCE_DIR set)
set -e
REF=${1:-$P3M_REFERENCE_DIR}
[ -n "$REF" ] || { echo "usage: sh oracle/build_ref.sh <reference_dir>" >&2; exit 2; }
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
OBJ="$OUT/obj"
[ -f "$REF/main.c" ] || { echo "reference sources not found at $REF" >&2; exit 1; }
mkdir -p "$OBJ"
CC=${CC:-gcc}
CFLAGS="-O3 -march=native -DNDEBUG -DUSE_RESTRICT -std=c99 -fPIC -w"
INC="-I$HERE/shim -I$REF"
SRCS="sort generate_system window-functions charge-assign common error ewald interpol io p3m-common p3m-ik realpart p3m-ik-i p3m-ad p3m-ad-i p3m-ad-self-forces domain-decomposition statistics tuning p3m-ik-real parameters p3m-ad-real q_ik q_ad q_ik_i q_ad_i find_error q p3m-ik-real-ns wtime"
pids=""
for s in $SRCS; do
  $CC $CFLAGS $INC -c "$REF/$s.c" -o "$OBJ/$s.o" &
  pids="$pids $!"
done
$CC $CFLAGS -I"$REF/tools" -c "$REF/tools/visit_writer.c" -o "$OBJ/visit_writer.o" &
pids="$pids $!"
$CC -O3 -std=c99 -fPIC -I"$HERE/shim" -c "$HERE/shim/fftw_shim.c" -o "$OBJ/fftw_shim.o" &
pids="$pids $!"
$CC -O3 -std=c99 -fPIC -I"$HERE/shim" -c "$HERE/shim/gsl_shim.c" -o "$OBJ/gsl_shim.o" &
pids="$pids $!"
$CC -O3 -std=c99 -fPIC -c "$HERE/dft.c" -o "$OBJ/dft.o" &
pids="$pids $!"
$CC $CFLAGS $INC -c "$HERE/ref_harness.c" -o "$OBJ/ref_harness.o" &
pids="$pids $!"
for p in $pids; do wait "$p"; done
LIBOBJS=""
for s in $SRCS visit_writer fftw_shim gsl_shim dft; do LIBOBJS="$LIBOBJS $OBJ/$s.o"; done
$CC $CFLAGS $INC -o "$OUT/p3m" "$REF/main.c" $LIBOBJS -lm
$CC -shared -o "$OUT/libp3mref.so" $LIBOBJS "$OBJ/ref_harness.o" -lm
echo "built $OUT/p3m and $OUT/libp3mref.so"
# The reference with the p3mg-backed method tables (p3m-standalone_b200/binding),
# compiled against the reference's own headers and linked with libp3mg.so
# (built first by p3m-standalone_b200/build.py): oracle/_ref/libp3mref_gpu.so
PKG="$HERE/../p3m-standalone_b200"
if [ -f "$PKG/libp3mg.so" ]; then
  BINC="-I$PKG/binding -I$HERE/../include"
  $CC $CFLAGS $INC $BINC -c "$PKG/binding/p3m-gpu.c" -o "$OBJ/p3m-gpu.o"
  $CC $CFLAGS $INC $BINC -c "$HERE/ref_binding_harness.c" -o "$OBJ/ref_binding_harness.o"
  $CC -shared -o "$OUT/libp3mref_gpu.so" $LIBOBJS "$OBJ/p3m-gpu.o" "$OBJ/ref_binding_harness.o" \
    -L"$PKG" -lp3mg -Wl,-rpath,'$ORIGIN/../../p3m-standalone_b200' -lm
  echo "built $OUT/libp3mref_gpu.so"
fi
