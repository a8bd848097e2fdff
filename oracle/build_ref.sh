#!/usr/bin/env bash
# Builds the reference DrNUM library's CPU path (FP64) from its sources where
# they lie, as the checker for this repository's oracle restatement.
# Outputs go only to oracle/_ref/ (git-ignored).  Nothing is copied from the
# reference into the repository; one generated header (drnum.h with the
# single-precision switch at drnum.h:43 commented out) is written to
# oracle/_ref/gen/ and found first through gcc's -I- include split.
#
# usage: oracle/build_ref.sh [reference-root]      (default /root/reference)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REFROOT="${1:-${DRNUM_REFERENCE:-/root/reference}}"
LIB="$REFROOT/src/drnumlib"
OUT="$HERE/_ref"
if [ ! -f "$LIB/drnum.h" ]; then
  echo "build_ref.sh: reference sources not found under $REFROOT" >&2
  exit 2
fi
mkdir -p "$OUT/gen" "$OUT/obj"
sed -e 's|^#define DRNUM_SINGLE_PRECISION|/* FP64 oracle build */|' "$LIB/drnum.h" > "$OUT/gen/drnum.h"

SRCS="patch.cpp cartesianpatch.cpp patchgrid.cpp patchgroups.cpp geometrytools.cpp
      codestring.cpp transformation.cpp math/coordtransform.cpp math/coordtransformvv.cpp
      rungekutta.cpp timeintegration.cpp debug.cpp blockcfd.cpp cartesianraster.cpp
      raster.cpp structuredhexraster.cpp levelsetobject.cpp levelsetdefinition.cpp
      spherelevelset.cpp levelsetobjectbc.cpp"
CXX="${CXX:-g++}"
FLAGS="-O2 -std=c++14 -fPIC -fpermissive -w -fopenmp -DOPEN_MP -ffp-contract=off
       -include $HERE/ref_fp64_shim.h
       -I$OUT/gen -I$HERE/ref_stubs -I- -I$OUT/gen -I$HERE/ref_stubs -I$LIB -I$LIB/math -I$LIB/iterators
       -I$LIB/fluxes -I$LIB/reconstruction"
OBJS=""
pids=""
for s in $SRCS; do
  o="$OUT/obj/$(echo "$s" | tr '/' '_' | sed 's/\.cpp$/.o/')"
  OBJS="$OBJS $o"
  $CXX $FLAGS -c "$LIB/$s" -o "$o" &
  pids="$pids $!"
done
for p in $pids; do wait $p; done
$CXX $FLAGS -c "$HERE/ref_driver.cpp" -o "$OUT/obj/ref_driver.o"
$CXX -shared -o "$OUT/libdrnum_ref.so" $OBJS "$OUT/obj/ref_driver.o" -L/usr/lib/gcc/x86_64-linux-gnu/13 -lgomp -lpthread
echo "built $OUT/libdrnum_ref.so"

# The reference in its shipped precision (drnum.h:43 defines
# DRNUM_SINGLE_PRECISION: `real` is float), unchanged header, for the
# like-for-like CPU baseline of the FP32-bulk path (timing sessions only).
FLAGS32="-O2 -std=c++14 -fPIC -fpermissive -w -fopenmp -DOPEN_MP -ffp-contract=off
         -I$HERE/ref_stubs -I- -I$HERE/ref_stubs -I$LIB -I$LIB/math -I$LIB/iterators
         -I$LIB/fluxes -I$LIB/reconstruction"
mkdir -p "$OUT/obj32"
OBJS32=""
pids=""
for s in $SRCS; do
  o="$OUT/obj32/$(echo "$s" | tr '/' '_' | sed 's/\.cpp$/.o/')"
  OBJS32="$OBJS32 $o"
  $CXX $FLAGS32 -c "$LIB/$s" -o "$o" &
  pids="$pids $!"
done
for p in $pids; do wait $p; done
$CXX $FLAGS32 -c "$HERE/ref_driver.cpp" -o "$OUT/obj32/ref_driver.o"
$CXX -shared -o "$OUT/libdrnum_ref_f32.so" $OBJS32 "$OUT/obj32/ref_driver.o" -L/usr/lib/gcc/x86_64-linux-gnu/13 \
     -lgomp -lpthread
echo "built $OUT/libdrnum_ref_f32.so"

# A DrNUM application driving drnum_b200 through the C++ binding
# include/drnum_b200_iterator.h: the reference's own RungeKutta and PatchGrid
# (from libdrnum_ref.so) over the product library (built first by
# drnum_b200/build.py).
B200="$HERE/../drnum_b200"
if [ -f "$B200/libdrnum_b200.so" ]; then
  $CXX $FLAGS -I"$HERE/../include" -c "$HERE/ref_app_b200.cpp" -o "$OUT/obj/ref_app_b200.o"
  $CXX -shared -o "$OUT/libdrnum_refapp.so" "$OUT/obj/ref_app_b200.o" -L"$OUT" -ldrnum_ref -L"$B200" -ldrnum_b200 \
       -Wl,-rpath,'$ORIGIN' -Wl,-rpath,'$ORIGIN/../../drnum_b200' -L/usr/lib/gcc/x86_64-linux-gnu/13 -lgomp -lpthread
  echo "built $OUT/libdrnum_refapp.so"
fi

# The reference's flux functors compiled for the device (sm_100a) against this
# repository's generic functor stage.  nvcc has no -I- split, so the headers
# are reached through a tree of symbolic links to the reference's files in
# $OUT/tree, with the generated FP64 drnum.h in place of the original.
if command -v nvcc > /dev/null 2>&1; then
  rm -rf "$OUT/tree"
  mkdir -p "$OUT/tree"
  (cd "$LIB" && find . -type d) | while read -r d; do mkdir -p "$OUT/tree/$d"; done
  (cd "$LIB" && find . -type f -name '*.h') | while read -r f; do ln -s "$LIB/$f" "$OUT/tree/$f"; done
  rm -f "$OUT/tree/drnum.h"
  cp "$OUT/gen/drnum.h" "$OUT/tree/drnum.h"
  nvcc -gencode arch=compute_100a,code=sm_100a -O3 -std=c++14 -fmad=false -shared -Xcompiler -fPIC -w \
       -include "$HERE/ref_fp64_shim.h" -I"$OUT/tree" -I"$HERE/ref_stubs" -I"$OUT/tree/fluxes" \
       -I"$OUT/tree/reconstruction" -I"$OUT/tree/iterators" -I"$OUT/tree/math" -I"$HERE/../include" \
       "$HERE/ref_functor_stage.cu" -o "$OUT/libref_functor_stage.so"
  rm -rf "$OUT/tree"
  echo "built $OUT/libref_functor_stage.so"
fi
