#!/bin/sh
# Builds oracle/_ref/libgrains_ref.so: the Grains3D reference (GRAINS_V1/Grains
# sources, compiled unmodified where they lie) + the single-rank MPI and
# Xerces DOM stand-ins in oracle/shim/ + the step harness ref_harness.cpp.
# TEST INFRASTRUCTURE: it pins the CPU restatement, produces the golden
# vectors under tests/golden/ and is the timed CPU baseline.  Outputs go to
# oracle/_ref/ only.
#
# Environment:
#   GRAINS_REFERENCE  root of the PacIFiC checkout (the directory holding
#                     GRAINS_V1/); default /root/reference
#   GRAINS_REF_CXX    C++ compiler (default g++)
#   JOBS              parallel compilations (default 8)
#
# Flags: -O3 as the reference's own GNU build (GRAINS_V1/Env/
# grains-OpenMPI-2.1.1-GNU-9.4.0.env.sh: -O3 without -march, so the x86-64
# baseline ISA and no FMA), plus -ffp-contract=off, which keeps every FP64
# expression rounded in source order (the restatement and the device FP64
# mode follow that order).  A change of flags rebuilds every object.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${GRAINS_REFERENCE:-/root/reference}/GRAINS_V1/Grains
OUT=$HERE/_ref
JOBS=${JOBS:-8}
[ -d "$REF" ] || { echo "reference tree not found: $REF (set GRAINS_REFERENCE)" >&2; exit 1; }
mkdir -p "$OUT/obj"
# the system g++ (its libstdc++ is the shared one Python processes load)
CXX=${GRAINS_REF_CXX:-g++}
FLAGS="-std=c++17 -O3 -ffp-contract=off -fPIC -w -I$HERE/shim -I$REF/include"
STAMP="$OUT/obj/flags"
if [ ! -f "$STAMP" ] || [ "$(cat "$STAMP")" != "$CXX $FLAGS" ]; then
  rm -f "$OUT"/obj/*.o
  echo "$CXX $FLAGS" > "$STAMP"
fi
SRCS=$(ls "$REF"/Base/src/*.cpp "$REF"/Component/src/*.cpp "$REF"/Geometry/src/*.cpp \
          "$REF"/TimeIntegration/src/*.cpp "$REF"/XML/src/*.cpp "$REF"/PostProcessing/src/*.cpp \
          "$REF"/Fluid/src/*.cpp)
for s in $SRCS "$HERE/shim/grains_shim.cpp" "$HERE/ref_harness.cpp"; do
  o="$OUT/obj/$(basename "$s" .cpp).o"
  if [ ! -f "$o" ] || [ "$s" -nt "$o" ]; then echo "$s"; fi
done | xargs -r -P "$JOBS" -I{} sh -c "$CXX $FLAGS -c {} -o $OUT/obj/\$(basename {} .cpp).o"
$CXX -shared -o "$OUT/libgrains_ref.so" "$OUT"/obj/*.o -lz
echo "built $OUT/libgrains_ref.so"
# the reference's Basilisk coupling interface over the same objects (the
# checker of the coupling library libgrains_b200_basilisk.so)
BAS=$REF/InterfaceCBasilisk
if [ ! -f "$OUT/basilisk.o" ] || [ "$BAS/src/InterfaceGrains3DBasilisk.cpp" -nt "$OUT/basilisk.o" ]; then
  $CXX $FLAGS -I"$BAS/include" -c "$BAS/src/InterfaceGrains3DBasilisk.cpp" -o "$OUT/basilisk.o"
fi
$CXX -shared -o "$OUT/libgrains_ref_basilisk.so" "$OUT/basilisk.o" \
    $(ls "$OUT"/obj/*.o | grep -v ref_harness.o) -lz
echo "built $OUT/libgrains_ref_basilisk.so"
