#!/bin/sh
# Builds oracle/_ref/libgrains_ref.so: the Grains3D reference (GRAINS_V1/Grains
# sources, compiled unmodified where they lie) + the single-rank MPI and
# Xerces DOM stand-ins in oracle/shim/ + the step harness ref_harness.cpp.
# TEST INFRASTRUCTURE: it pins the CPU restatement and produces the golden
# vectors under tests/golden/.  Needs the reference tree (default
# /root/reference); outputs go to oracle/_ref/ only.
#
# Flags: -O2 -ffp-contract=off, x86-64 baseline ISA (no FMA), as the
# reference's own g++ build on x86-64 (GRAINS_V1/Env, -O3 without -march).
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${GRAINS_REFERENCE:-/root/reference}/GRAINS_V1/Grains
OUT=$HERE/_ref
JOBS=${JOBS:-8}
[ -d "$REF" ] || { echo "reference tree not found: $REF" >&2; exit 1; }
mkdir -p "$OUT/obj"
# the system g++ (its libstdc++ is the shared one Python processes load)
CXX=${GRAINS_REF_CXX:-g++}
FLAGS="-std=c++17 -O2 -ffp-contract=off -fPIC -w -I$HERE/shim -I$REF/include"
SRCS=$(ls "$REF"/Base/src/*.cpp "$REF"/Component/src/*.cpp "$REF"/Geometry/src/*.cpp \
          "$REF"/TimeIntegration/src/*.cpp "$REF"/XML/src/*.cpp "$REF"/PostProcessing/src/*.cpp \
          "$REF"/Fluid/src/*.cpp)
for s in $SRCS "$HERE/shim/grains_shim.cpp" "$HERE/ref_harness.cpp"; do
  o="$OUT/obj/$(basename "$s" .cpp).o"
  if [ ! -f "$o" ] || [ "$s" -nt "$o" ]; then echo "$s"; fi
done | xargs -r -P "$JOBS" -I{} sh -c "$CXX $FLAGS -c {} -o $OUT/obj/\$(basename {} .cpp).o"
$CXX -shared -o "$OUT/libgrains_ref.so" "$OUT"/obj/*.o -lz
echo "built $OUT/libgrains_ref.so"
