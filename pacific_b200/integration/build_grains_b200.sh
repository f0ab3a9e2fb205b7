#!/bin/sh
# Builds oracle/_ref/grains_b200: the Grains3D executable -- the reference's
# own main() (GRAINS_V1/Main/src/main.cpp) and sources, compiled unmodified
# by oracle/build_ref.sh -- with the GrainsB200 application (GrainsB200.cpp)
# and its factory branch (grains_b200_factory.cpp, reached through
# --wrap on GrainsBuilderFactory::create), linked with libgrains_b200.so.
# An input file with <Grains3D Type="B200"> then runs its time loop on the GPU;
# Type="Standard" runs the reference's own serial step, in the same binary.
#
# Needs the reference tree (GRAINS_REFERENCE, default /root/reference), the
# reference objects of oracle/build_ref.sh and pacific_b200/libgrains_b200.so.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REPO=$(cd "$HERE/../.." && pwd)
REF=${GRAINS_REFERENCE:-/root/reference}/GRAINS_V1
OBJ=$REPO/oracle/_ref/obj
OUT=$REPO/oracle/_ref
CXX=${GRAINS_REF_CXX:-g++}
[ -d "$REF/Grains" ] || { echo "reference tree not found: $REF (set GRAINS_REFERENCE)" >&2; exit 1; }
[ -f "$OBJ/Grains.o" ] || { echo "reference objects missing: run oracle/build_ref.sh" >&2; exit 1; }
[ -f "$REPO/pacific_b200/libgrains_b200.so" ] || { echo "libgrains_b200.so missing" >&2; exit 1; }
FLAGS="-std=c++17 -O3 -ffp-contract=off -fPIC -w -I$REPO/oracle/shim -I$REF/Grains/include -I$REPO/include -I$HERE"
mkdir -p "$OUT/b200"
$CXX $FLAGS -c "$REF/Main/src/main.cpp" -o "$OUT/b200/main.o"
$CXX $FLAGS -c "$HERE/GrainsB200.cpp" -o "$OUT/b200/GrainsB200.o"
$CXX $FLAGS -c "$HERE/grains_b200_factory.cpp" -o "$OUT/b200/grains_b200_factory.o"
$CXX -o "$OUT/grains_b200" "$OUT/b200/main.o" "$OUT/b200/GrainsB200.o" \
    "$OUT/b200/grains_b200_factory.o" $(ls "$OBJ"/*.o | grep -v ref_harness.o) \
    -Wl,--wrap=_ZN20GrainsBuilderFactory6createEP10DOMElement \
    -L"$REPO/pacific_b200" -l:libgrains_b200.so -Wl,-rpath,"\$ORIGIN/../../pacific_b200" -lz
echo "built $OUT/grains_b200"
