#!/bin/bash
# Builds the reference solver (OpenSTC-MixingLayer, read-only sources under $REF, which the caller
# must set) for parity runs:
# .cu files through nvcc for sm_100a with relocatable device code, .cpp files through the host
# compiler (as the reference's CMake build does), FP64, fmt header-only, the single-rank MPI subset
# in oracle/ref/mpi.h, MAX_SPEC_NUMBER=9 / MAX_REAC_NUMBER=19.  Outputs go to oracle/_ref/ only:
#   openstc      the reference executable
#   ref_harness  oracle/ref/ref_harness.cu linked against every reference object except main()
# TEST INFRASTRUCTURE: these binaries are the checker for the oracle, never part of the product.
set -e
HERE="$(cd "$(dirname "$0")" && pwd)"
if [ -z "$REF" ]; then echo "REF must name the reference source tree (the directory holding src/)" >&2; exit 2; fi
OUT="$HERE/../_ref"
OBJ="$OUT/obj"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
CXX="${CXX:-g++}"
JOBS="${JOBS:-8}"
if [ ! -d "$REF/src" ]; then echo "reference sources not found at $REF" >&2; exit 2; fi
mkdir -p "$OBJ"
DEFS="-DMAX_SPEC_NUMBER=9 -DMAX_REAC_NUMBER=19 -DMAX_PASSIVE_SCALAR_NUMBER=5 -DFMT_HEADER_ONLY"
INCS="-I$HERE -I$REF/depends/include -I$REF/src"
# FMT_CONSTEVAL is emptied for nvcc so fmt's compile-time format checks do not trip its consteval handling
FLAGS="-std=c++20 -O3 -gencode arch=compute_100a,code=sm_100a -rdc=true $DEFS $INCS -DFMT_CONSTEVAL= -w"
CXXFLAGS="-std=c++20 -O3 $DEFS $INCS -I/usr/local/cuda/include -w"
CU_SRCS=$(cd "$REF/src" && ls *.cu stat_lib/*.cu)
CPP_SRCS=$(cd "$REF/src" && ls *.cpp gxl_lib/*.cpp)
export NVCC FLAGS REF OBJ CXX CXXFLAGS HERE
stale='o="$OBJ/$(echo {} | tr / _).o"; [ ! -f "$o" ] || [ "$REF/src/{}" -nt "$o" ] || [ "$HERE/mpi.h" -nt "$o" ]'
echo "$CU_SRCS" | xargs -P "$JOBS" -I{} bash -c "$stale"' && { $NVCC $FLAGS -c "$REF/src/{}" -o "$o" || exit 255; }; true'
echo "$CPP_SRCS" | xargs -P "$JOBS" -I{} bash -c "$stale"' && { $CXX $CXXFLAGS -c "$REF/src/{}" -o "$o" || exit 255; }; true'
$CXX $CXXFLAGS -c "$HERE/fmt_os_stub.cpp" -o "$OUT/fmt_os_stub.o"
$NVCC $FLAGS -c "$HERE/ref_harness.cu" -o "$OUT/ref_harness.o"
LINK="$NVCC -std=c++20 -gencode arch=compute_100a,code=sm_100a -rdc=true"
$LINK "$OBJ"/*.o "$OUT/fmt_os_stub.o" -o "$OUT/openstc"
# the harness reads the clock through __wrap_time (OSTC_REF_TIME fixes the inflow noise seed)
$LINK -Xlinker --wrap=time $(ls "$OBJ"/*.o | grep -v '/main.cu.o$') "$OUT/fmt_os_stub.o" "$OUT/ref_harness.o" -o "$OUT/ref_harness"
echo "built $OUT/openstc $OUT/ref_harness"
