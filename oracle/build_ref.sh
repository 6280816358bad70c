#!/usr/bin/env bash
# Builds the reference's own CPU path (fpaboim/gpufem src/FEM, src/SPRmatrix,
# src/LAops, src/Utils) as two shared libraries used ONLY as a test oracle and
# as the timed CPU baseline:
#
#   oracle/_ref/libref_fp32.so   fem_float = float  (as shipped)
#   oracle/_ref/libref_fp64.so   fem_float = double (overlay, see below)
#
# Nothing is copied into the repository: the sources are copied at build time
# into oracle/_ref/ (git-ignored) and patched there.  The FP64 overlay makes
# four mechanical edits, all required only because `fem_float` becomes double:
#   1. Utils/util.h          `#define fem_float float` -> double
#   2. Utils/fileIO.{h,cc}   drop writeNumTab(double), now a duplicate overload
#   3. SPRmatrix/SPRmatrix.cc drop the EIG (Eigen, float-only) format branch
#   4. -include cmath         (sqrt of double in FemData.cc)
# Linux shims: oracle/shims/windows.h, oracle/shims/CL/opencl.h; link stubs and
# the METIS dual-graph restatement: oracle/ref_stubs.cc; the C-ABI driver the
# tests call: oracle/ref_driver.cc.
#
# Usage: oracle/build_ref.sh REFERENCE_ROOT   (or GPUFEM_REFERENCE_ROOT in the environment)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${GPUFEM_REFERENCE_ROOT:-}}"
if [ -z "$REF" ]; then
  echo "build_ref.sh: give the reference root as an argument or in GPUFEM_REFERENCE_ROOT" >&2
  exit 2
fi
OUT="$HERE/_ref"
if [ ! -d "$REF/src/FEM" ]; then
  echo "build_ref.sh: reference sources not found at $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
# /usr/bin/g++ ships libgomp; a CXX from the environment may not.
CXX="${ORACLE_CXX:-/usr/bin/g++}"
CXXFLAGS="-O2 -fopenmp -fPIC -std=c++17 -fpermissive -w -include cmath -include windows.h -DNDEBUG"

prepare_tree() {  # $1 = dest dir
  local dst="$1"
  rm -rf "$dst"
  mkdir -p "$dst"
  for d in FEM SPRmatrix LAops Utils OpenCL; do
    cp -r "$REF/src/$d" "$dst/$d"
  done
  # case fixes for includes written on a case-insensitive file system
  ln -sf FemData.h "$dst/FEM/femdata.h"
  ln -sf Utils "$dst/utils"
  ln -sf OCLwrapper.h "$dst/OpenCL/Oclwrapper.h"
}

SRCS="FEM/StiffAlgo.cc FEM/StiffAlgoCPU.cc FEM/StiffAlgoGpuOmp.cc FEM/StiffAlgoGPU.cc
      FEM/fem.cc FEM/femColor.cc FEM/FemData.cc LAops/LAops.cc Utils/util.cc
      Utils/fileIO.cc SPRmatrix/SPRmatrix.cc SPRmatrix/ELLmatrix.cc
      SPRmatrix/ELLmatrix2.cc SPRmatrix/CSRmatrix.cc SPRmatrix/DIAmatrix.cc
      SPRmatrix/DENmatrix.cc"

build_variant() {  # $1 = tag (fp32|fp64)
  local tag="$1"
  local tree="$OUT/src_$tag"
  prepare_tree "$tree"
  local extra_srcs=""
  if [ "$tag" = "fp64" ]; then
    sed -i 's/^#define fem_float float/#define fem_float double/' "$tree/Utils/util.h"
    sed -i '/int writeNumTab(double num);/d' "$tree/Utils/fileIO.h"
    # remove the body of FileIO::writeNumTab(double) (from its signature to the closing brace)
    sed -i '/^int FileIO::writeNumTab(double num) {/,/^}/d' "$tree/Utils/fileIO.cc"
    sed -i '/#include "EIGmatrix.h"/d' "$tree/SPRmatrix/SPRmatrix.cc"
    sed -i '/else if (matformat == EIG)/,+1d' "$tree/SPRmatrix/SPRmatrix.cc"
    grep -q 'fem_float double' "$tree/Utils/util.h"
  else
    extra_srcs="SPRmatrix/EIGmatrix.cc"
  fi
  local objs=()
  local pids=()
  mkdir -p "$OUT/obj_$tag"
  for s in $SRCS $extra_srcs; do
    local o="$OUT/obj_$tag/$(basename "${s%.cc}").o"
    $CXX $CXXFLAGS -I"$HERE/shims" -I"$tree" -I"$REF/libs/eigen3.2" \
        -I"$REF/libs/metis/include" -c "$tree/$s" -o "$o" &
    pids+=($!)
    objs+=("$o")
  done
  for f in ref_stubs ref_driver; do
    local o="$OUT/obj_$tag/$f.o"
    $CXX $CXXFLAGS -I"$HERE/shims" -I"$tree" -I"$REF/libs/eigen3.2" \
        -I"$REF/libs/metis/include" -c "$HERE/$f.cc" -o "$o" &
    pids+=($!)
    objs+=("$o")
  done
  for p in "${pids[@]}"; do wait "$p"; done
  $CXX -shared -fopenmp -o "$OUT/libref_$tag.so" "${objs[@]}"
  echo "built $OUT/libref_$tag.so"
}

build_variant fp32
build_variant fp64
