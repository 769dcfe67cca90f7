#!/usr/bin/env bash
# Builds the reference cross-check libraries (test infrastructure only) from the reference's own headers, read in
# place from its source tree, with the serial Kokkos stand-in of oracle/ref/shim and the header-only fmt that
# ships with spdlog. Outputs go to oracle/_ref/ only:
#   libbvhref26.so  element trees of dop_26 (the reference's default bphase_kdop)
#   libbvhref6.so   element trees of dop_6 (built with BVH_BROADPHASE_6_DOP)
# The reference's own build system (CMake with Kokkos and DARMA/vt) is not used.
# Usage: ref_build.sh <reference src directory> (or REF_SRC in the environment).
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF_SRC="${1:-${REF_SRC:-}}"
if [ -z "$REF_SRC" ]; then
  echo "usage: ref_build.sh <reference src directory>" >&2
  exit 2
fi
CXX="${ORACLE_CXX:-/usr/bin/g++}"
FMT_INC="$(python3 -c 'import os, flashinfer; print(os.path.join(os.path.dirname(flashinfer.__file__), "data", "spdlog", "include"))' 2>/dev/null || true)"
if [ ! -d "$REF_SRC/bvh" ] || [ -z "$FMT_INC" ] || [ ! -f "$FMT_INC/spdlog/fmt/bundled/format.h" ]; then
  echo "reference sources or header-only fmt not found; oracle/_ref not built" >&2
  exit 0
fi
mkdir -p "$HERE/_ref"
FLAGS=(-std=c++20 -O2 -ffp-contract=off -fno-fast-math -fPIC -shared -DFMT_HEADER_ONLY -Wno-deprecated
       -I"$HERE/ref/shim" -I"$REF_SRC" -I"$FMT_INC")
"$CXX" "${FLAGS[@]}" "$HERE/ref/bvh_ref.cpp" -o "$HERE/_ref/libbvhref26.so" &
p26=$!
"$CXX" "${FLAGS[@]}" -DBVH_BROADPHASE_6_DOP "$HERE/ref/bvh_ref.cpp" -o "$HERE/_ref/libbvhref6.so"
wait "$p26"
