#!/usr/bin/env bash
# Build oracle/_ref/libboys_ref.so from the reference's src/lookup/boys.cpp,
# compiled unmodified where it lies (it has no dependencies beyond the C++
# standard library), plus the C shim in this directory.  The rest of the
# reference's integral code needs Eigen 3.4 (fetched by its CMake at configure
# time, absent here), so it is not built; the oracle restates it instead.
# Usage: oracle/build_ref.sh [reference-root]
#        (default: $PLANCK_REFERENCE_ROOT, else /root/reference)
set -euo pipefail
REF="${1:-${PLANCK_REFERENCE_ROOT:-/root/reference}}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
mkdir -p "$HERE/_ref"
if [ ! -f "$REF/src/lookup/boys.cpp" ]; then
  echo "reference sources not found under $REF; oracle/_ref not rebuilt" >&2
  exit 0
fi
g++ -std=c++23 -O2 -fPIC -shared -I"$REF/src" \
    "$REF/src/lookup/boys.cpp" "$HERE/ref_boys_shim.cpp" \
    -o "$HERE/_ref/libboys_ref.so"
echo "built $HERE/_ref/libboys_ref.so"
