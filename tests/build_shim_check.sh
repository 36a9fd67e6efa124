#!/usr/bin/env bash
# Compile the evd::internal forwarding shim (ppopp27-brdc-ae_b200/shim/
# evd_tridiag_shim.cpp) against the reference's own headers, with a small
# test driver, into tests/libshim_check.so linked to libbrdc_b200.so.  Test
# infrastructure: the compiler checks the shim's signatures against the
# reference's declarations.  Reads the reference tree (REF, by default its
# mount point in the build container); exits 1 and builds nothing where
# the tree is absent.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
ROOT="$(dirname "$HERE")"
REF="${REF:-/root/reference}"
[ -d "$REF/gpu/src" ] || { echo "reference sources not found under $REF" >&2; exit 1; }
CXX="${CXX:-g++}"
CUDA_INC="${CUDA_HOME:-/usr/local/cuda}/include"
LIBDIR="$ROOT/ppopp27-brdc-ae_b200/brdc"
OUT="$HERE/libshim_check.so"
SHIM="$ROOT/ppopp27-brdc-ae_b200/shim/evd_tridiag_shim.cpp"
if [ -f "$OUT" ] && [ "$OUT" -nt "$SHIM" ] && [ "$OUT" -nt "$HERE/shim_driver.cpp" ] &&
   [ "$OUT" -nt "$0" ] && [ "$OUT" -nt "$ROOT/include/brdc.h" ]; then
  exit 0
fi
"$CXX" -std=c++17 -O2 -fPIC -shared -Wall -Werror=return-type \
  -I"$REF/gpu/include" -I"$REF/gpu/src" -I"$CUDA_INC" \
  -o "$OUT" "$SHIM" "$HERE/shim_driver.cpp" \
  -L"$LIBDIR" -lbrdc_b200 -Wl,-rpath,'$ORIGIN/../ppopp27-brdc-ae_b200/brdc'
echo "$OUT"
