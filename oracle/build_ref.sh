#!/usr/bin/env bash
# Compile the reference CUDA prototype (values-only BR solver) from its own
# sources, without its CMake build, for sm_100a, into oracle/_ref/.  Test
# and benchmark infrastructure only (a checker and a timed comparison); the
# product never links it.  Reads the reference tree (REF, by default its
# mount point in the build container); where the tree is absent the script
# exits with status 1 and builds nothing.  The built library travels with
# the repository.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${REF:-/root/reference}"
OUT="$HERE/_ref"
NVCC="${NVCC:-nvcc}"
SRC="$REF/gpu/src"
[ -d "$SRC" ] || { echo "reference sources not found under $REF" >&2; exit 1; }
mkdir -p "$OUT"
LIB="$OUT/libref_brdc_gpu.so"
MERGE_LIB="$OUT/libref_merge.so"
if [ -f "$LIB" ] && [ "$LIB" -nt "$HERE/ref_shim.cu" ] && [ "$LIB" -nt "$0" ] &&
   [ -f "$MERGE_LIB" ] && [ "$MERGE_LIB" -nt "$HERE/ref_merge.cu" ] && [ "$MERGE_LIB" -nt "$0" ]; then
  exit 0
fi
FLAGS=(-gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -Xcompiler -fPIC
       -I"$REF/gpu/include" -I"$SRC" -diag-suppress 177,550)
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT
"$NVCC" "${FLAGS[@]}" -c "$SRC/handle.cu" -o "$TMP/handle.o"
"$NVCC" "${FLAGS[@]}" -c "$SRC/tridiag_solver.cu" -o "$TMP/tridiag_solver.o"
"$NVCC" "${FLAGS[@]}" -c "$SRC/ae_stage_stubs.cu" -o "$TMP/ae_stage_stubs.o"
"$NVCC" "${FLAGS[@]}" -x cu -c "$SRC/tridiag_solver_cpu.cpp" -o "$TMP/tridiag_solver_cpu.o"
"$NVCC" "${FLAGS[@]}" -c "$HERE/ref_shim.cu" -o "$TMP/ref_shim.o"
"$NVCC" -shared -gencode arch=compute_100a,code=sm_100a -o "$LIB" "$TMP"/*.o \
  -lcublas -lcusolver -ldl
# the reference's deflation kernels alone, driven on caller-supplied merge inputs
"$NVCC" "${FLAGS[@]}" -shared -o "$MERGE_LIB" "$HERE/ref_merge.cu"
echo "$LIB"
