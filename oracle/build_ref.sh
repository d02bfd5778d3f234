#!/usr/bin/env bash
# Build the parity checker from the reference's own sources (test
# infrastructure only).  Compiles oracle/ref_shim.cpp against the reference's
# header-only C++ in $AMIGO_REF_ROOT/include (default /root/reference) and
# links scipy's bundled OpenBLAS through oracle/blas_shim.c.
# Output: oracle/_ref/libamigo_ref.so (git-ignored; it travels with the tree).
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${AMIGO_REF_ROOT:-/root/reference}"
if [ ! -d "$REF/include" ]; then
  echo "build_ref.sh: reference sources not found at $REF; skipping" >&2
  exit 0
fi
OUT="$HERE/_ref"
mkdir -p "$OUT"
LIBDIR="$(python -c 'import scipy, os; print(os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs"))')"
OBLAS="$(ls "$LIBDIR"/libscipy_openblas*.so | head -1)"
gcc -O2 -fPIC -c "$HERE/blas_shim.c" -o "$OUT/blas_shim.o"
g++ -O2 -fPIC -shared -std=c++17 -fopenmp -DAMIGO_USE_OPENMP \
    -I"$HERE/ref_stub" -I"$REF/include" \
    "$HERE/ref_shim.cpp" "$OUT/blas_shim.o" \
    -o "$OUT/libamigo_ref.so.tmp" "$OBLAS" -Wl,-rpath,"$LIBDIR" -Wl,--no-undefined -fopenmp
mv "$OUT/libamigo_ref.so.tmp" "$OUT/libamigo_ref.so"
echo "built $OUT/libamigo_ref.so"
