#!/usr/bin/env bash
# Builds the reference fCWT CPU path from its own sources into oracle/_ref/,
# for use as the parity oracle and the timed CPU baseline only.
#
#   - compiles <ref>/src/fcwt/fcwt.cpp (read in place, never copied) together
#     with oracle/ref_shim.cpp into oracle/_ref/libfcwt_ref.so;
#   - the reference links the FFTW 3.3.10 single-precision binaries it ships in
#     <ref>/libs/; they are copied (not inspected) into oracle/_ref/ under the
#     sonames the loader looks for, so the library also loads on a machine
#     without the reference tree.
#
# Flags follow the reference's own builds: -mavx -O3 (setup.py:44-45), OpenMP
# for the daughter loop, asserts compiled out (Release). The reference source
# omits <cassert>/<cstring>, hence the -include flags.
#
# Usage: oracle/build_ref.sh [reference_root]
#   (default: $FCWT_REFERENCE_ROOT, else /root/reference)
set -euo pipefail
REF="${1:-${FCWT_REFERENCE_ROOT:-/root/reference}}"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
if [ ! -f "$REF/src/fcwt/fcwt.cpp" ]; then
    echo "build_ref: reference sources not found under $REF" >&2
    exit 1
fi
mkdir -p "$OUT"
cp -f "$REF/libs/libfftw3fl.so" "$OUT/libfftw3f.so.3"
cp -f "$REF/libs/libfftw3f_ompl.so" "$OUT/libfftw3f_omp.so.3"
chmod u+w "$OUT/libfftw3f.so.3" "$OUT/libfftw3f_omp.so.3"
g++ -std=c++17 -O3 -mavx -fopenmp -fPIC -shared -DNDEBUG \
    -include cassert -include cstring \
    -I"$REF/src/fcwt" -I"$REF/libs" \
    "$HERE/ref_shim.cpp" "$REF/src/fcwt/fcwt.cpp" \
    -L"$OUT" -l:libfftw3f.so.3 -l:libfftw3f_omp.so.3 \
    -Wl,-rpath,'$ORIGIN' \
    -o "$OUT/libfcwt_ref.so.tmp"
mv -f "$OUT/libfcwt_ref.so.tmp" "$OUT/libfcwt_ref.so"
echo "build_ref: $OUT/libfcwt_ref.so"
