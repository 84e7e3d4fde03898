#!/usr/bin/env bash
# Builds the reference's own CPU gridrec into oracle/_ref/ (test infrastructure).
#
#   oracle/_ref/libgridrec_ref.so     GridRec class, FP32, NR FFT  (gridrec/GPU)
#   oracle/_ref/libgridrec_ref64.so   the same sources with float -> double,
#                                     made on temporary copies outside the repo
#   oracle/_ref/libgridrec_refb.so    GridrecCPP 5.2 C API (centre, sampl, filter name)
#   oracle/_ref/libfbp_ref.so         OptimizedFBP (CPU filtered backprojection, the
#                                     ReconAlgorithm FBP comparator)
#   oracle/_ref/libprep_ref.so        ring removal, shift/half-padding and entropy of the
#                                     reference drivers (line ranges written to a
#                                     temporary directory, see prep_ref_driver.cpp)
#
# The sources are compiled where they lie under the reference tree; nothing of
# the reference is copied into this repository.  gridrec.cu is plain host C++
# when USE_GRIDREC_GPU is undefined, so an empty tomo_recon_config.h suffices.
#
# Usage: oracle/build_ref.sh [--if-present] [REFERENCE_ROOT]
#   REFERENCE_ROOT defaults to $GR_REFERENCE_ROOT, else /root/reference;
#   --if-present: exit 0 without building when the reference tree is absent.
set -euo pipefail
IF_PRESENT=0
if [ "${1:-}" = "--if-present" ]; then IF_PRESENT=1; shift; fi
REF="${1:-${GR_REFERENCE_ROOT:-/root/reference}}"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
GPU="$REF/gridrec/GPU"
CPP="$REF/gridrec/GridrecCPP/Gridrec5.2"
if [ ! -f "$GPU/gridrec.cu" ]; then
  [ "$IF_PRESENT" = 1 ] && exit 0
  echo "build_ref.sh: reference not found at $REF" >&2
  exit 1
fi
mkdir -p "$OUT"
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT
: > "$TMP/tomo_recon_config.h"
CXX="${CXX:-g++}"
FLAGS="-O2 -fPIC -shared -w -Wl,-Bsymbolic"

# Oracle A: reference GridRec, FP32.
$CXX $FLAGS -I"$TMP" -I"$GPU" -x c++ "$GPU/gridrec.cu" -x c++ \
  "$GPU/recon_algorithm.cpp" "$GPU/fft_nr.cpp" "$HERE/ref_driver.cpp" \
  -o "$OUT/libgridrec_ref.so"

# Oracle A64: the same algorithm in double (temporary copies, sed float->double).
mkdir -p "$TMP/f64"
for f in gridrec.h recon_algorithm.h recon_algorithm.cpp fft.h fft_nr.cpp; do
  sed 's/\bfloat\b/double/g' "$GPU/$f" > "$TMP/f64/$f"
done
sed 's/\bfloat\b/double/g' "$GPU/gridrec.cu" > "$TMP/f64/gridrec.cpp"
cp "$TMP/tomo_recon_config.h" "$TMP/f64/"
$CXX $FLAGS -DREAL=double -I"$TMP/f64" "$TMP/f64/gridrec.cpp" \
  "$TMP/f64/recon_algorithm.cpp" "$TMP/f64/fft_nr.cpp" "$HERE/ref_driver.cpp" \
  -o "$OUT/libgridrec_ref64.so"

# Oracle B: GridrecCPP 5.2 (grid_io.cpp needs netCDF and is left out).
$CXX $FLAGS -fpermissive -I"$CPP" "$CPP/grid.cpp" "$CPP/fftgr.cpp" \
  "$CPP/filters.cpp" "$CPP/pswf.cpp" "$CPP/grid_math.cpp" "$HERE/refb_driver.cpp" \
  -o "$OUT/libgridrec_refb.so"

# Oracle D: the reference's CPU OptimizedFBP.
$CXX $FLAGS -I"$GPU" -x c++ "$GPU/filteredbackprojection.cpp" "$GPU/recon_algorithm.cpp" \
  "$GPU/fft_nr.cpp" "$HERE/fbp_ref_driver.cpp" -o "$OUT/libfbp_ref.so"

# Oracle C: slice-pipeline steps of tomo_recon / find_shift.
FS="$REF/find_shift/src/main/find_shift.cpp"
TR="$GPU/tomo_recon.cpp"
sed -n '3905,3972p' "$TR" > "$TMP/ring_ref.inc"
sed -n '2078,2115p' "$FS" > "$TMP/entropy_ref.inc"
sed -n '3708,3807p' "$TR" > "$TMP/shiftpad_ref.inc"
sed -n '1975,2076p' "$FS" > "$TMP/xcorr_ref.inc"
grep -q 'void RingCorrectionSinogram' "$TMP/ring_ref.inc"
grep -q 'float entropy( float\* data' "$TMP/entropy_ref.inc"
grep -q 'float kk = k - xoffset' "$TMP/shiftpad_ref.inc"
grep -q 'void data_interp' "$TMP/xcorr_ref.inc"
$CXX $FLAGS -I"$TMP" "$HERE/prep_ref_driver.cpp" -o "$OUT/libprep_ref.so"

echo "built: $(ls "$OUT")"
