#!/usr/bin/env bash
# Builds oracle/_ref/libtd16ref.so from the reference's own native sources
# (read in place, unmodified) plus oracle/ref_driver.cu.  TEST INFRASTRUCTURE
# ONLY.  The reference checkout is taken from TD16_REFERENCE (this recipe's
# default is the build container's read-only checkout); where it is absent the
# recipe skips, and the prebuilt library (if any) is used as is.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${TD16_REFERENCE:-/root/reference}/emitter/src/native"
OUT="$HERE/_ref"
if [ ! -d "$REF" ]; then
  echo "reference sources not found at $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
NVCC="${NVCC:-$(command -v nvcc || echo /usr/local/cuda/bin/nvcc)}"
"$NVCC" -O3 -std=c++17 -gencode arch=compute_100a,code=sm_100a -lineinfo \
  -DMAX_N=17 -DMAX_DEPTH=9 -I "$REF" -Xcompiler -fPIC -shared \
  -o "$OUT/libtd16ref.so" \
  "$REF/backtracking/sorting_search.cu" "$REF/backtracking/slot_manager.cu" "$HERE/ref_driver.cu" \
  -lcudart
echo "$OUT/libtd16ref.so"
