#!/usr/bin/env bash
# Builds the reference rdcu from its own sources, unmodified, for sm_100a:
#   nvcc -arch=sm_100a -O3 rdcu.cu dp45.cu bdf.cu -lcufft -lcublas -lcusparse
# with the link-only cuDSS stand-in of oracle/cudss_stub (cuDSS is not installed in
# this image; the reference's DP45 path never calls it).  Output: oracle/_ref/rdcu_ref;
# and oracle/_ref/rdcu_ref_lu, the same sources with a solving stand-in for cuDSS
# (oracle/cudss_stub/cudss_lu.cpp, cuSOLVER's host sparse LU), whose BDF path runs.
# Test infrastructure: the binary produces golden fixtures and is the reference arm of
# bench.py; librdcu never links or calls it.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
# RDCU_REFERENCE_DIR: the reference checkout (default: the read-only copy on the build machine)
REF="${RDCU_REFERENCE_DIR:-/root/reference}"
OUT="$HERE/_ref"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
if [ ! -f "$REF/rdcu.cu" ]; then
  echo "reference sources not found at $REF" >&2
  exit 2
fi
mkdir -p "$OUT"
if [ -x "$OUT/rdcu_ref" ] && [ "$OUT/rdcu_ref" -nt "$REF/rdcu.cu" ] && [ "$OUT/rdcu_ref" -nt "$HERE/cudss_stub/cudss_stub.c" ] &&
   [ -x "$OUT/rdcu_ref_lu" ] && [ "$OUT/rdcu_ref_lu" -nt "$HERE/cudss_stub/cudss_lu.cpp" ]; then
  exit 0
fi
"$NVCC" -arch=sm_100a -O3 -w -I"$HERE/cudss_stub" \
  "$REF/rdcu.cu" "$REF/dp45.cu" "$REF/bdf.cu" "$HERE/cudss_stub/cudss_stub.c" \
  -lcufft -lcublas -lcusparse -Xlinker -rpath=/usr/local/cuda/lib64 -o "$OUT/rdcu_ref"
echo "built $OUT/rdcu_ref"
# the same sources with the solving cuDSS stand-in (cuSOLVER's host sparse LU): the
# reference's BDF path runs
"$NVCC" -arch=sm_100a -O3 -w -I"$HERE/cudss_stub" \
  "$REF/rdcu.cu" "$REF/dp45.cu" "$REF/bdf.cu" "$HERE/cudss_stub/cudss_lu.cpp" \
  -lcufft -lcublas -lcusparse -lcusolver -Xlinker -rpath=/usr/local/cuda/lib64 -o "$OUT/rdcu_ref_lu"
echo "built $OUT/rdcu_ref_lu"
