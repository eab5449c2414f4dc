#!/bin/bash
# Compiles the reference's own CPU code for the hot path, straight from the
# reference sources, into oracle/_ref/ (git-ignored; travels with the tree).
#   libref_scan.so : scan/main.cu (cpu_sum_scan, scan/main.cu:11-21) with its
#                    main() renamed, linked with scan/scan_gsrb.cu whose GPU
#                    code is compiled but never called.
# Nothing is copied into the repository; only the built library lands here.
#   usage: ref_build.sh [reference root]   (default: $GSRB_REFERENCE_ROOT, else /root/reference)
set -euo pipefail
REF=${1:-${GSRB_REFERENCE_ROOT:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
if [ ! -d "$REF/scan" ]; then
  echo "reference tree not found at $REF; skipping oracle/_ref" >&2
  exit 0
fi
mkdir -p "$OUT"
"$NVCC" -O2 -std=c++14 -shared -Xcompiler -fPIC -gencode arch=compute_100a,code=sm_100a \
  -Dmain=ref_scan_main -I"$REF/scan" \
  "$REF/scan/main.cu" "$REF/scan/scan_gsrb.cu" -o "$OUT/libref_scan.so"
echo "built $OUT/libref_scan.so"
