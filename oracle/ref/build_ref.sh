#!/bin/sh
# Builds oracle/_ref/ref_harness from the reference's own headers, where they
# lie (REF_DIR: the reference project's source tree; __graft_entry__.build()
# passes gmapf_b200/build.py's REF_DIR).  Host code only: the reference's
# CuQueue / CuNodesMap / V2Float are __host__ __device__ classes, compiled by
# nvcc for the CPU with contraction off (x86-64 SSE, IEEE binary32).
# Output goes to oracle/_ref/ and is never committed.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
if [ -z "$REF_DIR" ]; then
  echo "REF_DIR (the reference source tree) is not set; skipping" >&2
  exit 0
fi
OUT="$HERE/../_ref"
if [ ! -f "$REF_DIR/include/gmapf/misc/CuQueue.h" ]; then
  echo "reference headers not found under $REF_DIR/include; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
"$NVCC" -std=c++17 -O2 -w -Wno-deprecated-gpu-targets -x cu -Xcompiler -ffp-contract=off -include cfloat -include string \
  -I"$REF_DIR/include" "$HERE/ref_harness.cu" -o "$OUT/ref_harness"
echo "built $OUT/ref_harness"
