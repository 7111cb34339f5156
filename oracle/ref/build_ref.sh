#!/bin/sh
# Builds the pinning harness against the reference's own src/MortonLUT.h, in
# place in the read-only reference tree, into oracle/_ref/ (git-ignored).
# The rest of the reference cannot be built here: src/SVO.cu, src/BaseModel.*
# and src/IO.h need Eigen 3.4, which is fetched at configure time and is not
# available offline.
set -e
REF=${GPU_SVO_REF:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/../_ref"
mkdir -p "$OUT"
nvcc -std=c++17 -O1 -gencode arch=compute_100a,code=sm_100a -I"$REF/src" -o "$OUT/pin_morton" "$HERE/pin_morton.cu"
echo "$OUT/pin_morton"
