#!/bin/bash
# Build libdmffb200.so for B200 (sm_100a) in-tree.  Usage: dmff_b200/csrc/build.sh
set -e
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/../libdmffb200.so"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -lineinfo -O3 -std=c++17 \
    -Xcompiler -fPIC -shared ${DMFFB_NVCC_EXTRA} \
    -o "$OUT" "$HERE/engine.cu" "$HERE/noalloc.cu" "$HERE/md_force.cu" "$HERE/serving.cpp" -lcufft -lpthread
echo "built $OUT"
