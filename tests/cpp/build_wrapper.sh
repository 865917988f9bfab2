#!/bin/sh
# Build tests/cpp/gpu_wrapper_test.cpp: the reference's include/gpu/GpuPauliSum.h
# and its CPU headers (read in place from $PAULIB_REFERENCE_DIR, default
# /root/reference) linked against the in-tree libpaulib_b200.so.
#   build_wrapper.sh <out-binary>
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=$(cd "$HERE/../.." && pwd)
REF=${PAULIB_REFERENCE_DIR:-/root/reference}
CUDA=${CUDA_HOME:-/usr/local/cuda}
OUT=$1
OUTDIR=$(cd "$(dirname "$OUT")" && pwd)
# rpath relative to the binary, so the build travels with the working tree
REL=$(python3 -c "import os,sys; print(os.path.relpath(sys.argv[1], sys.argv[2]))" \
      "$ROOT/paulib_b200" "$OUTDIR")
g++ -std=c++20 -O2 -fopenmp -I"$REF/include" -I"$CUDA/include" "$HERE/gpu_wrapper_test.cpp" \
    -L"$ROOT/paulib_b200" -lpaulib_b200 -Wl,-rpath,"\$ORIGIN/$REL" \
    -L"$CUDA/lib64" -lcudart -o "$OUT"
