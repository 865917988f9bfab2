#!/bin/sh
# Build the C++ facade test against the in-tree library:  build.sh <out-binary>
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=$(cd "$HERE/../.." && pwd)
CUDA=${CUDA_HOME:-/usr/local/cuda}
g++ -std=c++17 -O1 -Wall -I"$ROOT/include" -I"$CUDA/include" "$HERE/facade_test.cpp" \
    -L"$ROOT/paulib_b200" -lpaulib_b200 -Wl,-rpath,"$ROOT/paulib_b200" \
    -L"$CUDA/lib64" -lcudart -o "$1"
