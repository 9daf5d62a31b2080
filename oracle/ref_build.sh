#!/bin/bash
# Build the reference's own hop kernels (from their sources in the read-only reference
# tree, with shim headers for its absent external submodule) into
# oracle/_ref/libqcu_ref_kernels.so.  Test infrastructure only.
set -e
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${QCU_REFERENCE_DIR:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -d "$REF/include" ]; then
    echo "reference tree not found at $REF; nothing to build" >&2
    exit 0
fi
mkdir -p "$OUT"
if [ "$OUT/libqcu_ref_kernels.so" -nt "$HERE/ref_wrap.cu" ] && [ -z "$FORCE" ]; then
    exit 0
fi
nvcc -gencode arch=compute_100a,code=sm_100a -O2 -std=c++17 -Xcompiler -fPIC -shared \
    -I "$HERE/ref_shim" -I "$REF/include" -w \
    -o "$OUT/libqcu_ref_kernels.so" "$HERE/ref_wrap.cu"
