#!/bin/sh
# Builds the reference harness (oracle/ref_harness.cu: CODAG's RLE v1 decoder compiled from
# CODAG's own headers) into oracle/_ref/ref_rlev1 (git-ignored; it travels with the working
# tree to the GPU machine).  CODAG's headers include <simt/atomic> from an un-vendored
# submodule; oracle/ref_shim provides those names from libcu++.
# Usage: oracle/build_ref.sh [path of the CODAG tree, default /root/reference]
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${1:-/root/reference}
mkdir -p "$HERE/_ref"
nvcc -gencode arch=compute_100a,code=sm_100a -O2 -std=c++17 -w --expt-relaxed-constexpr -DCUDA -DNOT_IMPL \
  -I "$HERE/ref_shim" -I "$REF/include" \
  "$HERE/ref_harness.cu" -o "$HERE/_ref/ref_rlev1"
echo "$HERE/_ref/ref_rlev1"
