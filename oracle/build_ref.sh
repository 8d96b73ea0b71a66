#!/bin/sh
# Builds the reference harnesses from CODAG's own sources into oracle/_ref/ (git-ignored;
# the built files travel with the working tree to the GPU machine).  TEST INFRASTRUCTURE ONLY.
#
#   oracle/_ref/ref_rlev1       CODAG's RLE v1 GPU decoder (oracle/ref_harness.cu, nvcc, sm_100a).
#                               CODAG's headers include <simt/atomic> from an un-vendored
#                               submodule (ogiroux/freestanding, unpinned); oracle/ref_shim
#                               provides those names from libcu++.
#   oracle/_ref/ref_rlev2_host  CODAG's RLE v2 encoder kernels run on the host
#                               (oracle/ref_rlev2_host.cpp, g++).  The host compiler cannot
#                               parse CUDA's <<<...>>> launch syntax, which appears only in
#                               CODAG's host launchers that the harness never calls, so the
#                               four headers it includes are copied into oracle/_ref/include
#                               with the launch configurations removed (nothing else changes);
#                               oracle/ref_shim_host stands in for the CUDA keywords and Thrust.
#
# Usage: oracle/build_ref.sh <CODAG source tree>   (or set CODAG_REFERENCE_DIR)
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${1:-$CODAG_REFERENCE_DIR}
if [ -z "$REF" ] || [ ! -d "$REF/include" ]; then
  echo "usage: $0 <CODAG source tree> (or set CODAG_REFERENCE_DIR)" >&2
  exit 1
fi
CUDA=${CUDA_HOME:-/usr/local/cuda}
OUT="$HERE/_ref"
mkdir -p "$OUT/include/rlev2"

nvcc -gencode arch=compute_100a,code=sm_100a -O2 -std=c++17 -w --expt-relaxed-constexpr -DCUDA -DNOT_IMPL \
  -I "$HERE/ref_shim" -I "$REF/include" \
  "$HERE/ref_harness.cu" -o "$OUT/ref_rlev1"

for h in common.h rlev2/utils.h rlev2/encoder.h rlev2/encoder_trans.h; do
  sed -E 's/<<<[^<>]*>>>//g' "$REF/include/$h" > "$OUT/include/$h"
done
g++ -std=c++20 -O2 -w -I "$HERE/ref_shim_host" -I "$OUT/include" -I "$CUDA/include" \
  "$HERE/ref_rlev2_host.cpp" -o "$OUT/ref_rlev2_host" -L "$CUDA/lib64" -lcudart -lpthread \
  -Wl,-rpath,"$CUDA/lib64"
echo "$OUT/ref_rlev1 $OUT/ref_rlev2_host"
