#!/usr/bin/env bash
# Build the reference's own CUDA interpreter (csrc/kernel_v1.cu +
# kernel_v1_impl.cuh + event_buffer.h), compiled from the sources where they
# lie in the read-only reference tree, into oracle/_ref/libref_kernel.so.
# The only addition is the typedef shim in oracle/ref_shim (the reference's
# vendored `ulib` header is absent).  Flags follow the reference's build.rs:58-61
# (-maxrregcount=128, -lineinfo) plus the sm_100a target.
# Output is test infrastructure: the reference arm of the parity tests and the
# reference-GPU timing line.  Nothing in the product links it.
# The reference tree: the first argument, else JQ_REFERENCE_ROOT, else the
# location this container mounts it at.
set -euo pipefail
REF=${1:-${JQ_REFERENCE_ROOT:-/root/reference}}
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
if [ ! -f "$REF/csrc/kernel_v1.cu" ]; then
  echo "reference tree not found at $REF; keeping prebuilt $OUT" >&2
  exit 0
fi
mkdir -p "$OUT"
nvcc -O3 -lineinfo -maxrregcount=128 -std=c++17 \
  -gencode arch=compute_100a,code=sm_100a \
  -Xcompiler -fPIC -shared \
  -I "$HERE/ref_shim" -I "$REF/csrc" \
  "$REF/csrc/kernel_v1.cu" -o "$OUT/libref_kernel.so"
echo "built $OUT/libref_kernel.so"
