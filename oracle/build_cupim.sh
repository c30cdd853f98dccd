#!/usr/bin/env bash
# Builds GPU-CUPIM's one-shot step, from the reference's own source where it lies, into
# oracle/_ref/libref_cupim.so (git-ignored; it travels to the GPU host with the tree).
# TEST INFRASTRUCTURE ONLY: tests/test_gpu_cupim_pin.py pins the oracle's one-shot
# restatement against it; the solver never links it.
#
# The reference's qap/ directory (qap.cu, layout.cu, layout.cuh, replica_pool_utils.cu) is put on
# the include path and compiled as it is; cupim_shim/random.cuh replaces its random-number
# header (cuRANDDx from mathdx is not vendored with the reference, perl-gpu/CMakeLists.txt:18-21).
# No copy of the reference source is written anywhere.  C++20 as the reference's CMakeLists
# sets; without relocatable device code, so its device-side thrust::reduce runs sequentially.
#
# The reference source path is $PIMQAP_REF_ROOT (default: the build container's read-only
# mount, named when used).  When it is absent the script does nothing and exits 0.
set -euo pipefail

REF_ROOT="${PIMQAP_REF_ROOT:-/root/reference}"
[ -n "${PIMQAP_REF_ROOT:-}" ] || echo "build_cupim.sh: PIMQAP_REF_ROOT unset, using $REF_ROOT"
QAP="$REF_ROOT/GPU-CUPIM/perl-gpu/src/lib/qap"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"

if [ ! -f "$QAP/qap.cu" ]; then
    echo "build_cupim.sh: $QAP/qap.cu not found, one-shot reference not built"
    exit 0
fi
mkdir -p "$OUT"
"$NVCC" -std=c++20 -O3 -gencode arch=compute_100a,code=sm_100a -ccbin /usr/bin/g++ \
    -Xcompiler -fPIC -shared -w -I "$HERE/cupim_shim" -I "$QAP" \
    "$HERE/cupim_harness.cu" -o "$OUT/libref_cupim.so"
echo "build_cupim.sh: built libref_cupim.so"
