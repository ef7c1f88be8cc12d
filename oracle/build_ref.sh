#!/usr/bin/env bash
# Builds the reference's four CUDA programs from their own sources, where they
# lie in the reference checkout, for sm_100a into oracle/_ref/bin/, and copies
# the reference's paper inputs into oracle/_ref/data/.  Parity oracle only:
# nothing in the product links or runs these.  Outputs stay in oracle/_ref/
# (git-ignored; carried to the GPU box with the working tree).
#   REF=/path/to/reference bash oracle/build_ref.sh
#   bash oracle/build_ref.sh --where   prints the reference checkout it reads (nothing if absent)
# Without a reference checkout (the GPU box) it builds nothing and exits 0.
set -euo pipefail
REF=${REF:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
if [ "${1:-}" = "--where" ]; then
    [ -d "$REF/cuda" ] && echo "$REF"
    exit 0
fi
[ -d "$REF/cuda" ] || { echo "reference checkout not found at $REF: nothing to build" >&2; exit 0; }
mkdir -p "$OUT/bin" "$OUT/data"
pids=()
for prog in cuprym_cyclic cuprym_cyclic_kernel_vectors cuprym_deformation cuprym_deformation_kernel_vectors; do
    src="$REF/cuda/$prog.cu"
    dst="$OUT/bin/$prog"
    if [ ! -x "$dst" ] || [ "$src" -nt "$dst" ]; then
        "$NVCC" -O3 -std=c++17 -ccbin /usr/bin/g++ -gencode=arch=compute_100a,code=sm_100a \
            "$src" -o "$dst" -Xlinker -l:libzstd.so.1 &
        pids+=($!)
    fi
done
# The reference's CPU eliminated square (cpu_apply_eliminated_square) behind a
# timing harness: the CPU baseline of the paper workloads.
dst="$OUT/bin/ref_cpu_square"
if [ ! -x "$dst" ] || [ "$REF/cuda/cuprym_cyclic.cu" -nt "$dst" ] || [ "$HERE/ref_cpu_square.cu" -nt "$dst" ]; then
    "$NVCC" -O3 -std=c++17 -ccbin /usr/bin/g++ -gencode=arch=compute_100a,code=sm_100a \
        -DREF_CYCLIC_SOURCE="\"$REF/cuda/cuprym_cyclic.cu\"" -I"$REF/cuda" \
        "$HERE/ref_cpu_square.cu" -o "$dst" -Xlinker -l:libzstd.so.1 &
    pids+=($!)
fi
for pid in "${pids[@]:-}"; do [ -n "$pid" ] && wait "$pid"; done
cp -u "$REF"/data/*.json "$OUT/data/"
echo "reference oracle binaries in $OUT/bin"
