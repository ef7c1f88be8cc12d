#!/usr/bin/env bash
# Builds the reference's four CUDA programs from their own sources, where they
# lie in the reference checkout, for sm_100a into oracle/_ref/bin/, and copies
# the reference's paper inputs into oracle/_ref/data/.  Parity oracle only:
# nothing in the product links or runs these.  Outputs stay in oracle/_ref/
# (git-ignored; carried to the GPU box with the working tree).
#   REF=/path/to/reference bash oracle/build_ref.sh
set -euo pipefail
REF=${REF:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
[ -d "$REF/cuda" ] || { echo "reference checkout not found at $REF" >&2; exit 1; }
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
for pid in "${pids[@]:-}"; do [ -n "$pid" ] && wait "$pid"; done
cp -u "$REF"/data/*.json "$OUT/data/"
echo "reference oracle binaries in $OUT/bin"
