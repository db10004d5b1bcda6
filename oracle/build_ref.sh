#!/usr/bin/env bash
# ORACLE -- test infrastructure only.  Compiles the reference CULS sources,
# where they lie, together with oracle/ref_harness.cu into
# oracle/_ref/rw_harness (git-ignored; it travels to the GPU box with the
# working tree).  The reference's own CMake build is not used: this compiles
# its .cu files directly with the flags its CMakeLists.txt sets
# (-std=c++17 -O3 --extended-lambda), plus `-include cstdio` (its print.cu
# needs it under CUDA 12.9) and a native sm_100a target.
#
#   oracle/build_ref.sh [path/to/CULS]      (default /root/reference)
set -euo pipefail
REF=${1:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
if [ ! -f "$REF/src/algorithms/rewrite.cu" ]; then
    echo "build_ref: no CULS sources at $REF" >&2
    exit 1
fi
mkdir -p "$OUT/obj"
FLAGS=(-gencode arch=compute_100a,code=sm_100a -std=c++17 -O3 --extended-lambda -include cstdio -w
       -I "$REF/src" -I "$REF/src/hash_table" -I "$REF/src/algorithms" -I "$REF/include")
SRCS=()
for f in "$REF"/src/*.cu "$REF"/src/aig/*.cu "$REF"/src/misc/*.cu "$REF"/src/algorithms/*.cu; do
    case "$(basename "$f")" in
        rewrite.cu) ;;  # compiled inside ref_harness.cu
        *) SRCS+=("$f") ;;
    esac
done
OBJS=()
pids=()
for f in "${SRCS[@]}" "$HERE/ref_harness.cu"; do
    o="$OUT/obj/$(basename "$f" .cu).o"
    OBJS+=("$o")
    if [ ! -f "$o" ] || [ "$f" -nt "$o" ]; then
        "$NVCC" "${FLAGS[@]}" -c "$f" -o "$o" &
        pids+=($!)
    fi
done
for p in "${pids[@]}"; do wait "$p"; done
"$NVCC" -gencode arch=compute_100a,code=sm_100a -o "$OUT/rw_harness" "${OBJS[@]}"
echo "$OUT/rw_harness"
