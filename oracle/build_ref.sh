#!/usr/bin/env bash
# Build the reference GPUDPD executable (xxin125/gpumdpd) from its own sources, untouched,
# into oracle/_ref/.  This is test and baseline infrastructure only: the binary is the
# reference's own CUDA build, used to generate golden fixtures on a GPU host and as the
# "reference" arm of bench.py.  Nothing in the product links or calls it.
#
# The stock Makefile targets sm_60 and fails on CUDA 12.9 because two sources use
# thrust::max_element/min_element without including <thrust/extrema.h>; the header is
# force-included on the command line instead of editing any source.
#
# Usage: oracle/build_ref.sh [SINGLE|DOUBLE|SHIM] [REF_SRC]
#   (mode default SINGLE, the reference's default; REF_SRC is the reference's src/
#   directory, from the second argument or the environment variable REF_SRC)
#   SHIM: the SINGLE build plus the plugins of gpumdpd_b200/shim/ (pair_style dpd/b200 and
#   mdpd/b200, bond_style harmonic/b200, fix nve/b200, which hand the reference's device
#   buffers to libdpd_b200), linked against the in-tree libdpd_b200.so
#   -> oracle/_ref/gpudpd_single_b200.
set -euo pipefail
MODE="${1:-SINGLE}"
PREC="$MODE"
[ "$MODE" = "SHIM" ] && PREC=SINGLE
REF_SRC="${2:-${REF_SRC:-}}"
if [ -z "$REF_SRC" ]; then
    echo "usage: $0 [SINGLE|DOUBLE|SHIM] REF_SRC   (the reference's src/ directory)" >&2
    exit 2
fi
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
OBJ="$OUT/obj_${PREC}"
if [ ! -d "$REF_SRC" ]; then
    echo "reference sources not found at $REF_SRC" >&2
    exit 1
fi
mkdir -p "$OBJ"
FLAGS=(-O3 -std=c++14 -gencode arch=compute_100a,code=sm_100a -I"$REF_SRC" "-D$PREC" -include thrust/extrema.h)
objs=()
pids=()
for src in "$REF_SRC"/*/*.cu; do
    rel="${src#$REF_SRC/}"
    o="$OBJ/${rel//\//_}.o"
    objs+=("$o")
    if [ ! -f "$o" ] || [ "$src" -nt "$o" ]; then
        nvcc "${FLAGS[@]}" -dc "$src" -o "$o" &
        pids+=($!)
        # keep at most 8 compilers in flight
        if [ "${#pids[@]}" -ge 8 ]; then
            for p in "${pids[@]}"; do wait "$p"; done
            pids=()
        fi
    fi
done
for p in "${pids[@]}"; do wait "$p"; done
lower="$(echo "$PREC" | tr 'A-Z' 'a-z')"
if [ "$MODE" = "SHIM" ]; then
    REPO="$(cd "$HERE/.." && pwd)"
    shims=()
    for src in "$REPO"/gpumdpd_b200/shim/*.cu; do
        o="$OBJ/shim_$(basename "$src" .cu).o"
        nvcc "${FLAGS[@]}" -I"$REPO/include" -dc "$src" -o "$o"
        shims+=("$o")
    done
    nvcc "${FLAGS[@]}" "${objs[@]}" "${shims[@]}" -L"$REPO/gpumdpd_b200" -ldpd_b200 \
        -Xlinker -rpath -Xlinker '$ORIGIN/../../gpumdpd_b200' -o "$OUT/gpudpd_single_b200"
    echo "built $OUT/gpudpd_single_b200"
    exit 0
fi
nvcc "${FLAGS[@]}" "${objs[@]}" -o "$OUT/gpudpd_${lower}"
echo "built $OUT/gpudpd_${lower}"
if [ "$PREC" = "SINGLE" ]; then
    # Saru known-answer harness: the reference's pair_dpd.cu compiled inside
    # oracle/ref_saru_harness.cu, linked with the reference's pair registry object.
    nvcc "${FLAGS[@]}" -rdc=true "$HERE/ref_saru_harness.cu" "$OBJ/force_pair.cu.o" -o "$OUT/ref_saru"
    echo "built $OUT/ref_saru"
fi
