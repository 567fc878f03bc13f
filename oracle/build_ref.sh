#!/usr/bin/env bash
# Recipe for oracle/_ref/libvxref.so — TEST INFRASTRUCTURE ONLY.
#
# Compiles the reference's own hot-path CUDA sources, read in place from
# $VX_REFERENCE_ROOT/cuda (default /root/reference; nothing is copied into
# this repository), for sm_100a
# with the reference's default cargo features (forge-ntt, forge-ntt-batch,
# forge-fri, forge-permute: build.rs:214-244), and links them with
# ref_driver.cu (the prove_lean_inner orchestration restated over those
# launchers) and the C oracle's host transcript into one shared library.
# The .so is git-ignored and travels with the working tree.
set -euo pipefail
REF=${VX_REFERENCE_ROOT:-/root/reference}
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
NVCC=${NVCC:-nvcc}
if [ ! -d "$REF/cuda" ]; then
  echo "reference sources not found at $REF; skipping oracle/_ref" >&2
  exit 0
fi
mkdir -p "$OUT/obj"
ARCH="-gencode arch=compute_100a,code=sm_100a"
DEFS="-DFORGE_NTT=1 -DFORGE_NTT_BATCH=1 -DFORGE_FRI=1 -DFORGE_PERMUTE=1"
SRCS="circle_ntt circle_ntt_layer_forge circle_ntt_batch_forge twiddles batch_inverse constraint blake2s \
merkle_hash_leaves_forge fri fri_fold_line_forge fri_fold_circle_forge permute permute_forge \
merkle_leaves_lifted bit_reverse_wide accumulate_lift fields circle_ntt_stwo circle_ntt_stwo_batch pack_leaves grind grind_m31_output \
barycentric_eval gather"
pids=()
for s in $SRCS; do
  obj="$OUT/obj/$s.o"
  if [ ! -f "$obj" ] || [ "$REF/cuda/$s.cu" -nt "$obj" ]; then
    $NVCC $ARCH -O3 -Xcompiler -fPIC $DEFS -I"$REF/cuda/include" -c "$REF/cuda/$s.cu" -o "$obj" &
    pids+=($!)
  fi
done
for p in "${pids[@]}"; do wait "$p"; done
$NVCC $ARCH -O3 -std=c++17 -Xcompiler -fPIC -I"$HERE" -c "$HERE/ref_driver.cu" -o "$OUT/obj/ref_driver.o"
gcc -O3 -fPIC -fopenmp -std=c11 -c "$HERE/vx_oracle.c" -o "$OUT/obj/vx_oracle.o"
$NVCC $ARCH -shared -Xcompiler -fPIC -Xlinker -Bsymbolic "$OUT"/obj/*.o -lgomp -o "$OUT/libvxref.so"
echo "$OUT/libvxref.so"
