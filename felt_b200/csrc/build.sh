#!/usr/bin/env bash
# Builds libfelt_gpu.so (sm_100a) in-tree. Usage: build.sh [out_dir]
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="${1:-$HERE/..}"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
FLAGS=(-gencode arch=compute_100a,code=sm_100a -lineinfo -O3 -std=c++17 -fmad=false
       -Xcompiler -fPIC -Xcompiler -fvisibility=hidden --expt-relaxed-constexpr
       -I"$HERE/../include")
SRCS=(fg_engine.cu fg_polys.cu fg_ray.cu fg_image.cu fg_query.cu fg_capi.cu fg_prof.cu fg_noalloc.cu fg_server.cu fg_tune.cu)
OBJS=()
PIDS=()
mkdir -p "$OUT/_build"
for s in "${SRCS[@]}"; do
  o="$OUT/_build/${s%.cu}.o"
  if [[ ! -f "$o" || "$HERE/$s" -nt "$o" || -n "$(find "$HERE" -name '*.cuh' -newer "$o" -print -quit)" || -n "$(find "$HERE/../include" "$HERE/../../include" -newer "$o" -print -quit)" ]]; then
    "$NVCC" "${FLAGS[@]}" -c "$HERE/$s" -o "$o" &
    PIDS+=($!)
  fi
  OBJS+=("$o")
done
for p in "${PIDS[@]}"; do wait "$p"; done
"$NVCC" -gencode arch=compute_100a,code=sm_100a -shared -Xcompiler -fPIC "${OBJS[@]}" -o "$OUT/libfelt_gpu.so" -lcudart
echo "built $OUT/libfelt_gpu.so"
