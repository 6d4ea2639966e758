#!/bin/bash
# Builds oracle/_ref/ref_driver from the reference's own sources in place
# (/root/reference/compress.cu and MurmurHash2_64.cu) for the CPU: Thrust's CPP device
# system plus the host shims in oracle/ref_shim (CUDA runtime calls -> host memory,
# the absent moderngpu headers, Thrust 2.x's removed pinned_allocator). Outputs go to
# oracle/_ref only. The rest of the reference (the operators) needs moderngpu, which
# the reference does not vendor, and is not built.
set -e
REF=${REF:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
[ -d "$REF" ] || { echo "reference sources not present; skipping"; exit 0; }
mkdir -p "$OUT"
FLAGS="-std=c++17 -O1 -DTHRUST_DEVICE_SYSTEM=THRUST_DEVICE_SYSTEM_CPP -DTHRUST_HOST_SYSTEM=THRUST_HOST_SYSTEM_CPP"
# the LIKE matcher (struct gpu_regex, filter.cu) is self-contained: its lines are cut from
# the reference file into the build folder and compiled for the host with the rest
sed -n '/^struct gpu_regex/,/^};/p' "$REF/filter.cu" > "$OUT/gpu_regex.inc"
g++ $FLAGS -I"$HERE/ref_shim" -I/usr/local/cuda/include -include "$HERE/ref_shim/cuda_host_shim.h" \
  -include algorithm -DREF_COMPRESS_CU="\"$REF/compress.cu\"" -DREF_GPU_REGEX="\"$OUT/gpu_regex.inc\"" \
  -c "$HERE/ref_driver.cpp" -o "$OUT/ref_driver.o"
g++ -O1 -include cstddef -x c++ -c "$REF/MurmurHash2_64.cu" -o "$OUT/murmur.o"
g++ -o "$OUT/ref_driver" "$OUT/ref_driver.o" "$OUT/murmur.o"
echo "built $OUT/ref_driver"
