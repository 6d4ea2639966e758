#!/bin/bash
# Builds, from the reference's own sources in place (ALENKA_REF, default
# /root/reference), for the CPU:
#   oracle/_ref/ref_driver  its codec (compress.cu), MurmurHash64A and LIKE matcher,
#                           driven by oracle/ref_driver.cpp to write golden vectors
#   oracle/_ref/alenka_ref  the whole reference CLI (bison front end, operators, codec)
#                           under Thrust's OpenMP device system (oracle/ref.mk)
#   oracle/_ref/alenka_frontend, frontend_dump
#                           the reference's front end (parser, CLI) linked against
#                           alenka_b200/libalenka_b200.so instead of its operators
# The host shims in oracle/ref_shim stand in for the CUDA runtime calls (host memory),
# Thrust 2.x's removed pinned_allocator and the moderngpu primitives the reference does
# not vendor. Outputs go to oracle/_ref only.
set -e
REF=${ALENKA_REF:-/root/reference}
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
# the whole reference (bison front end, operators, codec) for the CPU: oracle/_ref/alenka_ref;
# and its front end linked against alenka_b200/libalenka_b200.so (built first):
# oracle/_ref/alenka_frontend and oracle/_ref/frontend_dump
make -s -j"$(nproc)" -f "$HERE/ref.mk" REF="$REF" "$OUT/alenka_ref" frontend
echo "built $OUT/alenka_ref, $OUT/alenka_frontend, $OUT/frontend_dump"
