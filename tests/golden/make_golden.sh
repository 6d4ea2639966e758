#!/bin/bash
# Regenerates the golden vectors from the reference's own code: builds
# oracle/_ref/ref_driver from the reference sources (oracle/build_ref.sh; ALENKA_REF
# names the checkout), then writes
#   ref_codec/<case>.seg     segment files written by the reference's pfor_compress
#   ref_codec/<case>.values  the values encoded (the reference's pfor_decompress
#                            returns exactly these; the driver checks it)
#   murmur64a.txt            "<seed> <hex bytes|-> <MurmurHash64A>" lines
#   like_gpu_regex.txt       the reference's LIKE matcher over fixed entries and patterns
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=$(cd "$HERE/../.." && pwd)
bash "$ROOT/oracle/build_ref.sh"
TMP=$(mktemp -d)
"$ROOT/oracle/_ref/ref_driver" codec "$TMP"
for f in "$TMP"/*.decoded; do
  b=$(basename "$f" .decoded)
  cmp -s "$f" "$TMP/$b.values" || { echo "reference decode differs for $b"; exit 1; }
done
mkdir -p "$HERE/ref_codec"
cp "$TMP"/*.seg "$TMP"/*.values "$HERE/ref_codec/"
"$ROOT/oracle/_ref/ref_driver" murmur "$HERE/murmur64a.txt"
"$ROOT/oracle/_ref/ref_driver" like "$HERE/like_gpu_regex.txt"
rm -rf "$TMP"
echo "golden vectors written to $HERE"
