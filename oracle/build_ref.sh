#!/bin/bash
# Builds the reference's own gsi (FIST-CMS/General-Simulator) into oracle/_ref/
# as an executed cross-check of the oracle.  The reference tree ships with
# unresolved merge conflicts and a C++17 hang, so the recipe works on a copy
# under /tmp (never inside this repository):
#   1. keep the HEAD side of every conflict block (<<<<<<< HEAD .. =======),
#      drop the origin side (======= .. >>>>>>> origin/master);
#   2. src/input.cu: "p=p++;" -> "p++;" (under C++17 the original statement
#      leaves p unchanged and INPUT::standardize never ends on {..} scripts);
#   3. nvcc -O2 for sm_100a, -lcurand -lcufft, as the reference's makefile.
# The binary only runs on a GPU box; it is test infrastructure.
# Usage: REF=<path of the reference tree> oracle/build_ref.sh
set -e
if [ -z "$REF" ]; then echo "set REF to the reference tree (the directory holding src/ and include/)"; exit 1; fi
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
if [ ! -d "$REF/src" ]; then echo "reference tree not found at $REF"; exit 1; fi
TMP=$(mktemp -d /tmp/gsref.XXXXXX)
cp -r "$REF/src" "$REF/include" "$TMP/"
for f in $(grep -rl '^<<<<<<< ' "$TMP/src" "$TMP/include"); do
  awk 'BEGIN{s=0} /^<<<<<<< /{s=1;next} /^=======/{if(s==1){s=2;next}} /^>>>>>>> /{if(s==2){s=0;next}} {if(s!=2)print}' \
    "$f" > "$f.tmp" && mv "$f.tmp" "$f"
done
sed -i 's/p=p++;/p++;/' "$TMP/src/input.cu"
mkdir -p "$OUT"
cd "$TMP/src"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
objs=""
for c in *.cu; do
  "$NVCC" -O2 -gencode arch=compute_100a,code=sm_100a -w -c "$c" -o "${c%.cu}.o" &
  objs="$objs ${c%.cu}.o"
done
wait
"$NVCC" -O2 -gencode arch=compute_100a,code=sm_100a -o "$OUT/gsi" $objs -lcurand -lcufft
rm -rf "$TMP"
echo "built $OUT/gsi"
