#!/bin/bash
# Makes a scratch copy of the reference's LONESTAR tree that compiles with
# CUDA 12 for sm_100a, so that the reference's own harness sources (skel.cu,
# apps/*/support.cu, rt/src/*.cu, moderngpu's context) can be linked with this
# library's gg_main.  The reference tree itself is only read.
#
#   usage: lonestar_tree.sh <reference LONESTAR dir> <scratch dir>
#
# The copy gets six source-level shims.  The first five are needed only because
# the tree was written for CUDA 8-11 and later hipified in place:
#   1. every *.prehip file (the CUDA original) is copied over its hipified twin;
#   2. moderngpu's util/mgpucontext.h and util/mgpualloc.h, hipified with no
#      .prehip original, get their hip* names mapped back to cuda*;
#   3. cub/cub.cuh stops including the texture-reference iterator (texture
#      references were removed in CUDA 12);
#   4. calls of the pre-Volta warp intrinsics __ballot/__any/__all/__shfl*
#      become their *_sync forms over __activemask(), which is what the
#      implicit-mask originals meant (CUDA 12 rejects them for sm_70+);
#   5. CUB 1.3.2's inline-PTX shfl.{up,down,idx}.b32 become shfl.sync over
#      the active mask.
# The sixth touches only the reference's own traversal kernels
# (apps/*/kernel_*.cu), which baseline/build.sh compiles; this library's
# gg_main does not use them:
#   6. their worklists get 4 x (edges + vertices) slots instead of n (BFS),
#      2m (SSSP) or m (PR).  BFS marks a vertex with a plain load/compare/store,
#      so racing parents can queue it more than once in one level; the queue
#      reservation checks only its first slot against the capacity (an assert),
#      so an overfull level writes past the array.  The slot count changes no
#      result.
# Test, example and tuning programs in the tree are left alone.
set -euo pipefail
SRC=${1:?reference LONESTAR dir}
DST=${2:?scratch dir}
if [ ! -d "$SRC/skelapp" ]; then
  echo "no Lonestar tree at $SRC" >&2
  exit 1
fi
STAMP="$DST/.gsrb_tree_stamp"
SELF_SUM=$(cksum < "$0")
if [ -f "$STAMP" ] && [ "$(cat "$STAMP")" = "$SELF_SUM" ]; then
  exit 0
fi
rm -rf "$DST"
mkdir -p "$(dirname "$DST")"
cp -r "$SRC" "$DST"
chmod -R u+w "$DST"
cd "$DST"

# 1
find . -name '*.prehip' -print0 | while IFS= read -r -d '' f; do cp "$f" "${f%.prehip}"; done

# 2
for h in include/mgpu/include/util/mgpucontext.h include/mgpu/include/util/mgpualloc.h; do
  sed -i -e 's#hip/hip_runtime\.h#cuda_runtime.h#' -e 's/hipDeviceProp_t/cudaDeviceProp/g' \
         -e 's/\bhip\([A-Z]\)/cuda\1/g' "$h"
done

# 3
sed -i '/iterator\/tex_ref_input_iterator\.cuh/d' rt/include/cub/cub/cub.cuh

# 4
find rt/include apps include/mgpu/include \
     \( -name '*.cu' -o -name '*.cuh' -o -name '*.h' -o -name '*.hpp' \) \
     -not -path '*/test/*' -not -path '*/examples/*' -not -path '*/tune/*' \
     -not -path '*/experimental/*' -not -path '*/hip/*' -print0 |
  xargs -0 sed -i -E \
     -e 's/(^|[^_a-zA-Z0-9])__(ballot|any|all)\(/\1__\2_sync(__activemask(), /g' \
     -e 's/(^|[^_a-zA-Z0-9])__shfl(_up|_down|_xor)?\(/\1__shfl\2_sync(__activemask(), /g'

# 5
for f in rt/include/cub/cub/util_ptx.cuh \
         rt/include/cub/cub/warp/specializations/warp_reduce_shfl.cuh \
         rt/include/cub/cub/warp/specializations/warp_scan_shfl.cuh; do
  sed -i -E 's/shfl\.(up|down|idx)\.b32 ([^;]*);/{ .reg .b32 gsrbm; activemask.b32 gsrbm; shfl.sync.\1.b32 \2, gsrbm; }/g' "$f"
done

# 6
for f in apps/bfs/kernel_*.cu apps/sssp/kernel_*.cu apps/pr/kernel_*.cu; do
  sed -i -E 's/PipeContextT<Worklist2>\((gg\.nnodes|gg\.nedges\*2|hg\.nedges)\)/PipeContextT<Worklist2>((size_t)4 * ((size_t)gg.nedges + gg.nnodes))/' "$f"
done

echo "$SELF_SUM" > "$STAMP"
echo "scratch Lonestar tree ready at $DST"
