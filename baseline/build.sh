#!/bin/bash
# Builds the reference's own GPU programs for sm_100a, straight from the
# reference sources, into baseline/_ref/ (git-ignored; travels with the tree).
# They are the baseline that the new build is timed against and the source of
# the golden outputs for graph parity (tests/golden/make_ref_lonestar.py);
# nothing in the library links or calls them.
#
#   reduce_{gsrb,gcpusrb,ccg}   Reduce/test_reduce.cu + Reduce/reduce_<v>.cu
#                    (Reduce/compile.sh, for sm_100a)
#   scan_{gsrb,gcpusrb,ccg}     scan/main.cu + scan/scan_<v>.cu (scan/compile.sh)
#   allSyncPrims-1kernel        Heterosync/main.cu (Heterosync/Makefile, -rdc)
#   lonestar/{bfs,sssp,pr}_{gsrb,gcpusrb,ccg}
#                    LONESTAR/apps/<app>/kernel_<v>.cu + support.cu + skel.cu +
#                    rt/src + moderngpu context (apps/bfs/compile.sh), compiled
#                    from the scratch copy that
#                    tpds22-artifact_b200/dropin/lonestar_tree.sh makes (CUDA-12
#                    shims), plus cuda12_cdp_removed.h force-included for the
#                    kernel files.
# The GSRB / GCPUSRB forms spin on their barriers without a bound: run them
# only with grids the occupancy calculator confirms co-resident.
#
#   usage: baseline/build.sh [reference root]   (default: $GSRB_REFERENCE_ROOT, else /root/reference)
set -euo pipefail
REF=${1:-${GSRB_REFERENCE_ROOT:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
ARCH="-gencode arch=compute_100a,code=sm_100a"
TREE=${GSRB_LONESTAR_TREE:-/tmp/gsrb_lonestar_tree}
if [ ! -d "$REF/scan" ]; then
  echo "reference tree not found at $REF; skipping baseline/_ref" >&2
  exit 0
fi
mkdir -p "$OUT" "$OUT/lonestar"

newer() {  # newer <target> <sources...>: true when the target must be rebuilt
  local t=$1 f; shift
  [ -e "$t" ] || return 0
  for f in "$@"; do [ "$f" -nt "$t" ] && return 0; done
  return 1
}

pids=()
for v in gsrb gcpusrb ccg; do
  if newer "$OUT/reduce_$v" "$REF/Reduce/reduce_$v.cu" "$0"; then
    "$NVCC" -O3 -w $ARCH -rdc=true -I"$REF/Reduce" "$REF/Reduce/reduce_$v.cu" "$REF/Reduce/test_reduce.cu" \
      -o "$OUT/reduce_$v" & pids+=($!)
  fi
  if newer "$OUT/scan_$v" "$REF/scan/scan_$v.cu" "$0"; then
    "$NVCC" -O3 -w $ARCH -rdc=true -I"$REF/scan" "$REF/scan/scan_$v.cu" "$REF/scan/main.cu" \
      -o "$OUT/scan_$v" & pids+=($!)
  fi
done
if newer "$OUT/allSyncPrims-1kernel" "$REF/Heterosync/main.cu" "$0"; then
  "$NVCC" -O3 -w $ARCH -rdc=true -I"$REF/Heterosync" "$REF/Heterosync/main.cu" \
    -o "$OUT/allSyncPrims-1kernel" & pids+=($!)
fi

# Lonestar: the scratch copy with the CUDA-12 shims, then the reference's link line
bash "$HERE/../tpds22-artifact_b200/dropin/lonestar_tree.sh" "$REF/LONESTAR" "$TREE"
LSG="-O3 -w -std=c++14 $ARCH -DTHRUST_IGNORE_CUB_VERSION_CHECK -I$TREE/rt/include -I$TREE/rt/include/mgpu/include -I$TREE/rt/include/cub"
O=${GSRB_REF_OBJ:-/tmp/gsrb_ref_obj}
mkdir -p "$O"
build_obj() {  # build_obj <out> <source> [extra flags]
  local o=$1 s=$2; shift 2
  if newer "$o" "$s" "$TREE/.gsrb_tree_stamp" "$0"; then "$NVCC" $LSG "$@" -dc "$s" -o "$o"; fi
}
build_obj "$O/skel.o" "$TREE/skelapp/skel.cu" & pids+=($!)
for s in csr_graph ggc_rt instr; do build_obj "$O/$s.o" "$TREE/rt/src/$s.cu" & pids+=($!); done
build_obj "$O/mgpucontext.o" "$TREE/include/mgpu/src/mgpucontext.cu" & pids+=($!)
build_obj "$O/mgpuutil.o" "$TREE/include/mgpu/src/mgpuutil.cpp" & pids+=($!)
if newer "$O/bmk2.o" "$TREE/rt/src/bmk2.c"; then gcc -O3 -c -I"$TREE/rt/include" "$TREE/rt/src/bmk2.c" -o "$O/bmk2.o"; fi
for a in bfs sssp pr; do
  build_obj "$O/${a}_support.o" "$TREE/apps/$a/support.cu" & pids+=($!)
  for v in gsrb gcpusrb ccg; do
    build_obj "$O/${a}_$v.o" "$TREE/apps/$a/kernel_$v.cu" -include "$HERE/cuda12_cdp_removed.h" & pids+=($!)
  done
done
for p in "${pids[@]}"; do wait "$p"; done

HARNESS="$O/skel.o $O/csr_graph.o $O/ggc_rt.o $O/instr.o $O/mgpucontext.o $O/mgpuutil.o $O/bmk2.o"
for a in bfs sssp pr; do
  for v in gsrb gcpusrb ccg; do
    t="$OUT/lonestar/${a}_$v"
    if newer "$t" "$O/${a}_$v.o" "$O/${a}_support.o" "$O/skel.o"; then
      "$NVCC" $ARCH -o "$t" "$O/${a}_$v.o" "$O/${a}_support.o" $HARNESS -lcurand -lcudadevrt -lz
    fi
  done
done
echo "built the reference programs into $OUT"
