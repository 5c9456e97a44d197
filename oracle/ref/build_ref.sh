#!/usr/bin/env bash
# Builds the reference's own CPU code for this path into oracle/_ref/ so the
# oracle restatement can be checked against it.  Test infrastructure only.
#
# What is built (all outputs go to oracle/_ref/, which git ignores):
#   td_ref               TopDown-rtree.cu compiled unchanged with nvcc.  Run with
#                        no visible GPU, its CUDA calls fail and only its CPU
#                        build (TD:572-627) and CPU DFS query (TD:776-798) run;
#                        it prints their timings and digests.
#   libref_bu_m{F}.so    Host build of BotomUp-rtree.cu's CPU path: the key
#                        kernel and Interleave (BU:73-123, run on one emulated
#                        thread), the min-shift/scale block (BU:704-721), qsort +
#                        packing (BU:780-830), and RtreeSearch / Overlap /
#                        RtreeSearch1 (BU:439-590), at fanout m = F.
#   libref_td_m{F}.so    Host build of TopDown-rtree.cu's level offsets
#                        (TD:504-524), CPU build (TD:575-624) and RtreeSearch /
#                        RtreeSearch1 (TD:56-93), at fanout M = F.
#   libref_gpc.so        Host build of the reference's GPC clip core
#                        (vector_map_overlay_gpc_kernel.cu:115-750, 890-1709).
#   libref_readdata.so   Host build of readData, the polygon file reader
#                        (vector_map_overlay_gpc_kernel.cu:752-888), with its
#                        cudaMalloc / cudaMemcpy as host allocations and copies.
#
# The reference files are read where they lie; the line ranges below are
# extracted into oracle/_ref/*.slice.inc (build intermediates, never committed)
# and compiled together with the project-written shim headers and harnesses in
# this directory.  Each range is checked against a marker string first, so a
# changed reference fails loudly instead of compiling the wrong lines.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$(cd "$HERE/.." && pwd)/_ref"
REF="${PRT_REFERENCE_DIR:-/root/reference}"
BU="$REF/BotomUp-rtree.cu"
TD="$REF/TopDown-rtree.cu"
GPC="$REF/vector_map_overlay_gpc_kernel.cu"
mkdir -p "$OUT"
for f in "$BU" "$TD" "$GPC"; do
  [ -r "$f" ] || { echo "build_ref: missing $f" >&2; exit 1; }
done

# slice FILE FIRST LAST MARKER : print lines FIRST..LAST after checking that
# line FIRST contains MARKER.
slice() {
  local file="$1" first="$2" last="$3" marker="$4"
  if ! sed -n "${first}p" "$file" | grep -qF -- "$marker"; then
    echo "build_ref: $file:$first does not contain '$marker'" >&2
    exit 1
  fi
  echo "#line $first \"$file\""
  sed -n "${first},${last}p" "$file"
}

CXXFLAGS="-O2 -fPIC -shared -ffp-contract=off -w"

# ---- BU (bottom-up) CPU path ------------------------------------------------
{
  slice "$BU" 12 16 "#define LEAF 0"
  slice "$BU" 18 20 "#define datatype bounding_box"
  slice "$BU" 25 54 "typedef struct key"
  slice "$BU" 57 70 "CalcuateZOrderValue(bounding_box"
  slice "$BU" 73 123 "__global__ void CalcuateZOrderValue"
  slice "$BU" 439 559 "int RtreeSearch(rtree_node"
  slice "$BU" 574 590 "int RtreeSearch1(rtree_node"
  slice "$BU" 632 640 "void ResetMBR1"
} > "$OUT/bu_defs.slice.inc"
{
  slice "$BU" 704 721 "for (i= 0; i < num_contours; i++) {"
} > "$OUT/bu_shift.slice.inc"
{
  slice "$BU" 780 830 "qsort(pointers,num_contours"
} > "$OUT/bu_pack.slice.inc"
for F in 10 16 32; do
  g++ $CXXFLAGS -Dm=$F -DM=$((2*F-1)) -I"$HERE" -I"$OUT" \
      -o "$OUT/libref_bu_m$F.so" "$HERE/bu_ref_harness.cpp"
done

# ---- TD (top-down) CPU path --------------------------------------------------
{
  slice "$TD" 10 10 "#define MINERROR"
  slice "$TD" 15 39 "struct MBR{"
  slice "$TD" 56 93 "int RtreeSearch(int * nodes_index"
} > "$OUT/td_defs.slice.inc"
{
  slice "$TD" 504 524 "int b = 1;"
} > "$OUT/td_offsets.slice.inc"
{
  slice "$TD" 575 624 "while(p < offset.size() - 1){"
} > "$OUT/td_build.slice.inc"
for F in 10 16 32; do
  g++ $CXXFLAGS -DM=$F -I"$HERE" -I"$OUT" \
      -o "$OUT/libref_td_m$F.so" "$HERE/td_ref_harness.cpp"
done

# ---- GPC clip core -------------------------------------------------------------
{
  slice "$GPC" 115 750 "__device__ void gpc_polygon_clip"
  slice "$GPC" 890 1709 "__device__ void gpc_free_polygon"
} > "$OUT/gpc_core.slice.inc"
g++ $CXXFLAGS -I"$HERE" -I"$OUT" -o "$OUT/libref_gpc.so" "$HERE/gpc_ref_harness.cpp"

# ---- readData (the polygon file reader) ------------------------------------------
{
  slice "$GPC" 752 888 "void readData(char * base_filename"
} > "$OUT/readdata.slice.inc"
g++ $CXXFLAGS -I"$HERE" -I"$OUT" -o "$OUT/libref_readdata.so" "$HERE/readdata_harness.cpp"

# ---- TD program, unchanged -------------------------------------------------------
if command -v nvcc >/dev/null 2>&1; then
  nvcc -O2 -w -gencode arch=compute_100a,code=sm_100a -o "$OUT/td_ref" "$TD"
fi
# the slices are build intermediates only: drop them once compiled
rm -f "$OUT"/*.slice.inc
echo "build_ref: ok -> $OUT"
