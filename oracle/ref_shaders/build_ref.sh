#!/bin/sh
# Builds oracle/_ref/libref_shaders.so: the reference's raster, grid-build
# and VoxelBVH-ingestion shaders compiled as C++ straight from the reference checkout.  Test
# infrastructure only; the outputs are git-ignored and nothing in the product
# links them.  The only source change is mechanical and made on the fly:
# Slang attributes / system-value semantics are stripped and the `.xxx`
# scalar swizzle is spelled as a float3 broadcast.  Skips (exit 0) when the
# reference checkout is absent.
set -e
HERE="$(cd "$(dirname "$0")" && pwd)"
# the reference checkout: VOX_REFERENCE_DIR, else a sibling of this repository
REF="${VOX_REFERENCE_DIR:-$HERE/../../../reference}"
OUT="$HERE/../_ref"
if [ ! -d "$REF/raster/shaders" ]; then
    echo "reference checkout not found at $REF; skipping oracle/_ref"
    exit 0
fi
mkdir -p "$OUT"
for s in gaussian_prim gaussian_frag_alloc gaussian_frag_color fanout_scatter_prim_idxs fanout_compute_fragment_idxs; do
    sed -e '/^#define PNANOVDB_/d' \
        -e '/^#include "PNanoVDB/d' \
        -e 's/\[require([^]]*)\]//g' \
        -e 's/\[shader("compute")\]//g' \
        -e 's/\[numthreads([^]]*)\]//g' \
        -e 's/ : SV_Group[A-Za-z]*//g' \
        -e 's/\([A-Za-z_][A-Za-z_0-9.]*\)\.xxx/float3(\1)/g' \
        "$REF/raster/shaders/$s.slang" > "$OUT/$s.inc"
done
# VoxelBVH Gaussian ingestion; `.xyz` reads of a float4 become `.xyz()`
for s in voxelbvh_gaussians_to_ijkl voxelbvh_find_range_starts voxelbvh_scatter_range_headers; do
    sed -e 's/\[shader("compute")\]//g' \
        -e 's/\[numthreads([^]]*)\]//g' \
        -e 's/ : SV_Group[A-Za-z]*//g' \
        -e 's/\.xyz\b/.xyz()/g' \
        "$REF/raster/shaders/voxelbvh/$s.slang" > "$OUT/$s.inc"
done
# Grid build (raster/GridBuild.cpp:361-650): the node2 part of PNanoVDBExt.h is
# used unchanged (compiled without PNANOVDB_C, which leaves out its NanoVDB
# conversion section); the shaders lose their PNanoVDB includes (the shim
# pnanovdb_gridbuild.h supplies generic primitives and stubs the header calls),
# include the copied workgroup_scan, and HLSL `inout T x` becomes `T& x`.
cp "$REF/nanovdb_editor/PNanoVDBExt.h" "$OUT/PNanoVDBExt.inc"
for s in grid_build_init grid_build_set_masks grid_build_count_new grid_build_scatter_new grid_build_finalize \
         grid_build_blindmetadata grid_build_compute_bbox workgroup_scan; do
    sed -e '/^#define PNANOVDB_/d' \
        -e '/^#include "PNanoVDB/d' \
        -e 's/#include <workgroup_scan.slang>/#include "workgroup_scan.inc"/' \
        -e 's/\[require([^]]*)\]//g' \
        -e 's/\[shader("compute")\]//g' \
        -e 's/\[numthreads([^]]*)\]//g' \
        -e 's/ : SV_Group[A-Za-z]*//g' \
        -e 's/inout \([A-Za-z_][A-Za-z_0-9]*\) /\1\& /g' \
        "$REF/raster/shaders/$s.slang" > "$OUT/$s.inc"
done
${CXX:-g++} -O2 -fPIC -std=c++17 -ffp-contract=off -w -Wno-narrowing \
    -I"$HERE" -I"$HERE/../../include" -I"$OUT" \
    -shared -o "$OUT/libref_shaders.so" "$HERE/ref_driver.cpp" "$HERE/ref_gridbuild.cpp"
echo "built $OUT/libref_shaders.so"
