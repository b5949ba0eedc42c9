#!/usr/bin/env bash
# Builds the REFERENCE CPU hex path from its own source files, where they lie under
# the read-only reference checkout, into oracle/_ref/ (git-ignored; travels with the
# repository snapshot).  No reference build system is run: g++ compiles the few
# translation units directly.  Test infrastructure only.
#
#   oracle/_ref/ice_generate_phase_cpu   reference CLI (hex_phase/apps/generate_hex_phase.cpp)
#   oracle/_ref/ref_hex_harness          oracle/ref_hex_harness.cpp over the same sources
#   oracle/_ref/ref_drop_harness         oracle/ref_drop_harness.cpp over the header-only drop
#                                        tracer, src/projected_area.cpp, src/water_refractive_index.cpp
#   oracle/_ref/ref_record_harness       oracle/ref_record_harness.cpp: one drop record's trace, binning
#                                        and stored CDF by the reference's drop intersector, Fresnel
#                                        split, PhaseMassAccumulator and build_host_cdf (the timed
#                                        reference arm)
#   oracle/_ref/ref_ice_harness          oracle/ref_ice_harness.cpp over hex_atlas/src/ice_optics.cpp
#   oracle/_ref/ref_atlas_harness        oracle/ref_atlas_harness.cpp over hex_atlas/src/atlas.cpp and
#                                        hex_trace/src/hex_trace.cpp (area rule, atlas nodes)
#   oracle/_ref/ice_precompute_atlas_cpu reference CLI (hex_atlas/apps/precompute_atlas.cpp), CPU build
#   oracle/_ref/ref_rainbow_harness      oracle/ref_rainbow_harness.cpp over the header-only Table-II
#                                        diffraction (include/rainbow/rainbow_diffraction.hpp)
#   oracle/_ref/ref_optics_harness       oracle/ref_optics_harness.cpp over the header-only patch optics
#                                        (include/rainbow/patch_optical_evaluator.hpp)
#   oracle/_ref/ref_patch_harness        oracle/ref_patch_harness.cpp over the header-only patch
#                                        construction (include/rainbow/patch_geometry.hpp)
#   oracle/_ref/ref_query_harness        oracle/ref_query_harness.cpp over the header-only ray / patch
#                                        intersection and query direction grid
#
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]   (default $ICP_REFERENCE_ROOT, else /root/reference)
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
ref="${1:-${ICP_REFERENCE_ROOT:-/root/reference}}"
out="$here/_ref"
if [ ! -d "$ref/hex_phase" ]; then
    echo "build_ref.sh: reference sources not found at $ref (prebuilt files in $out are used as-is)" >&2
    exit 0
fi
mkdir -p "$out"
flags=(-std=c++20 -O2 -fno-fast-math -ffp-contract=off
       -I"$ref/hex_trace/include" -I"$ref/hex_phase/include" -I"$ref/include")
srcs=("$ref/hex_phase/src/phase_table.cpp" "$ref/hex_phase/src/phase_generate.cpp"
      "$ref/hex_phase/src/orientation_plan.cpp" "$ref/hex_trace/src/hex_trace.cpp"
      "$ref/src/npy_writer.cpp")
g++ "${flags[@]}" "$ref/hex_phase/apps/generate_hex_phase.cpp" "${srcs[@]}" -o "$out/ice_generate_phase_cpu"
g++ "${flags[@]}" "$here/ref_hex_harness.cpp" "${srcs[@]}" -o "$out/ref_hex_harness"
g++ -std=c++20 -O2 -fno-fast-math -ffp-contract=off -I"$ref/include" "$here/ref_drop_harness.cpp" \
    "$ref/src/projected_area.cpp" "$ref/src/water_refractive_index.cpp" -o "$out/ref_drop_harness"
g++ "${flags[@]}" "$here/ref_record_harness.cpp" "$ref/hex_phase/src/phase_table.cpp" "$ref/src/npy_writer.cpp" \
    -o "$out/ref_record_harness"
g++ -std=c++20 -O2 -fno-fast-math -ffp-contract=off -I"$ref/include" "$here/ref_rainbow_harness.cpp" \
    -o "$out/ref_rainbow_harness"
g++ -std=c++20 -O2 -fno-fast-math -ffp-contract=off -I"$ref/include" "$here/ref_optics_harness.cpp" \
    -o "$out/ref_optics_harness"
g++ -std=c++20 -O2 -fno-fast-math -ffp-contract=off -I"$ref/include" "$here/ref_patch_harness.cpp" \
    -o "$out/ref_patch_harness"
g++ -std=c++20 -O2 -fno-fast-math -ffp-contract=off -I"$ref/include" "$here/ref_query_harness.cpp" \
    -o "$out/ref_query_harness"
if [ -f "$ref/hex_atlas/src/ice_optics.cpp" ]; then
    g++ -std=c++20 -O2 -fno-fast-math -ffp-contract=off -I"$ref/hex_atlas/include" "$here/ref_ice_harness.cpp" \
        "$ref/hex_atlas/src/ice_optics.cpp" -o "$out/ref_ice_harness"
    g++ "${flags[@]}" -I"$ref/hex_atlas/include" "$here/ref_atlas_harness.cpp" "$ref/hex_atlas/src/atlas.cpp" \
        "$ref/hex_trace/src/hex_trace.cpp" -o "$out/ref_atlas_harness"
    g++ "${flags[@]}" -I"$ref/hex_atlas/include" "$ref/hex_atlas/apps/precompute_atlas.cpp" \
        "$ref/hex_atlas/src/atlas.cpp" "$ref/hex_atlas/src/ice_optics.cpp" "$ref/hex_trace/src/hex_trace.cpp" \
        "$ref/src/npy_writer.cpp" -o "$out/ice_precompute_atlas_cpu"
fi
echo "built $out/ice_generate_phase_cpu $out/ref_hex_harness $out/ref_drop_harness $out/ref_record_harness $out/ref_ice_harness $out/ref_atlas_harness $out/ice_precompute_atlas_cpu $out/ref_rainbow_harness $out/ref_optics_harness $out/ref_patch_harness $out/ref_query_harness"
