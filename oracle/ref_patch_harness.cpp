// ref_patch_harness.cpp -- drives the reference's patch construction
// (PatchConstruction::make, include/rainbow/patch_geometry.hpp, compiled from the reference
// checkout by oracle/build_ref.sh) over a vertex lattice written by the tests, with the
// compaction order of device/patch_build.cu (patch_id order).  Test infrastructure only.
//
//   ref_patch_harness IN OUT
//   IN : u32 width, height; f32 half_extent; OutgoingVertex[4 * width * height]
//   OUT: u32 status[cell_count]; u32 count; u32 histogram[8]; OutgoingPatch[count]; PatchAabb[count]
#include <rainbow/patch_geometry.hpp>

#include <cstdio>
#include <vector>

using namespace rainbow;

int main(int argc, char** argv)
{
    if (argc != 3) {
        std::fprintf(stderr, "usage: ref_patch_harness IN OUT\n");
        return 2;
    }
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 3;
    std::uint32_t wh[2];
    float extent;
    if (std::fread(wh, 4, 2, in) != 2 || std::fread(&extent, 4, 1, in) != 1) return 4;
    RaindropTraceConfig config{};
    config.grid_width = wh[0];
    config.grid_height = wh[1];
    config.grid_half_extent = extent;
    PatchBuildLayout layout{};
    if (!PatchBuildLayout::try_make(config, layout)) return 5;
    std::vector<OutgoingVertex> vertices(4ull * layout.vertices_per_path);
    if (std::fread(vertices.data(), sizeof(OutgoingVertex), vertices.size(), in) != vertices.size()) return 6;
    std::fclose(in);
    std::vector<std::uint32_t> status(layout.cell_count);
    std::vector<OutgoingPatch> patches;
    std::vector<PatchAabb> boxes;
    std::uint32_t histogram[8] = {};
    for (std::uint32_t id = 0; id < layout.cell_count; ++id) {
        const auto r = PatchConstruction::make(vertices.data(), layout, id);
        status[id] = static_cast<std::uint32_t>(r.patch.status);
        ++histogram[status[id]];
        if (has_patch_geometry(r.patch.status)) {
            patches.push_back(r.patch);
            boxes.push_back(r.aabb);
        }
    }
    FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 7;
    const std::uint32_t count = std::uint32_t(patches.size());
    std::fwrite(status.data(), 4, status.size(), o);
    std::fwrite(&count, 4, 1, o);
    std::fwrite(histogram, 4, 8, o);
    std::fwrite(patches.data(), sizeof(OutgoingPatch), patches.size(), o);
    std::fwrite(boxes.data(), sizeof(PatchAabb), boxes.size(), o);
    return std::fclose(o) == 0 ? 0 : 8;
}
