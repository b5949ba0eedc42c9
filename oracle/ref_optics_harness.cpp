// ref_optics_harness.cpp -- drives the reference's per-direction optics
// (PatchOpticalEvaluator::evaluate_direction, include/rainbow/patch_optical_evaluator.hpp,
// compiled from the reference checkout by oracle/build_ref.sh) on inputs written by the tests'
// fixture generator.  Test infrastructure only: its outputs pin the CPU oracle.
//
//   ref_optics_harness IN OUT [folded]
//   IN : u64 hit_storage_count; u32 vertex_count, patch_count, direction_count,
//        second_input_count, input_polarization, with_focal; f32 incident[3], basis_x[3];
//        FocalPhaseConfig; OutgoingVertex[vertex_count]; OutgoingPatch[patch_count];
//        Vec3[direction_count]; u64 offsets[direction_count + 1];
//        PatchQuerySummary[direction_count]; PatchQueryHit[hit_storage_count];
//        Field32[second_input_count]
//   OUT: PatchOpticalResult[direction_count], then FocalOpticalResult[direction_count]
//        when with_focal
//   With "folded": every NeedsRefinement patch first gets its FoldedPatchRecord
//   (FoldedPatchBuilder::prepare, the default FoldedPatchConfig, focal estimates when with_focal),
//   in compact-index order, and the directions are evaluated with that FoldedPatchView (the
//   reference's evaluate_folded_optics); OUT then continues with u32 record_count,
//   u32 record_indices[patch_count], FoldedPatchRecord[record_count].
#include <rainbow/folded_patch_builder.hpp>
#include <rainbow/patch_optical_evaluator.hpp>

#include <cstring>

#include <cstdio>
#include <vector>

using namespace rainbow;

template <class T> static bool read_n(FILE* f, std::vector<T>& v, size_t n)
{
    v.resize(n);
    return n == 0 || std::fread(v.data(), sizeof(T), n, f) == n;
}

int main(int argc, char** argv)
{
    const bool with_folded = argc == 4 && std::strcmp(argv[3], "folded") == 0;
    if (argc != 3 && !with_folded) {
        std::fprintf(stderr, "usage: ref_optics_harness IN OUT [folded]\n");
        return 2;
    }
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 3;
    std::uint64_t storage = 0;
    std::uint32_t head[6];
    float dirs[6];
    FocalPhaseConfig focal{};
    if (std::fread(&storage, 8, 1, in) != 1 || std::fread(head, 4, 6, in) != 6 || std::fread(dirs, 4, 6, in) != 6 ||
        std::fread(&focal, sizeof focal, 1, in) != 1)
        return 4;
    std::vector<OutgoingVertex> vertices;
    std::vector<OutgoingPatch> patches;
    std::vector<Vec3> directions;
    std::vector<std::uint64_t> offsets;
    std::vector<PatchQuerySummary> summaries;
    std::vector<PatchQueryHit> hits;
    std::vector<Field32> second;
    if (!read_n(in, vertices, head[0]) || !read_n(in, patches, head[1]) || !read_n(in, directions, head[2]) ||
        !read_n(in, offsets, size_t(head[2]) + 1) || !read_n(in, summaries, head[2]) || !read_n(in, hits, storage) ||
        !read_n(in, second, head[3]))
        return 5;
    std::fclose(in);
    PatchOpticsParams p{};
    p.vertices = vertices.data();
    p.patches = patches.data();
    p.directions = directions.data();
    p.offsets = offsets.data();
    p.summaries = summaries.data();
    p.hits = hits.data();
    p.hit_storage_count = storage;
    p.vertex_count = head[0];
    p.patch_count = head[1];
    p.direction_count = head[2];
    p.second_input_fields = head[3] ? second.data() : nullptr;
    p.second_input_count = head[3];
    p.input_polarization = static_cast<IncidentPolarization>(head[4]);
    p.incident_direction = {dirs[0], dirs[1], dirs[2]};
    p.incident_basis_x = {dirs[3], dirs[4], dirs[5]};
    std::vector<std::uint32_t> indices(patches.size(), 0xffffffffu);
    std::vector<FoldedPatchRecord> records;
    FoldedPatchView view{};
    if (with_folded) {
        for (std::uint32_t i = 0; i < patches.size(); ++i) {
            if (patches[i].status != PatchCellStatus::NeedsRefinement) continue;
            indices[i] = std::uint32_t(records.size());
            records.push_back(FoldedPatchBuilder::prepare(vertices.data(), head[0], patches[i], i, p.incident_direction,
                                                          head[5] ? &focal : nullptr, FoldedPatchConfig{}));
        }
        view = {indices.data(), records.data(), std::uint32_t(patches.size()), std::uint32_t(records.size())};
    }
    std::vector<PatchOpticalResult> out(head[2]);
    std::vector<FocalOpticalResult> fout(head[2]);
    for (std::uint32_t i = 0; i < head[2]; ++i)
        out[i] = head[5] ? PatchOpticalEvaluator::evaluate_direction(p, i, &focal, &fout[i], view)
                         : PatchOpticalEvaluator::evaluate_direction(p, i, nullptr, nullptr, view);
    FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 6;
    std::fwrite(out.data(), sizeof(PatchOpticalResult), out.size(), o);
    if (head[5]) std::fwrite(fout.data(), sizeof(FocalOpticalResult), fout.size(), o);
    if (with_folded) {
        const std::uint32_t n = std::uint32_t(records.size());
        std::fwrite(&n, 4, 1, o);
        std::fwrite(indices.data(), 4, indices.size(), o);
        std::fwrite(records.data(), sizeof(FoldedPatchRecord), records.size(), o);
    }
    return std::fclose(o) == 0 ? 0 : 7;
}
