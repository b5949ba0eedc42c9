// ref_query_harness.cpp -- drives the reference's ray / bilinear patch intersection
// (BilinearPatchIntersector::intersect, include/rainbow/bilinear_patch_intersection.hpp) and its
// query direction grid (QueryDirectionGrid, include/rainbow/query_direction_grid.hpp), compiled
// from the reference checkout by oracle/build_ref.sh.  Test infrastructure only.
//
//   ref_query_harness intersect IN OUT   IN: u32 n; n x (f32 corners[12], f32 direction[3])
//                                        OUT: n x BilinearRayHits (48 B)
//   ref_query_harness directions NT NP AX AY AZ EX EY EZ OUT
//                                        OUT: Vec3[NT * NP] (the reference's query directions)
#include <rainbow/bilinear_patch_intersection.hpp>
#include <rainbow/query_direction_grid.hpp>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

using namespace rainbow;

int main(int argc, char** argv)
{
    if (argc == 4 && !std::strcmp(argv[1], "intersect")) {
        FILE* in = std::fopen(argv[2], "rb");
        if (!in) return 3;
        std::uint32_t n = 0;
        if (std::fread(&n, 4, 1, in) != 1) return 4;
        std::vector<float> rows(size_t(n) * 15);
        if (std::fread(rows.data(), 4, rows.size(), in) != rows.size()) return 5;
        std::fclose(in);
        std::vector<BilinearRayHits> out(n);
        for (std::uint32_t i = 0; i < n; ++i) {
            const float* r = rows.data() + size_t(i) * 15;
            BilinearPatchGeometry g{};
            for (unsigned k = 0; k < 4; ++k) g.corners[k] = {r[3 * k], r[3 * k + 1], r[3 * k + 2]};
            out[i] = BilinearPatchIntersector::intersect(g, {r[12], r[13], r[14]});
        }
        FILE* o = std::fopen(argv[3], "wb");
        if (!o) return 6;
        std::fwrite(out.data(), sizeof(BilinearRayHits), n, o);
        return std::fclose(o) == 0 ? 0 : 7;
    }
    if (argc == 11 && !std::strcmp(argv[1], "directions")) {
        RaindropTraceConfig c{};
        c.incident_direction = {float(std::atof(argv[4])), float(std::atof(argv[5])), float(std::atof(argv[6]))};
        c.incident_basis_x = {float(std::atof(argv[7])), float(std::atof(argv[8])), float(std::atof(argv[9]))};
        const auto grid = QueryDirectionGrid::make(c, std::uint32_t(std::atoi(argv[2])), std::uint32_t(std::atoi(argv[3])));
        const auto d = grid.directions();
        FILE* o = std::fopen(argv[10], "wb");
        if (!o) return 6;
        std::fwrite(d.data(), sizeof(Vec3), d.size(), o);
        return std::fclose(o) == 0 ? 0 : 7;
    }
    std::fprintf(stderr, "usage: ref_query_harness intersect IN OUT | directions NT NP AX AY AZ EX EY EZ OUT\n");
    return 2;
}
