// ref_rainbow_harness.cpp -- drives the reference's Table-II diffraction
// (include/rainbow/rainbow_diffraction.hpp, compiled from the reference checkout by
// oracle/build_ref.sh) on inputs written by the tests' fixture generator.  Test
// infrastructure only: it produces the expected outputs that pin the CPU oracle.
//
//   ref_rainbow_harness table                 stdin: one radius (float) per line
//                                             stdout: "ok sigma" per line, sigma as %a
//   ref_rainbow_harness grid IN OUT           IN:  u32 nt, u32 np, f64 cfg[4], u32 has_edges,
//                                                  u32 pad, FocalOpticalResult[nt*np],
//                                                  then u32 edges[nt*np] when has_edges
//                                             OUT: u32 edges[nt*np] (the given ones, or
//                                                  detect()'s), DiffractionResult[nt*np]
#include <rainbow/rainbow_diffraction.hpp>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

using namespace rainbow;

static bool read_exact(FILE* f, void* p, size_t n) { return std::fread(p, 1, n, f) == n; }

int main(int argc, char** argv)
{
    if (argc >= 2 && !std::strcmp(argv[1], "table")) {
        float r;
        while (std::scanf("%f", &r) == 1) {
            double s = -1;
            const bool ok = RainbowDiffraction::table_sigma_degrees(r, s);
            std::printf("%d %a\n", ok ? 1 : 0, s);
        }
        return 0;
    }
    if (argc != 4 || std::strcmp(argv[1], "grid")) {
        std::fprintf(stderr, "usage: ref_rainbow_harness table | grid IN OUT\n");
        return 2;
    }
    FILE* in = std::fopen(argv[2], "rb");
    if (!in) return 3;
    std::uint32_t head[2], flags[2];
    double cfg[4];
    if (!read_exact(in, head, sizeof head) || !read_exact(in, cfg, sizeof cfg) || !read_exact(in, flags, sizeof flags))
        return 4;
    const size_t n = size_t(head[0]) * head[1];
    std::vector<FocalOpticalResult> focal(n);
    std::vector<RainbowTransition> edges(n);
    std::vector<DiffractionResult> out(n);
    if (!read_exact(in, focal.data(), n * sizeof(FocalOpticalResult))) return 5;
    DiffractionParams p{};
    p.focal = focal.data();
    p.transitions = edges.data();
    p.results = out.data();
    p.theta_count = head[0];
    p.phi_count = head[1];
    p.config = {cfg[0], cfg[1], cfg[2], cfg[3]};
    if (flags[0]) {
        if (!read_exact(in, edges.data(), n * sizeof(RainbowTransition))) return 6;
    } else {
        for (size_t i = 0; i < n; ++i) edges[i] = RainbowDiffraction::detect(p, std::uint32_t(i));
    }
    std::fclose(in);
    for (size_t i = 0; i < n; ++i) out[i] = RainbowDiffraction::filter(p, std::uint32_t(i));
    FILE* o = std::fopen(argv[3], "wb");
    if (!o) return 7;
    std::fwrite(edges.data(), sizeof(RainbowTransition), n, o);
    std::fwrite(out.data(), sizeof(DiffractionResult), n, o);
    return std::fclose(o) == 0 ? 0 : 8;
}
