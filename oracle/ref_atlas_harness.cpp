// ref_atlas_harness.cpp -- drives the REFERENCE deterministic atlas precompute
// (hex_atlas/src/atlas.cpp over hex_trace, compiled from the reference's own sources by
// oracle/build_ref.sh into oracle/_ref/).  TEST INFRASTRUCTURE ONLY: it generates the golden
// values that the library's area rule and atlas trace are pinned to.
//
// Modes:
//   area R L kx ky kz S
//       stdout: one line per quadrature ray "face x y z weight" (hexadecimal floating point),
//       or "error <message>" when make_area_rule throws.
//   nodes R L n_int n_ext wavelength T P NT NP S max_hits tail out.bin
//       every incident node (i, j) of the T x P intervals, traced by atlas::trace_cpu; out.bin
//       holds per node 16 binary64 header values (theta, phi, k[3], e0[3], projected_area,
//       escaped, unresolved, histogram_relative_error, rays, outputs, max_balance_error,
//       max_interface_balance_error) followed by the NT*NP cell masses.
//   edges NT
//       stdout: the NT+1 saved u edges (rainbow::make_phase_u_edges) in hexadecimal floating point.
#include <ice_crystal/atlas.hpp>
#include <rainbow/phase_cdf_math.hpp>

#include <cstdio>
#include <cstdlib>
#include <exception>
#include <fstream>
#include <string>
#include <vector>

using namespace iceCrystal;

namespace
{
double num(const char* s) { return std::strtod(s, nullptr); }
std::uint32_t u32(const char* s) { return static_cast<std::uint32_t>(std::strtoul(s, nullptr, 10)); }

int area(char** a)
{
    const HexPrism h{num(a[0]), num(a[1])};
    Vec3 k{num(a[2]), num(a[3]), num(a[4])};
    normalize(k, k);
    try {
        for (const auto& r : atlas::make_area_rule(h, k, u32(a[5])))
            std::printf("%u %a %a %a %a\n", r.entry.face, r.entry.position.x, r.entry.position.y, r.entry.position.z,
                        r.projected_weight_mm2);
    } catch (const std::exception& e) {
        std::printf("error %s\n", e.what());
    }
    return 0;
}

int nodes(char** a)
{
    atlas::Settings s;
    s.prism = {num(a[0]), num(a[1])};
    s.interior_index = num(a[2]);
    s.exterior_index = num(a[3]);
    s.wavelength_nm = num(a[4]);
    s.incident_theta_intervals = u32(a[5]);
    s.incident_phi_intervals = u32(a[6]);
    s.theta_count = u32(a[7]);
    s.phi_count = u32(a[8]);
    s.area_subdivisions = u32(a[9]);
    s.max_internal_hits = u32(a[10]);
    s.tail_tolerance = num(a[11]);
    std::ofstream out(a[12], std::ios::binary);
    for (std::uint32_t i = 0; i <= s.incident_theta_intervals; ++i)
        for (std::uint32_t j = 0; j <= s.incident_phi_intervals; ++j) {
            const auto n = atlas::make_node(s, i, j);
            const auto r = atlas::trace_cpu(s, n);
            const auto& k = n.trace.incident_direction;
            const auto& e = n.grid.frame.e0;
            const double head[16] = {n.theta, n.phi, k.x, k.y, k.z, e.x, e.y, e.z, r.projected_area_mm2, r.escaped_mm2,
                                     r.unresolved_mm2, r.histogram_relative_error, double(r.audit.rays),
                                     double(r.audit.outputs), r.audit.maximum_balance_error,
                                     r.audit.maximum_interface_balance_error};
            out.write(reinterpret_cast<const char*>(head), sizeof head);
            out.write(reinterpret_cast<const char*>(r.mass_mm2.data()),
                      std::streamsize(r.mass_mm2.size() * sizeof(double)));
        }
    return out ? 0 : 1;
}
} // namespace

int main(int argc, char** argv)
{
    try {
        const std::string mode = argc > 1 ? argv[1] : "";
        if (mode == "area" && argc == 8) return area(argv + 2);
        if (mode == "nodes" && argc == 15) return nodes(argv + 2);
        if (mode == "edges" && argc == 3) {
            for (double e : rainbow::make_phase_u_edges(u32(argv[2]))) std::printf("%a\n", e);
            return 0;
        }
        std::fprintf(stderr, "usage: ref_atlas_harness area R L kx ky kz S | nodes R L n_int n_ext nm T P NT NP S hits tail out\n");
        return 2;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
}
