// ref_drop_harness.cpp -- driver over the REFERENCE drop sources (header-only tracer and
// shape, src/projected_area.cpp, src/water_refractive_index.cpp), compiled by
// oracle/build_ref.sh into oracle/_ref/ref_drop_harness.  Test infrastructure only: it
// produces the reference's own values for the drop host inputs and for the four-family
// path tracer, which pin the oracle restatement and the product's host helpers.
//
//   water     stdin "lambda_nm T_C p_Pa" lines -> "index density"  (evaluate_water_optics)
//   water_state  the same -> "index density pressure_residual bracket_width"
//   shape     stdin "radius_mm sphere" lines -> "c0..c7 inner outer" (RaindropShape::try_make)
//   area      stdin "c0..c7 radius_mm kx ky kz" lines -> "area_mm2"  (compute_projected_area)
//   frame     stdin "alpha_deg" lines -> float ki(3) and incident_basis_x(3) of the config the
//             rainbow_generate CLI builds (apps/generate_phase.cpp:209-217)
//   families  radius sphere n_int kx ky kz grid out.bin: RaindropPathTracer unpolarized trace
//             over the vertex lattice; per vertex 41 float64:
//               origin(3) direction(3) e0(3), then per family R,TT,TRT,TRRT:
//               status, exit direction(3), exit position(3), unpolarized flux power
//             The tracer's Jones columns are amplitude responses; the flux power multiplies
//             0.5 (|col0|^2 + |col1|^2) by n_t cos_t / (n_i cos_i) of both transmissions,
//             taken from the logged boundary queries.
//   vertices  radius sphere n_int kx ky kz grid out.bin [wavelength_nm [c0 .. c7]]: the same
//             lattice trace as raw records (u32 width, height; f32 half_extent, incident[3],
//             basis_x[3]; OutgoingVertex[4 n]; Field32[4 n], the second response column); an
//             optional wavelength (default 700 nm) and explicit shape coefficients (with the
//             bounding radii, half extent and reference distances derived from them as
//             RaindropShape::try_make and make_config do)
//   config    radius sphere n_int kx ky kz grid wavelength_nm [c0 .. c7]: the RaindropTraceConfig
//             of those settings, its 116 bytes as hex
//   time      radius sphere n_int kx ky kz grid row0 rows [c0 .. c7]: traces lattice rows
//             [row0, row0+rows) with RaindropPathTracer::trace_vertex_unpolarized and prints
//             "vertices hits seconds" (the reference's CPU drop tracer; optional coefficients
//             replace the Table-I shape, with the bounding radii of RaindropShape::try_make).
#include <rainbow/phase_cdf_math.hpp>
#include <rainbow/projected_area.hpp>
#include <rainbow/raindrop_paths.hpp>
#include <rainbow/raindrop_settings.hpp>
#include <rainbow/water_refractive_index.hpp>

#include <array>
#include <chrono>
#include <limits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

using namespace rainbow;

namespace {

struct Logged {
    BoundaryRay ray;
    BoundaryHit hit;
};

// Forwards to the reference intersector and keeps every query of the current vertex.
struct RecordingIntersector {
    RaindropIntersector inner;
    std::vector<Logged> log;
    BoundaryHit intersect(const BoundaryRay& r)
    {
        const BoundaryHit h = inner.intersect(r);
        log.push_back({r, h});
        return h;
    }
};

double dotd(const Vec3 a, const Vec3 b) { return double(a.x) * b.x + double(a.y) * b.y + double(a.z) * b.z; }
double norm2(const Complex32 c) { return double(c.real) * c.real + double(c.imag) * c.imag; }
double field_power(const Field32& f) { return norm2(f.x) + norm2(f.y); }

int families(int argc, char** argv)
{
    if (argc != 10) {
        std::fprintf(stderr, "families radius sphere n_int kx ky kz grid out.bin\n");
        return 1;
    }
    RaindropSettings s;
    s.radius_mm = std::strtof(argv[2], nullptr);
    s.force_sphere = std::atoi(argv[3]) != 0;
    s.interior_index = std::strtof(argv[4], nullptr);
    s.incident_direction = {std::strtof(argv[5], nullptr), std::strtof(argv[6], nullptr), std::strtof(argv[7], nullptr)};
    s.grid_width = s.grid_height = (std::uint32_t)std::atoi(argv[8]);
    const RaindropTraceConfig cfg = s.make_config();
    const std::uint32_t count = cfg.vertex_count();
    std::vector<OutgoingVertex> v(4 * (size_t)count);
    std::vector<Field32> second(4 * (size_t)count);
    RecordingIntersector rec{RaindropIntersector{cfg.shape}, {}};
    std::vector<double> out;
    out.reserve(41 * (size_t)count);
    const double ni = cfg.exterior_index, nw = cfg.interior_index;
    for (std::uint32_t idx = 0; idx < count; ++idx) {
        rec.log.clear();
        RaindropPathTracer::trace_vertex_unpolarized(cfg, idx, rec, v.data(), second.data());
        const Vec3 o = rec.log.empty() ? Vec3{} : rec.log[0].ray.physical_origin;
        out.insert(out.end(), {double(o.x), double(o.y), double(o.z), double(cfg.incident_direction.x),
                               double(cfg.incident_direction.y), double(cfg.incident_direction.z),
                               double(cfg.incident_basis_x.x), double(cfg.incident_basis_x.y),
                               double(cfg.incident_basis_x.z)});
        for (unsigned f = 0; f < 4; ++f) {
            const OutgoingVertex& x = v[f * (size_t)count + idx];
            double power = 0;
            if (x.status == VertexStatus::Valid) {
                power = 0.5 * (field_power(x.field) + field_power(second[f * (size_t)count + idx]));
                if (f > 0 && rec.log.size() > f) {
                    const Vec3 n0 = rec.log[0].hit.outward_normal;
                    const double ci0 = -dotd(cfg.incident_direction, n0);
                    const double ct0 = -dotd(rec.log[1].ray.direction, n0);
                    const Vec3 nf = rec.log[f].hit.outward_normal;
                    const double cif = dotd(rec.log[f].ray.direction, nf);
                    const double ctf = dotd(x.direction_drop, nf);
                    power *= (nw * ct0) / (ni * ci0) * (ni * ctf) / (nw * cif);
                }
            }
            out.insert(out.end(), {double(x.status), double(x.direction_drop.x), double(x.direction_drop.y),
                                   double(x.direction_drop.z), double(x.position_drop.x), double(x.position_drop.y),
                                   double(x.position_drop.z), power});
        }
    }
    FILE* fp = std::fopen(argv[9], "wb");
    if (!fp) return 1;
    const size_t n = std::fwrite(out.data(), sizeof(double), out.size(), fp);
    std::fclose(fp);
    return n == out.size() ? 0 : 1;
}

// The reference's unpolarized lattice trace as raw records: u32 width, height; f32 half_extent,
// incident[3], basis_x[3]; OutgoingVertex[4 * count]; Field32[4 * count] (second column).
// Settings from argv[2..8], an optional wavelength at argv[first] and optional coefficients
// at argv[first + 1 .. first + 8].
RaindropTraceConfig lattice_config(int argc, char** argv, int first)
{
    RaindropSettings s;
    s.radius_mm = std::strtof(argv[2], nullptr);
    s.force_sphere = std::atoi(argv[3]) != 0;
    s.interior_index = std::strtof(argv[4], nullptr);
    s.incident_direction = {std::strtof(argv[5], nullptr), std::strtof(argv[6], nullptr), std::strtof(argv[7], nullptr)};
    s.grid_width = s.grid_height = (std::uint32_t)std::atoi(argv[8]);
    if (argc > first) s.wavelength_nm = std::strtof(argv[first], nullptr);
    RaindropTraceConfig cfg = s.make_config();
    if (argc == first + 9) {
        const float inf = std::numeric_limits<float>::infinity();
        float sum = 0.0f;
        for (int k = 0; k < 8; ++k) cfg.shape.coefficients[k] = std::strtof(argv[first + 1 + k], nullptr);
        for (int k = 1; k < 8; ++k) sum = ::nextafterf(sum + ::fabsf(cfg.shape.coefficients[k]), inf);
        const float center = 1.0f + cfg.shape.coefficients[0];
        cfg.shape.inner_radius = ::nextafterf(center - sum - 0x1p-20f, -inf);
        cfg.shape.outer_radius = ::nextafterf(center + sum + 0x1p-20f, inf);
        cfg.grid_half_extent = cfg.shape.outer_radius * 1.01f;
        cfg.reference_distance = cfg.outgoing_reference_distance = 2.0f * cfg.shape.outer_radius;
    }
    return cfg;
}

int config(int argc, char** argv)
{
    if (argc != 10 && argc != 18) {
        std::fprintf(stderr, "config radius sphere n_int kx ky kz grid wavelength_nm [c0 .. c7]\n");
        return 1;
    }
    const RaindropTraceConfig cfg = lattice_config(argc, argv, 9);
    const unsigned char* b = reinterpret_cast<const unsigned char*>(&cfg);
    for (size_t i = 0; i < sizeof cfg; ++i) std::printf("%02x", b[i]);
    std::printf("\n");
    return 0;
}

int vertices(int argc, char** argv)
{
    if (argc != 10 && argc != 11 && argc != 19) {
        std::fprintf(stderr, "vertices radius sphere n_int kx ky kz grid out.bin [wavelength_nm [c0 .. c7]]\n");
        return 1;
    }
    const RaindropTraceConfig cfg = lattice_config(argc, argv, 10);
    const std::uint32_t count = cfg.vertex_count();
    std::vector<OutgoingVertex> v(4 * (size_t)count);
    std::vector<Field32> second(4 * (size_t)count);
    RaindropIntersector intersector{cfg.shape};
    for (std::uint32_t idx = 0; idx < count; ++idx)
        RaindropPathTracer::trace_vertex_unpolarized(cfg, idx, intersector, v.data(), second.data());
    FILE* fp = std::fopen(argv[9], "wb");
    if (!fp) return 1;
    const std::uint32_t wh[2] = {cfg.grid_width, cfg.grid_height};
    const float frame[7] = {cfg.grid_half_extent, cfg.incident_direction.x, cfg.incident_direction.y,
                            cfg.incident_direction.z, cfg.incident_basis_x.x, cfg.incident_basis_x.y,
                            cfg.incident_basis_x.z};
    bool ok = std::fwrite(wh, 4, 2, fp) == 2 && std::fwrite(frame, 4, 7, fp) == 7;
    ok = ok && std::fwrite(v.data(), sizeof(OutgoingVertex), v.size(), fp) == v.size();
    ok = ok && std::fwrite(second.data(), sizeof(Field32), second.size(), fp) == second.size();
    return std::fclose(fp) == 0 && ok ? 0 : 1;
}

int time_rows(int argc, char** argv)
{
    if (argc != 11 && argc != 19) {
        std::fprintf(stderr, "time radius sphere n_int kx ky kz grid row0 rows [c0 .. c7]\n");
        return 1;
    }
    RaindropSettings s;
    s.radius_mm = std::strtof(argv[2], nullptr);
    s.force_sphere = std::atoi(argv[3]) != 0;
    s.interior_index = std::strtof(argv[4], nullptr);
    s.incident_direction = {std::strtof(argv[5], nullptr), std::strtof(argv[6], nullptr), std::strtof(argv[7], nullptr)};
    s.grid_width = s.grid_height = (std::uint32_t)std::atoi(argv[8]);
    RaindropTraceConfig cfg = s.make_config();
    if (argc == 19) {
        const float inf = std::numeric_limits<float>::infinity();
        float sum = 0.0f;
        for (int k = 0; k < 8; ++k) cfg.shape.coefficients[k] = std::strtof(argv[11 + k], nullptr);
        for (int k = 1; k < 8; ++k) sum = ::nextafterf(sum + ::fabsf(cfg.shape.coefficients[k]), inf);
        const float center = 1.0f + cfg.shape.coefficients[0];
        cfg.shape.inner_radius = ::nextafterf(center - sum - 0x1p-20f, -inf);
        cfg.shape.outer_radius = ::nextafterf(center + sum + 0x1p-20f, inf);
        cfg.grid_half_extent = cfg.shape.outer_radius * 1.01f;
        cfg.reference_distance = cfg.outgoing_reference_distance = 2.0f * cfg.shape.outer_radius;
    }
    const std::uint32_t row0 = (std::uint32_t)std::atoi(argv[9]), rows = (std::uint32_t)std::atoi(argv[10]);
    const std::uint32_t count = cfg.vertex_count();
    std::vector<OutgoingVertex> v(4 * (size_t)count);
    std::vector<Field32> second(4 * (size_t)count);
    RaindropIntersector isect{cfg.shape};
    const auto t0 = std::chrono::steady_clock::now();
    std::uint64_t n = 0, hits = 0;
    for (std::uint32_t y = row0; y < row0 + rows && y < cfg.grid_height; ++y)
        for (std::uint32_t x = 0; x < cfg.grid_width; ++x) {
            const std::uint32_t idx = y * cfg.grid_width + x;
            RaindropPathTracer::trace_vertex_unpolarized(cfg, idx, isect, v.data(), second.data());
            ++n;
            hits += v[idx].status != VertexStatus::Miss;
        }
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("%llu %llu %.9f\n", (unsigned long long)n, (unsigned long long)hits, sec);
    return 0;
}

} // namespace

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::fprintf(stderr, "usage: ref_drop_harness water|shape|area|frame|families|vertices|config ...\n");
        return 1;
    }
    const std::string mode = argv[1];
    std::cout.precision(17);
    try {
        if (mode == "families") return families(argc, argv);
        if (mode == "vertices") return vertices(argc, argv);
        if (mode == "config") return config(argc, argv);
        if (mode == "time") return time_rows(argc, argv);
        std::string line;
        while (std::getline(std::cin, line)) {
            if (line.empty()) continue;
            std::istringstream in(line);
            if (mode == "water") {
                double l, t, p;
                in >> l >> t >> p;
                try {
                    const auto w = evaluate_water_optics(l, t, p);
                    std::cout << w.refractive_index << ' ' << w.density_kg_m3 << '\n';
                } catch (const std::exception&) {
                    std::cout << "nan nan\n";
                }
            } else if (mode == "water_state") {
                double l, t, p;
                in >> l >> t >> p;
                try {
                    const auto w = evaluate_water_optics(l, t, p);
                    std::cout << w.refractive_index << ' ' << w.density_kg_m3 << ' ' << w.density_pressure_residual_pascal
                              << ' ' << w.density_bracket_width_kg_m3 << '\n';
                } catch (const std::exception&) {
                    std::cout << "nan nan nan nan\n";
                }
            } else if (mode == "shape") {
                float r;
                int sphere;
                in >> r >> sphere;
                RaindropShape sh;
                if (!RaindropShape::try_make(r, sphere != 0, sh)) {
                    std::cout << "invalid\n";
                    continue;
                }
                for (float c : sh.coefficients) std::cout << double(c) << ' ';
                std::cout << double(sh.inner_radius) << ' ' << double(sh.outer_radius) << '\n';
            } else if (mode == "area") {
                std::array<double, 8> c{};
                double r;
                std::array<double, 3> k{};
                for (double& x : c) in >> x;
                in >> r >> k[0] >> k[1] >> k[2];
                try {
                    std::cout << compute_projected_area(c, r, k).area_mm2 << '\n';
                } catch (const std::exception&) {
                    std::cout << "nan\n";
                }
            } else if (mode == "frame") {
                double alpha;
                in >> alpha;
                // the CLI's inclination -> settings mapping
                const double angle = alpha * phase_cdf_pi / 180.0;
                RaindropSettings s;
                s.radius_mm = 1.0f;
                s.incident_direction = {static_cast<float>(std::cos(angle)), static_cast<float>(-std::sin(angle)), 0};
                const auto c = s.make_config();
                std::cout << double(c.incident_direction.x) << ' ' << double(c.incident_direction.y) << ' '
                          << double(c.incident_direction.z) << ' ' << double(c.incident_basis_x.x) << ' '
                          << double(c.incident_basis_x.y) << ' ' << double(c.incident_basis_x.z) << '\n';
            } else {
                std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
                return 1;
            }
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_drop_harness: %s\n", e.what());
        return 2;
    }
    return 0;
}
