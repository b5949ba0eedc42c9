// ref_record_harness.cpp -- one drop record's work (trace + bin + stored CDF) done by the
// REFERENCE's own CPU code, compiled by oracle/build_ref.sh into oracle/_ref/ref_record_harness.
// Test infrastructure only (the timed reference arm of bench.py); never linked into the product.
//
// The reference has no CPU path for a whole drop record (its drop records come from the OptiX
// lattice trace); this driver composes its CPU-compilable parts into the record the B200 path
// computes, as the drop oracle does:
//   rays       the counter RNG of the prism path (iceCrystal::sample_uniform,
//              hex_trace/include/ice_crystal/math.hpp:136-146) on a disk covering the silhouette
//              (radius = the shape's conservative outer radius, 2 r_out + 1 before the centre);
//   surface    RaindropIntersector (FP32 solve with its FP64 fallback,
//              include/rainbow/raindrop_intersection.hpp:337-382);
//   interface  DielectricInterface::split on the two-column unpolarised Jones response
//              (include/rainbow/dielectric_interface.hpp), exactly the step of
//              RaindropPathTracer::trace_impl (include/rainbow/raindrop_paths.hpp:41-107), with
//              the chain continued past the tracer's fixed three internal boundaries to
//              max_internal_hits, as the record path does;
//   power      0.5 (|col0|^2 + |col1|^2) times n_t cos_t / (n_i cos_i) of the entry and exit
//              transmissions (the flux form of the tracer's amplitude responses);
//   binning    PhaseMassAccumulator::add (hex_phase/src/phase_table.cpp:41-76) on
//              make_phase_grid(nt, np, ki);
//   CDF        build_host_cdf (hex_phase/src/phase_table.cpp:111-187).
//
//   record  radius n_int kx ky kz nt np max_hits seed total first count c0 .. c7 cdf
//     traces ray ids [first, first + count) of a `total`-ray record, bins every exit, and when
//     cdf != 0 builds the stored CDF of the binned masses; prints
//     "rays hits exits trace_seconds cdf_seconds checksum".
#include <rainbow/dielectric_interface.hpp>
#include <rainbow/raindrop_settings.hpp>

#include <ice_crystal/math.hpp>
#include <ice_crystal/phase_table.hpp>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <string>
#include <vector>

namespace {

unsigned long long u64(const char* s) { return std::strtoull(s, nullptr, 10); }
double norm2(const rainbow::Complex32 c) { return double(c.real) * c.real + double(c.imag) * c.imag; }
double response_power(const rainbow::JonesResponse32& r)
{
    return 0.5 * (norm2(r.column[0].x) + norm2(r.column[0].y) + norm2(r.column[1].x) + norm2(r.column[1].y));
}
double dotd(const rainbow::Vec3 a, const rainbow::Vec3 b) { return double(a.x) * b.x + double(a.y) * b.y + double(a.z) * b.z; }

int record(int argc, char** argv)
{
    if (argc != 23) {
        std::fprintf(stderr, "record radius n_int kx ky kz nt np max_hits seed total first count c0 .. c7 cdf\n");
        return 1;
    }
    rainbow::RaindropSettings s;
    s.radius_mm = std::strtof(argv[2], nullptr);
    s.interior_index = std::strtof(argv[3], nullptr);
    s.incident_direction = {std::strtof(argv[4], nullptr), std::strtof(argv[5], nullptr), std::strtof(argv[6], nullptr)};
    rainbow::RaindropTraceConfig cfg = s.make_config();
    const auto nt = (std::uint32_t)u64(argv[7]), np = (std::uint32_t)u64(argv[8]);
    const auto max_hits = (unsigned)u64(argv[9]);
    const std::uint64_t seed = u64(argv[10]), total = u64(argv[11]), first = u64(argv[12]), count = u64(argv[13]);
    // explicit shape coefficients, with the bounding radii RaindropShape::try_make derives
    const float inf = std::numeric_limits<float>::infinity();
    float sum = 0.0f;
    for (int k = 0; k < 8; ++k) cfg.shape.coefficients[k] = std::strtof(argv[14 + k], nullptr);
    for (int k = 1; k < 8; ++k) sum = ::nextafterf(sum + ::fabsf(cfg.shape.coefficients[k]), inf);
    const float center = 1.0f + cfg.shape.coefficients[0];
    cfg.shape.inner_radius = ::nextafterf(center - sum - 0x1p-20f, -inf);
    cfg.shape.outer_radius = ::nextafterf(center + sum + 0x1p-20f, inf);
    const bool cdf = std::atoi(argv[22]) != 0;

    const rainbow::Vec3 w = cfg.incident_direction;
    const rainbow::TransverseFrame frame{cfg.incident_basis_x, w.cross(cfg.incident_basis_x).normalized()};
    const float disk = cfg.shape.outer_radius, back = 2.0f * cfg.shape.outer_radius + 1.0f;
    const double weight = 3.14159265358979323846 * double(disk) * disk * double(s.radius_mm) * s.radius_mm / double(total);
    const float ni = cfg.exterior_index, nw = cfg.interior_index;
    rainbow::RaindropIntersector isect{cfg.shape};
    iceCrystal::PhaseMassAccumulator hist(iceCrystal::make_phase_grid(nt, np, {double(w.x), double(w.y), double(w.z)}));

    const auto t0 = std::chrono::steady_clock::now();
    std::uint64_t hits = 0, exits = 0;
    auto bin = [&](const rainbow::Vec3 d, double power) {
        // the accumulator takes unit binary64 directions: the binary32 exit direction, promoted
        // and normalised
        const double x = d.x, y = d.y, z = d.z, n = std::sqrt(x * x + y * y + z * z);
        hist.add(iceCrystal::Vec3{x / n, y / n, z / n}, weight * power);
        ++exits;
    };
    for (std::uint64_t id = first; id < first + count; ++id) {
        const double u0 = iceCrystal::sample_uniform(seed, id, 0), u1 = iceCrystal::sample_uniform(seed, id, 1);
        const float r = disk * (float)std::sqrt(u0), a = (float)(2.0 * 3.14159265358979323846 * u1);
        const rainbow::Vec3 p = (frame.e0 * (r * std::cos(a)) + frame.e1 * (r * std::sin(a))) - w * back;
        const rainbow::BoundaryHit entry = isect.intersect({p, w, 0.0f, false});
        if (entry.code != rainbow::BoundaryCode::Hit) continue;
        ++hits;
        rainbow::JonesResponseRay active{w, frame, rainbow::JonesResponse32::identity()};
        const auto b = rainbow::DielectricInterface::split(active, entry.outward_normal, ni, nw);
        if (!b.is_valid) continue;
        bin(b.reflected.direction, response_power(b.reflected.field));
        if (!b.has_transmission) continue;
        const double ci0 = -dotd(w, entry.outward_normal), ct0 = -dotd(b.transmitted.direction, entry.outward_normal);
        const double into = (double(nw) * ct0) / (double(ni) * ci0);
        active = b.transmitted;
        rainbow::Vec3 prev = entry.position;
        for (unsigned k = 0; k < max_hits; ++k) {
            const rainbow::BoundaryHit hit = isect.intersect({prev, active.direction, 0x1p-17f, true});
            if (hit.code != rainbow::BoundaryCode::Hit) break;
            const auto sp = rainbow::DielectricInterface::split(active, -hit.outward_normal, nw, ni);
            if (!sp.is_valid) break;
            if (sp.has_transmission) {
                const double cif = dotd(active.direction, hit.outward_normal);
                const double ctf = dotd(sp.transmitted.direction, hit.outward_normal);
                bin(sp.transmitted.direction, response_power(sp.transmitted.field) * into * (double(ni) * ctf) /
                                                  (double(nw) * cif));
            }
            active = sp.reflected;
            prev = hit.position;
        }
    }
    const auto t1 = std::chrono::steady_clock::now();
    double checksum = 0.0, cdf_seconds = 0.0;
    const std::vector<double> masses = hist.masses();
    if (cdf) {
        const auto c0 = std::chrono::steady_clock::now();
        const iceCrystal::HostCdf out = iceCrystal::build_host_cdf(hist.grid(), masses, nt, np);
        cdf_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - c0).count();
        checksum = out.report.g_stored;
    } else {
        for (double m : masses) checksum += m;
    }
    std::printf("%llu %llu %llu %.9f %.9f %.17g\n", (unsigned long long)count, (unsigned long long)hits,
                (unsigned long long)exits, std::chrono::duration<double>(t1 - t0).count(), cdf_seconds, checksum);
    return 0;
}

} // namespace

int main(int argc, char** argv)
{
    try {
        if (argc >= 2 && std::string(argv[1]) == "record") return record(argc, argv);
        std::fprintf(stderr, "usage: ref_record_harness record ...\n");
        return 1;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_record_harness: %s\n", e.what());
        return 2;
    }
}
