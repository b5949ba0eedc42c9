// ref_hex_harness.cpp -- drives the REFERENCE hex path (compiled from the reference's own
// sources by oracle/build_ref.sh into oracle/_ref/) for parity pinning and CPU timing.
//
// TEST INFRASTRUCTURE ONLY: never linked into the product.
//
// Modes (all numbers little-endian binary64 / uint64 in the output file):
//   masses  : full orientation plan -> PhaseMassAccumulator::masses() + audits,
//             following hex_phase/apps/generate_hex_phase.cpp:79-140 (CPU branch).
//   trace   : per-ray RayAudit + outgoing (direction, power) for rays [first, first+count)
//             of one node, via trace_batch_cpu (hex_trace/src/hex_trace.cpp:47-71).
//   time    : trace + accumulate rays [first, first+count) of one node, print rays/s.
#include <ice_crystal/phase_generate.hpp>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

using namespace iceCrystal;

namespace
{
double num(const char* s) { return std::strtod(s, nullptr); }
std::uint64_t u64(const char* s) { return std::strtoull(s, nullptr, 10); }

void put(std::ofstream& f, const void* p, std::size_t n) { f.write(static_cast<const char*>(p), std::streamsize(n)); }

PhaseGenerationSettings settings(char** a)
{
    // a: R L kix kiy kiz ior ext nt np max_hits tail
    PhaseGenerationSettings s;
    s.prism = {num(a[0]), num(a[1])};
    s.interior_index = num(a[5]);
    s.exterior_index = num(a[6]);
    const auto nt = static_cast<std::uint32_t>(u64(a[7])), np = static_cast<std::uint32_t>(u64(a[8]));
    s.grid = make_phase_grid(nt, np, {num(a[2]), num(a[3]), num(a[4])});
    s.out_nt = nt;
    s.out_np = np;
    s.wavelength_nm = 550;
    s.max_internal_hits = static_cast<std::uint32_t>(u64(a[9]));
    s.tail_tolerance = num(a[10]);
    return s;
}
} // namespace

int main(int argc, char** argv)
{
    try
    {
        if (argc < 2) { std::cerr << "usage: ref_hex_harness masses|trace|time ...\n"; return 1; }
        const std::string mode = argv[1];
        if (mode == "masses" && argc == 16)
        {
            // masses R L kix kiy kiz ior ext nt np max_hits tail plan.csv batch out.bin
            auto s = settings(argv + 2);
            const auto plan = read_orientation_plan(argv[13]);
            const std::uint64_t batch = u64(argv[14]);
            PhaseMassAccumulator h(s.grid);
            CompositionAudit audit;
            for (const auto& n : plan.nodes) audit.expected_area.add(n.weight * node_area(s, n));
            for (const auto& n : plan.nodes)
            {
                const auto c = node_trace_settings(s, n);
                const double scale = n.weight * node_area(s, n) / double(n.samples);
                for (std::uint64_t first = 0; first < n.samples;)
                {
                    const auto count = std::min<std::uint64_t>(batch, n.samples - first);
                    const auto b = trace_batch_cpu(c, first, count);
                    const auto t = summarize_phase_rays(b.audits, s.max_balance_error);
                    merge_summary(audit.trace, t);
                    audit.escaped_area.add(scale * t.escaped_power_sum);
                    audit.unresolved_area.add(scale * t.unresolved_power_sum);
                    h.add(b.outgoing, n.rotation, scale);
                    first += count;
                }
            }
            const auto mass = h.masses();
            const auto st = h.statistics();
            std::ofstream f(argv[15], std::ios::binary);
            put(f, mass.data(), mass.size() * 8);
            const double d[] = {st.point_mass, st.point_axial, st.forward_mass, st.backward_mass,
                                audit.expected_area.value, audit.escaped_area.value, audit.unresolved_area.value,
                                audit.trace.maximum_balance_error, audit.trace.maximum_interface_balance_error};
            put(f, d, sizeof d);
            const std::uint64_t u[] = {st.samples, st.boundary_snapped_samples, audit.trace.outputs, audit.trace.rays,
                                       audit.trace.status_counts[0], audit.trace.status_counts[1],
                                       audit.trace.status_counts[2], audit.trace.status_counts[3],
                                       audit.trace.status_counts[4], audit.trace.status_counts[5],
                                       audit.trace.status_counts[6], audit.trace.status_counts[7],
                                       audit.trace.accepted ? 1u : 0u};
            put(f, u, sizeof u);
            return f ? 0 : 3;
        }
        if (mode == "trace" && argc == 16)
        {
            // trace R L kix kiy kiz ior ext seed total max_hits tail first count out.bin
            HexPrism p{num(argv[2]), num(argv[3])};
            const auto c = make_trace_settings(p, {num(argv[4]), num(argv[5]), num(argv[6])}, num(argv[8]),
                                               num(argv[7]), u64(argv[10]), u64(argv[9]),
                                               static_cast<std::uint32_t>(u64(argv[11])), num(argv[12]));
            const auto b = trace_batch_cpu(c, u64(argv[13]), static_cast<std::size_t>(u64(argv[14])), ~std::size_t{0} / 512);
            std::ofstream f(argv[15], std::ios::binary);
            for (std::size_t i = 0; i < b.audits.size(); ++i)
            {
                const auto& a = b.audits[i];
                const double r[] = {double(static_cast<unsigned>(a.status)), double(a.output_count), a.escaped_power,
                                    a.unresolved_power, double(a.internal_hits), a.max_interface_balance_error};
                put(f, r, sizeof r);
            }
            for (const auto& o : b.outgoing)
            {
                const double r[] = {o.direction.x, o.direction.y, o.direction.z, o.power_fraction};
                put(f, r, sizeof r);
            }
            return f ? 0 : 3;
        }
        if (mode == "time" && argc == 16)
        {
            // time R L kix kiy kiz ior ext nt np max_hits tail seed first count   (identity orientation)
            auto s = settings(argv + 2);
            OrientationNode n;
            n.weight = 1;
            n.seed = u64(argv[13]);
            n.samples = u64(argv[14]) + u64(argv[15]);
            const auto c = node_trace_settings(s, n);
            const double scale = node_area(s, n) / double(n.samples);
            PhaseMassAccumulator h(s.grid);
            const auto t0 = std::chrono::steady_clock::now();
            std::uint64_t outputs = 0;
            for (std::uint64_t first = u64(argv[14]); first < n.samples;)
            {
                const auto count = std::min<std::uint64_t>(4096, n.samples - first);
                const auto b = trace_batch_cpu(c, first, count);
                outputs += b.outgoing.size();
                h.add(b.outgoing, n.rotation, scale);
                first += count;
            }
            const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            std::printf("{\"rays\": %llu, \"outputs\": %llu, \"seconds\": %.6f}\n",
                        static_cast<unsigned long long>(u64(argv[15])), static_cast<unsigned long long>(outputs), dt);
            return 0;
        }
        std::cerr << "bad arguments\n";
        return 1;
    }
    catch (const std::exception& e)
    {
        std::cerr << "ref_hex_harness: " << e.what() << '\n';
        return 2;
    }
}
