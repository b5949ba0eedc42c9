// ice_precompute_atlas -- drop-in for the reference's atlas precompute
// (hex_atlas/apps/precompute_atlas.cpp) on the B200 C ABI (include/icp_b200.h).
//
// Same options, duplicate-option rejection, material rule (ice: the Warren & Brandt 2008
// index at --wavelength-nm, --ior refused; constant: --ior required), progress lines and exit
// codes (0 after <out>.part was renamed to <out>; 2 with "ice_precompute_atlas: <msg>" for
// any error, the .part directory kept).  Output: <out>/{metadata.json, mass_mm2.npy
// [incident_theta][incident_phi][theta][phi] <f8, u_edges.npy}.
// --batch-rays and --max-work-mib are accepted and validated; they size the reference's
// per-ray histogram columns, which the device path does not use (its histogram is exact
// fixed point), so they set no limit here.  --modules is accepted and ignored.
#include <charconv>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <locale>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "icp_b200.h"
#include "icp_cli_options.hpp"
#include "icp_host_math.hpp"
#include "icp_record_io.hpp"

namespace {

namespace io = icp::io;

struct Options {
    std::string out;
    icp_atlas_settings s{0, 0, 0, 1.0, 0, 0, 0, 0, 0, 2048, 1e-12, 1e-10, 1e-10};
    double wavelength = 0;
    uint32_t batch_rays = 64, max_work_mib = 512;
    bool ice = true;
    int device = 0;
    icp_ice_state optical{};
};

template <class T> T number(std::string_view v)
{
    T x{};
    const auto r = std::from_chars(v.data(), v.data() + v.size(), x);
    if (r.ec != std::errc{} || r.ptr != v.data() + v.size()) throw std::invalid_argument("Invalid number: " + std::string(v));
    if constexpr (std::is_floating_point_v<T>)
        if (!std::isfinite(x)) throw std::invalid_argument("Invalid finite number.");
    return x;
}

std::string last_error()
{
    char buf[1024];
    icp_last_error(buf, sizeof buf);
    return buf;
}

void check(int status)
{
    if (status != ICP_OK) throw std::runtime_error(last_error());
}

Options parse(int argc, char** argv)
{
    Options o;
    auto& s = o.s;
    using V = icp::cli::Values;
    auto real = [](double& x) { return icp::cli::Flag{1, [&x](const V& v) { x = number<double>(v[0]); }}; };
    auto u32 = [](uint32_t& x) { return icp::cli::Flag{1, [&x](const V& v) { x = number<uint32_t>(v[0]); }}; };
    const icp::cli::Table table = {
        {"--out", {1, [&](const V& v) { o.out = std::string(v[0]); }}},
        {"--modules", {1, [](const V&) {}}},
        {"--device", {1, [&](const V& v) { o.device = number<int>(v[0]); }}},
        {"--radius-mm", real(s.circumradius_mm)},
        {"--length-mm", real(s.length_mm)},
        {"--material", {1, [&](const V& v) {
             if (v[0] == "ice") o.ice = true;
             else if (v[0] == "constant") o.ice = false;
             else throw std::invalid_argument("Material must be ice or constant.");
         }}},
        {"--ior", real(s.interior_index)},
        {"--exterior-ior", real(s.exterior_index)},
        {"--wavelength-nm", real(o.wavelength)},
        {"--incident-theta-intervals", u32(s.theta_intervals)},
        {"--incident-phi-intervals", u32(s.phi_intervals)},
        {"--theta", u32(s.nt)},
        {"--phi", u32(s.np)},
        {"--area-subdivisions", u32(s.subdivisions)},
        {"--batch-rays", u32(o.batch_rays)},
        {"--max-work-mib", u32(o.max_work_mib)},
        {"--max-internal-hits", u32(s.max_internal_hits)},
        {"--tail-tolerance", real(s.tail_tolerance)},
        {"--max-unresolved-fraction", real(s.max_unresolved_fraction)},
        {"--max-balance-error", real(s.max_balance_error)},
    };
    auto either = [](const std::string&) { return std::string("Duplicate option or missing argument."); };
    const std::set<std::string> seen = icp::cli::apply(argc, argv, table, icp::cli::Style{true, true, either, either});
    if (o.out.empty()) throw std::invalid_argument("--out required.");
    if (!seen.count("--wavelength-nm")) throw std::invalid_argument("--wavelength-nm is required (vacuum nm).");
    if (o.device < 0) throw std::invalid_argument("Negative CUDA device ordinal.");
    if (!o.batch_rays || !o.max_work_mib) throw std::invalid_argument("Invalid atlas settings.");
    if (o.ice) {
        if (seen.count("--ior"))
            throw std::invalid_argument("Ice index is evaluated from wavelength; --ior requires explicit --material constant.");
        check(icp_ice_index(o.wavelength, &o.optical));
        o.s.interior_index = o.optical.n;
    } else {
        if (!seen.count("--ior")) throw std::invalid_argument("Constant material requires --ior.");
        if (!(o.wavelength > 0)) throw std::invalid_argument("Invalid atlas settings.");
        o.optical = icp_ice_state{o.wavelength, o.s.interior_index, 0, 0, 0, 0};
    }
    return o;
}

void vec(std::ostream& m, const double* v) { m << '[' << v[0] << ',' << v[1] << ',' << v[2] << ']'; }

void material(std::ostream& m, const Options& o)
{
    const auto& s = o.optical;
    m << "{\"model\":\"" << (o.ice ? "ice_ih_warren_brandt_2008_real_only" : "constant")
      << "\",\"wavelength_convention\":\"vacuum_nm\",\"wavelength_nm\":" << s.wavelength_nm
      << ",\"wavelength_requested_nm\":" << s.wavelength_nm << ",\"wavelength_evaluated_nm\":" << s.wavelength_nm
      << ",\"interior_index\":" << s.n << ",\"exterior_index\":" << o.s.exterior_index
      << ",\"interior_index_evaluated_fp64\":" << s.n << ",\"interior_index_solver_fp64\":" << s.n
      << ",\"automatic_ice_dispersion\":" << (o.ice ? "true" : "false")
      << ",\"absorption\":false,\"birefringence\":false,\"absorption_model\":\"ignored_k_equals_zero\",\"kappa_solver\":0";
    if (o.ice)
        m << ",\"source_doi\":\"10.1029/2007JD009744\",\"reference_state\":\"ice_Ih_near_melting_compilation\""
          << ",\"supported_nm\":[200,1100],\"n_interpolation\":\"linear_n_in_log_vacuum_wavelength\""
          << ",\"kappa_interpolation\":\"linear_log_kappa_in_log_vacuum_wavelength\""
          << ",\"temperature_dependence_computed\":false,\"kappa_evaluated_not_used\":" << s.kappa << ",\"bracket_nm\":["
          << s.lower_nm << ',' << s.upper_nm << "],\"log_wavelength_fraction\":" << s.log_wavelength_fraction;
    m << '}';
}

int run(int argc, char** argv)
{
    if (argc == 2 && std::string_view(argv[1]) == "--help") {
        std::cout << "ice_precompute_atlas --out DIR --radius-mm R --length-mm L --wavelength-nm NM\n"
                     " --material ice (default, WB2008 n(lambda), 200..1100nm) | --material constant --ior N\n"
                     " --incident-theta-intervals T --incident-phi-intervals P --theta NT --phi NP --area-subdivisions S\n"
                     " [--max-internal-hits 2048 --tail-tolerance 1e-12 --batch-rays 64 --max-work-mib 512]\n"
                     " [--max-unresolved-fraction 1e-10 --max-balance-error 1e-10 --exterior-ior 1 --device 0]\n"
                     "B200: every quadrature ray traced on the device, exact fixed-point histograms. No random "
                     "seeds, smoothing, or CPU fallback.\n";
        return 0;
    }
    const Options o = parse(argc, argv);
    const auto& s = o.s;
    std::cout << std::setprecision(17) << "material=" << (o.ice ? "ice_wb2008_real_only" : "constant")
              << " wavelength_nm=" << o.wavelength << " n=" << s.interior_index
              << " kappa_evaluated_not_used=" << o.optical.kappa << '\n';
    if (!s.theta_intervals || !s.phi_intervals || !s.nt || !s.np)
        throw std::invalid_argument("Invalid atlas settings.");
    const uint64_t ni = uint64_t(s.theta_intervals) + 1, nj = uint64_t(s.phi_intervals) + 1,
                   cells = uint64_t(s.nt) * s.np;
    if (ni * nj * cells > (uint64_t(1) << 34)) throw std::length_error("Atlas exceeds 128 GiB of cell masses.");
    io::StagingDirectory dir(o.out);
    try {
        icp_context* ctx = nullptr;
        check(icp_context_create(o.device, &ctx));
        struct Guard {
            icp_context* c;
            ~Guard() { icp_context_destroy(c); }
        } guard{ctx};
        double* d_mass = nullptr;
        check(icp_device_alloc(ctx, cells * sizeof(double), reinterpret_cast<void**>(&d_mass)));
        struct Free {
            icp_context* c;
            void* p;
            ~Free() { icp_device_free(c, p); }
        } free_mass{ctx, d_mass};
        std::vector<double> mass(ni * nj * cells);
        std::ostringstream nodes;
        nodes.imbue(std::locale::classic());
        nodes << std::setprecision(17);
        uint64_t total = 0;
        for (uint32_t i = 0; i < ni; ++i)
            for (uint32_t j = 0; j < nj; ++j) {
                icp_atlas_node_report r{};
                check(icp_atlas_trace_node(ctx, &s, i, j, d_mass, &r));
                check(icp_memcpy_d2h(ctx, mass.data() + (uint64_t(i) * nj + j) * cells, d_mass, cells * sizeof(double)));
                icp_atlas_incident n{};
                check(icp_atlas_incident_node(s.theta_intervals, s.phi_intervals, i, j, &n));
                if (i || j) nodes << ",\n";
                nodes << "{\"i\":" << i << ",\"j\":" << j << ",\"theta\":" << n.theta << ",\"phi\":" << n.phi << ",\"ki\":";
                vec(nodes, n.ki);
                nodes << ",\"e0\":";
                vec(nodes, n.e0);
                nodes << ",\"projected_area_mm2\":" << r.projected_area_mm2 << ",\"escaped_mm2\":" << r.escaped_mm2
                      << ",\"unresolved_mm2\":" << r.unresolved_mm2
                      << ",\"histogram_relative_error\":" << r.histogram_relative_error << ",\"rays\":" << r.rays
                      << ",\"outputs\":" << r.outputs << ",\"max_balance_error\":" << r.max_balance_error
                      << ",\"max_interface_balance_error\":" << r.max_interface_balance_error << "}";
                total += r.rays;
                std::cout << "atlas_node=" << i << ',' << j << " rays=" << r.rays
                          << " residual=" << r.unresolved_mm2 / r.projected_area_mm2 << '\n';
            }
        io::write_npy_f64(dir.staging() / "mass_mm2.npy", {ni, nj, s.nt, s.np}, mass.data(), mass.size());
        std::vector<double> edges(s.nt + 1);
        check(icp_u_edges(s.nt, edges.data()));
        io::write_npy_f64(dir.staging() / "u_edges.npy", {uint64_t(s.nt) + 1}, edges.data(), edges.size());
        std::ofstream m(dir.staging() / "metadata.json", std::ios::binary | std::ios::trunc);
        m.exceptions(std::ios::badbit | std::ios::failbit);
        m.imbue(std::locale::classic());
        m << std::setprecision(17);
        m << "{\n\"schema\":\"ice.single_particle_atlas.v1\",\"complete\":true,"
          << "\"backend\":\"cuda_fixed_point_exact_histogram\",\"generator_version\":\"icp_b200.deterministic_atlas.v1\",\n"
          << "\"dtype\":\"<f8\",\"order\":\"C\",\"mass_axes\":[\"incident_theta\",\"incident_phi\",\"theta\",\"phi\"],\n"
          << "\"incident_theta_intervals\":" << s.theta_intervals << ",\"incident_phi_intervals\":" << s.phi_intervals
          << ",\n\"theta_count\":" << s.nt << ",\"phi_count\":" << s.np << ",\n"
          << "\"geometry\":{\"shape\":\"regular_hexagonal_prism\",\"circumradius_mm\":" << s.circumradius_mm
          << ",\"full_length_mm\":" << s.length_mm << ",\"body_long_axis\":[0,1,0]},\n\"material\":";
        material(m, o);
        m << ",\n\"symmetry\":\"D6h_O3_full_24_scalar_unpolarized\",\n"
          << "\"incident_reconstruction\":\"bilinear_theta_phi_in_spherical_incident_frame\",\n"
          << "\"incident_formula\":\"k=(sin(t)cos(p),cos(t),sin(t)sin(p));e0=(cos(t)cos(p),-sin(t),cos(t)sin(p));"
             "e1=k_cross_e0\",\n"
          << "\"area_quadrature\":{\"rule\":\"composite_equal_area_GL2xGL3\",\"subdivisions\":" << s.subdivisions
          << ",\"randomness\":false},\n"
          << "\"transport\":{\"path_rule\":\"R_and_T_R_power_m_T\",\"polarization\":\"two_input_JonesFlux\","
             "\"interference\":false,\"diffraction\":false,\n\"tail_tolerance\":"
          << s.tail_tolerance << ",\"max_internal_hits\":" << s.max_internal_hits
          << ",\"max_unresolved_fraction\":" << s.max_unresolved_fraction << ",\"max_balance_error\":"
          << s.max_balance_error << "},\n"
          << "\"pole_policy\":\"axis_mass_uniform_in_azimuth_in_histogram_end_cap\",\n"
          << "\"accumulation\":\"exact_64bit_fixed_point_2^-62_of_node_quadrature_weight\",\n\"nodes\":[\n"
          << nodes.str() << "],\n\"total_rays\":" << total << ",\"numerical_convergence_certified\":false\n}\n";
        m.close();
        dir.commit();
        std::cout << "atlas_complete nodes=" << ni * nj << " rays=" << total << '\n';
        return 0;
    } catch (...) {
        std::cerr << "Atlas generation failed. Incomplete .part retained; no ray omission or fallback.\n";
        throw;
    }
}

} // namespace

int main(int argc, char** argv)
{
    try {
        return run(argc, argv);
    } catch (const std::exception& e) {
        std::cerr << "ice_precompute_atlas: " << e.what() << '\n';
        return 2;
    }
}
