// ice_generate_phase -- drop-in for the reference CLI of the same name
// (hex_phase/apps/generate_hex_phase.cpp:33-173) on the B200 C ABI (include/icp_b200.h).
//
// Same options, defaults, duplicate-option rejection and exit codes: 1 with
// "ice_generate_phase: <msg>" for invalid arguments, 2 with <out>.part/failure.json when
// generation or a quality gate fails, 0 after <out>.part was renamed to <out>.
// Extensions (new flags only): --trace-precision fp32|fp64 (default fp32: the FP32 trace
// with exact fixed-point power bookkeeping; fp64: the reference's binary64 arithmetic and
// per-ray tolerances).  --modules is accepted and ignored (kernels are linked in).
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
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

namespace H = icp::host;
namespace io = icp::io;

struct Options {
    std::string out, orientations;
    double R = 0, L = 0, ki[3] = {0, 0, 0}, ior = 0, external_ior = 1, wavelength = 0;
    uint32_t nt = 0, np = 0, ct = 0, cp = 0;
    uint64_t batch = 4096, max_records = 4ull * 1024 * 1024;
    uint32_t max_hits = 1024;
    double tail = 1e-12, max_unresolved = 1e-10, max_balance = 1e-10, max_hist_err = 1e-10;
    double max_l1 = 1e-10, max_lost = 1e-12, max_tv = 1;
    int device = 0;
    uint32_t precision = ICP_FP32;
    std::set<std::string> seen;
};

template <class T> T number(std::string_view s)
{
    T v{};
    const auto r = std::from_chars(s.data(), s.data() + s.size(), v);
    if (r.ec != std::errc{} || r.ptr != s.data() + s.size()) throw std::invalid_argument("Malformed numeric option.");
    return v;
}

Options parse(int argc, char** argv)
{
    Options o;
    using V = icp::cli::Values;
    auto real = [](double& x) { return icp::cli::Flag{1, [&x](const V& v) { x = number<double>(v[0]); }}; };
    auto u32 = [](uint32_t& x) { return icp::cli::Flag{1, [&x](const V& v) { x = number<uint32_t>(v[0]); }}; };
    auto u64 = [](uint64_t& x) { return icp::cli::Flag{1, [&x](const V& v) { x = number<uint64_t>(v[0]); }}; };
    const icp::cli::Table table = {
        {"--out", {1, [&](const V& v) { o.out = std::string(v[0]); }}},
        {"--orientations", {1, [&](const V& v) { o.orientations = std::string(v[0]); }}},
        {"--modules", {1, [](const V&) {}}},
        {"--radius-mm", real(o.R)},
        {"--length-mm", real(o.L)},
        {"--ki", {3, [&](const V& v) { for (int k = 0; k < 3; ++k) o.ki[k] = number<double>(v[k]); }}},
        {"--ior", real(o.ior)},
        {"--external-ior", real(o.external_ior)},
        {"--wavelength-nm", real(o.wavelength)},
        {"--theta", u32(o.nt)},
        {"--phi", u32(o.np)},
        {"--cdf-theta", u32(o.ct)},
        {"--cdf-phi", u32(o.cp)},
        {"--batch-size", u64(o.batch)},
        {"--max-output-records", u64(o.max_records)},
        {"--max-internal-hits", u32(o.max_hits)},
        {"--tail-tolerance", real(o.tail)},
        {"--max-unresolved-fraction", real(o.max_unresolved)},
        {"--max-balance-error", real(o.max_balance)},
        {"--max-histogram-relative-error", real(o.max_hist_err)},
        {"--cdf-max-l1", real(o.max_l1)},
        {"--cdf-max-lost-mass", real(o.max_lost)},
        {"--max-coarsening-tv", real(o.max_tv)},
        {"--device", {1, [&](const V& v) { o.device = number<int>(v[0]); }}},
        {"--trace-precision", {1, [&](const V& v) {
             if (v[0] == "fp32") o.precision = ICP_FP32;
             else if (v[0] == "fp64") o.precision = ICP_FP64;
             else throw std::invalid_argument("--trace-precision must be fp32 or fp64");
         }}},
    };
    const icp::cli::Style style{true, false, [](const std::string& f) { return "Duplicate option: " + f; },
                                [](const std::string& f) { return "Missing value: " + f; }};
    o.seen = icp::cli::apply(argc, argv, table, style);
    for (const char* k : {"--out", "--orientations", "--radius-mm", "--length-mm", "--ki", "--ior", "--wavelength-nm",
                          "--theta", "--phi"})
        if (!o.seen.count(k)) throw std::invalid_argument(std::string("Required option: ") + k);
    if (o.device < 0) throw std::invalid_argument("Negative CUDA device ordinal.");
    if (!o.nt || !o.np || (uint64_t)o.nt * o.np > 0xffffffffull || o.nt > 32u * 65535u || o.np > 0x7fffffffu)
        throw std::invalid_argument("Unsupported phase grid dimensions.");
    H::V k;
    H::Frame f;
    if (!H::normalize({o.ki[0], o.ki[1], o.ki[2]}, k) || !H::make_frame(k, f))
        throw std::invalid_argument("Invalid incident direction.");
    if (!o.seen.count("--cdf-theta")) o.ct = o.nt;
    if (!o.seen.count("--cdf-phi")) o.cp = o.np;
    const double half = 0.5 * (o.L / o.R);
    if (!(H::finite(o.R) && H::finite(o.L) && o.R > 0 && o.L > 0 && H::finite(half) && half > 0))
        throw std::invalid_argument("Invalid hex trace geometry, direction/frame, indices, sample count or termination policy.");
    if (!(o.ior > 0 && o.external_ior > 0 && H::finite(o.ior) && H::finite(o.external_ior) && H::finite(o.tail) &&
          o.tail >= 0 && o.tail < 1 && o.max_hits > 0))
        throw std::invalid_argument("Invalid hex trace geometry, direction/frame, indices, sample count or termination policy.");
    if (!(o.wavelength > 0) || !H::finite(o.wavelength) || !o.batch || !o.max_records || !o.ct || !o.cp ||
        o.ct > o.nt || o.cp > o.np || o.nt % o.ct || o.np % o.cp)
        throw std::invalid_argument("Invalid wavelength, capacity, or coarsening dimensions.");
    for (double t : {o.max_unresolved, o.max_balance, o.max_hist_err})
        if (!H::finite(t) || t < 0 || t >= 1) throw std::invalid_argument("Invalid quality tolerance.");
    if (!H::finite(o.max_l1) || o.max_l1 < 0 || o.max_l1 > 2 || !H::finite(o.max_lost) || o.max_lost < 0 ||
        o.max_lost > 1 || !H::finite(o.max_tv) || o.max_tv < 0 || o.max_tv > 1)
        throw std::invalid_argument("Invalid CDF quality policy.");
    if (o.batch > 0xffffffffull) throw std::invalid_argument("Batch size exceeds 32-bit range.");
    return o;
}

std::string last_error()
{
    char buf[2048];
    icp_last_error(buf, sizeof buf);
    return buf;
}

const char* kStatus[8] = {"exhausted", "tail_tolerance_reached", "interaction_limit", "ambiguous_boundary",
                          "invalid_input", "numerical_failure", "output_overflow", "replay_mismatch"};

std::ofstream json_out(const std::filesystem::path& p)
{
    std::ofstream f(p, std::ios::binary | std::ios::trunc);
    if (!f) throw std::runtime_error("Cannot open metadata output.");
    f.exceptions(std::ios::badbit | std::ios::failbit);
    f.imbue(std::locale::classic());
    f << std::setprecision(17);
    return f;
}

void write_failure(const std::filesystem::path& path, const std::string& reason, const icp_record_report& r)
{
    auto f = json_out(path);
    f << "{\n  \"complete\": false,\n  \"error\": " << io::json_quote(reason) << ",\n  \"processed_rays\": " << r.trace.rays
      << ",\n  \"status_counts\": {";
    for (int i = 0; i < 8; ++i) f << (i ? "," : "") << io::json_quote(kStatus[i]) << ':' << r.trace.status_counts[i];
    f << "}\n}\n";
}

// metadata.json in the reference schema (hex_phase/src/phase_generate.cpp:280-358).
void write_metadata(const std::filesystem::path& path, const Options& o, const io::Plan& plan, const icp_grid& g,
                    const icp_record_report& r, double per_ray_tolerance)
{
    auto f = json_out(path);
    const double area = r.expected_area_mm2;
    auto vec = [&](const double* v) { f << '[' << v[0] << ',' << v[1] << ',' << v[2] << ']'; };
    f << "{\n  \"schema\": \"rainbow.phase_cdf.numpy.v2\",\n  \"complete\": true,\n"
      << "  \"generator_version\": \"icp_b200.hex_phase.v1\",\n  \"backend\": "
      << io::json_quote(o.precision == ICP_FP32 ? "b200_fused_trace_fp32_fixed_point_histogram_cooperative_cdf"
                                                : "b200_fused_trace_fp64_fixed_point_histogram_cooperative_cdf")
      << ",\n  \"dtype\": \"<f8\",\n  \"order\": \"C\",\n"
      << "  \"theta_count\": " << o.ct << ",\n  \"phi_count\": " << o.cp << ",\n"
      << "  \"density_measure\": \"solid_angle_sr\",\n  \"cell_model\": \"constant_density_per_spherical_cell\",\n"
      << "  \"coordinates\": \"u=(1-cos(theta))/2; v=(phi+pi)/(2*pi)\",\n"
      << "  \"cdf_axis_order\": [\"phi_cell\",\"theta_edge\"],\n"
      << "  \"normalization\": \"integral_p_domega_equals_one\",\n"
      << "  \"direction_convention\": \"physical_propagation\",\n"
      << "  \"coordinate_contract_id\": \"ice.phase_cdf.ensemble_coordinates.v1\",\n"
      << "  \"sampling_frame_layout\": \"rows_xyz_columns_e0_e1_k\",\n"
      << "  \"sampling_frame_map\": \"local_column_to_ensemble_reference_column\",\n"
      << "  \"theta_zero\": \"forward\",\n  \"theta_pi\": \"backward\",\n  \"azimuth_periodic\": true,\n"
      << "  \"input_polarization\": \"unpolarized\",\n  \"incident_total_intensity\": 1,\n"
      << "  \"single_scattering_albedo\": 1,\n  \"stage\": \"incoherent\",\n"
      << "  \"wavelength_nm\": " << o.wavelength << ",\n  \"interior_index\": " << o.ior
      << ",\n  \"exterior_index\": " << o.external_ior << ",\n  \"query_frame_axis\": ";
    vec(g.ki);
    f << ",\n  \"query_frame_e0\": ";
    vec(g.e0);
    f << ",\n  \"sampling_frame_columns\": [[" << g.e0[0] << ',' << g.e1[0] << ',' << g.ki[0] << "],[" << g.e0[1] << ','
      << g.e1[1] << ',' << g.ki[1] << "],[" << g.e0[2] << ',' << g.e1[2] << ',' << g.ki[2] << "]],\n"
      << "  \"geometry\": {\"shape\": \"regular_hexagonal_prism\",\"body_long_axis\": [0,1,0],\"circumradius_mm\": " << o.R
      << ",\"full_length_mm\": " << o.L << ",\"projected_area_mm2\": " << area << ",\"projected_area_m2\": " << area * 1e-6
      << ",\"projected_area_method\": \"number_weighted_mean_of_convex_face_projections\"},\n"
      << "  \"cross_sections\": {\"model\": \"geometric_nonabsorbing\",\"scattering_mm2\": " << area
      << ",\"extinction_mm2\": " << area << ",\"absorption_mm2\": 0,\"scattering_m2\": " << area * 1e-6
      << ",\"extinction_m2\": " << area * 1e-6
      << ",\"absorption_m2\": 0,\"wave_scattering_cross_section_computed\": false,"
      << "\"assignment\": \"Csca=Cext=number_mean_Aproj; Cabs=0 (transport model)\"},\n"
      << "  \"material\": {\"model\": \"caller_supplied_real_index_at_wavelength\",\"wavelength_convention\": "
         "\"vacuum_nm\",\"absorption_model\": \"ignored_k_equals_zero\",\"birefringence\": false,"
         "\"automatic_ice_dispersion\": false},\n"
      << "  \"diffraction_policy\": {\"computed\": false,\"selected_output_includes_diffraction\": false},\n"
      << "  \"inter_path_interference\": false,\n  \"tir_relative_phase_retained\": true,\n"
      << "  \"orientation\": {\"representation\": \"weighted_discrete_SO3_number_measure\",\"rotation\": "
         "\"active_Hamilton_quaternion_wxyz_body_to_ensemble\",\"rows\": "
      << plan.nodes.size() << ",\"csv_sha256\": \"" << plan.sha256 << "\",\"input_weight_sum\": " << plan.input_weight_sum
      << ",\"roundoff_weight_normalization\": " << 1 / plan.input_weight_sum
      << ",\"plan_embedded\": false,\"retain_input_csv_for_reproduction\": true,\"symmetry_reduction\": false},\n"
      << "  \"sampling\": {\"generator\": \"counter_splitmix64_open52_v1\",\"planned_rays\": " << plan.total_samples
      << ",\"processed_rays\": " << r.trace.rays << ",\"outgoing_samples\": " << r.trace.outputs
      << ",\"batch_size\": " << o.batch << ",\"max_output_records_per_batch\": " << o.max_records
      << ",\"weight\": \"orientation_number_mass * Aproj / node_samples * path_power\","
      << "\"trace_precision\": \"" << (o.precision == ICP_FP32 ? "fp32" : "fp64") << "\"},\n"
      << "  \"transport_audit\": {\"escaped_mm2\": " << r.escaped_area_mm2 << ",\"unresolved_mm2\": "
      << r.unresolved_area_mm2 << ",\"unresolved_fraction\": " << r.unresolved_area_mm2 / area
      << ",\"maximum_balance_error\": " << r.trace.max_ray_balance
      << ",\"maximum_interface_balance_error\": " << r.trace.max_interface_balance
      << ",\"max_internal_hits\": " << o.max_hits << ",\"tail_tolerance_per_ray\": " << o.tail
      << ",\"max_unresolved_fraction\": " << o.max_unresolved << ",\"max_balance_error\": " << o.max_balance
      << ",\"per_ray_balance_tolerance\": " << per_ray_tolerance
      << ",\"cdf_normalized_to_resolved_escaped_mass\": true,\"status_counts\": {";
    for (int i = 0; i < 8; ++i) f << (i ? "," : "") << io::json_quote(kStatus[i]) << ':' << r.trace.status_counts[i];
    f << "}},\n  \"histogram\": {\"theta_count\": " << o.nt << ",\"phi_count\": " << o.np
      << ",\"mass_mm2\": " << r.histogram_mass_mm2 << ",\"relative_mass_audit_error\": " << r.histogram_relative_error
      << ",\"maximum_accepted_relative_mass_error\": " << o.max_hist_err
      << ",\"g_rays\": " << r.point_axial_mm2 / r.point_mass_mm2 << ",\"forward_axis_mass_mm2\": " << r.forward_mass_mm2
      << ",\"backward_axis_mass_mm2\": " << r.backward_mass_mm2
      << ",\"pole_policy\": \"axis_mass_uniform_in_azimuth_in_histogram_end_cap\",\"pole_roundoff_tolerance\": "
      << (o.precision == ICP_FP32 ? 0x1p-15 : 256 * 2.220446049250313e-16)
      << ",\"accumulation\": \"exact_fixed_point_2^-44_per_ray_power_then_binary64\""
      << ",\"boundary_snapped_samples\": " << r.trace.snapped
      << ",\"shared_memory_table_fallback_adds\": " << r.trace.fallback_adds << "},\n"
      << "  \"storage_processing\": {\"gaussian_sigma_degrees\": 0,\"mass_conservative_aggregation\": true,"
      << "\"coarsening_tv\": " << r.cdf.coarsening_tv << ",\"maximum_accepted_coarsening_tv\": " << o.max_tv
      << ",\"aggregation_integral_relative_change\": " << r.cdf.aggregation_relative_error
      << ",\"g_source\": " << r.cdf.g_source << ",\"g_stored\": " << r.cdf.g_stored << "},\n"
      << "  \"hg\": {\"g\": " << r.cdf.g_stored
      << ",\"method\": \"first_moment_of_saved_cell_pdf\",\"target\": \"saved_cdf\","
      << "\"cosine_convention\": \"dot(incident_propagation,outgoing_propagation)\"},\n"
      << "  \"quality\": {\"source_coverage_certified\": false,\"angular_convergence_certified\": false,"
      << "\"orientation_convergence_certified\": false,\"continuous_wave_solution_certified\": false,"
      << "\"cdf_l1_mass_error\": " << r.cdf.l1_error << ",\"cdf_maximum_cell_mass_error\": " << r.cdf.maximum_cell_error
      << ",\"cdf_lost_positive_cells\": " << r.cdf.lost_cells << ",\"cdf_lost_probability_mass\": " << r.cdf.lost_mass
      << ",\"maximum_accepted_l1_mass_error\": " << o.max_l1
      << ",\"maximum_accepted_lost_probability_mass\": " << o.max_lost << ",\"cdf_mass\": " << r.cdf.cdf_mass
      << "},\n  \"timing\": {\"trace_seconds\": " << r.seconds_trace << ",\"cdf_seconds\": " << r.seconds_cdf << "}\n}\n";
}

int run(const Options& o)
{
    const io::Plan plan = io::read_plan(o.orientations);
    icp_grid g{};
    g.nt = o.nt;
    g.np = o.np;
    H::V k;
    H::Frame fr;
    H::normalize({o.ki[0], o.ki[1], o.ki[2]}, k);
    H::make_frame(k, fr);
    g.ki[0] = k.x; g.ki[1] = k.y; g.ki[2] = k.z;
    g.e0[0] = fr.e0.x; g.e0[1] = fr.e0.y; g.e0[2] = fr.e0.z;
    g.e1[0] = fr.e1.x; g.e1[1] = fr.e1.y; g.e1[2] = fr.e1.z;
    // preflight every node before producing output (generate_hex_phase.cpp:82-88)
    std::vector<icp_orientation> nodes;
    for (const auto& n : plan.nodes) {
        icp_hex_node hn{};
        hn.circumradius_mm = o.R;
        hn.length_mm = o.L;
        if (!H::rotation(n.q[0], n.q[1], n.q[2], n.q[3], hn.rotation))
            throw std::invalid_argument("Quaternion must be unit length (w,x,y,z).");
        double area = 0;
        if (icp_hex_node_area(&hn, &g, &area)) throw std::invalid_argument(last_error());
        const double w = n.weight * area;
        if (!(w > 0) || !H::finite(w) || !(w / double(n.samples) > 0))
            throw std::runtime_error("Orientation area weight over/underflow.");
        nodes.push_back({{n.q[0], n.q[1], n.q[2], n.q[3]}, n.weight, n.samples, n.seed});
    }
    io::StagingDirectory dir(o.out);
    icp_record_report rep{};
    // per-ray acceptance bound: the reference's in binary64; binary32 conserves power exactly
    // in fixed point, and its per-ray balance is therefore checked with the same tolerance
    const double per_ray_tol = o.max_balance;
    try {
        icp_context* ctx = nullptr;
        if (icp_context_create(o.device, &ctx)) throw std::runtime_error(last_error());
        icp_hex_record rec{};
        rec.circumradius_mm = o.R;
        rec.length_mm = o.L;
        for (int i = 0; i < 3; ++i) rec.ki[i] = o.ki[i];
        rec.exterior_index = o.external_ior;
        rec.interior_index = o.ior;
        rec.tail_tolerance = o.tail;
        rec.balance_tolerance = per_ray_tol;
        rec.nt = o.nt; rec.np = o.np; rec.ct = o.ct; rec.cp = o.cp;
        rec.max_internal_hits = o.max_hits;
        rec.batch_size = (uint32_t)o.batch;
        rec.max_output_records = o.max_records;
        rec.precision = o.precision;
        rec.policy = {o.max_l1, o.max_lost, o.max_tv};
        std::vector<double> a(o.cp + 1), t((size_t)o.cp * (o.ct + 1)), u(o.ct + 1);
        const int st = icp_hex_generate(ctx, &rec, nodes.data(), (uint32_t)nodes.size(), a.data(), t.data(), u.data(), &rep);
        const std::string msg = st ? last_error() : std::string();
        icp_context_destroy(ctx);
        if (st) throw std::runtime_error(msg);
        // validate_composition (hex_phase/src/phase_generate.cpp:264-279)
        if (rep.trace.rejected_rays || rep.trace.rays != plan.total_samples || rep.trace.invalid)
            throw std::runtime_error("Hex trace is NOT accepted. Inspect per-ray statuses and unresolved power; do not renormalize it away.");
        const double area = rep.expected_area_mm2, esc = rep.escaped_area_mm2, unres = rep.unresolved_area_mm2;
        if (!(area > 0) || !(esc > 0) || !H::finite(esc) || !H::finite(unres) || unres < 0)
            throw std::runtime_error("Invalid integrated cross sections.");
        if (unres / area > o.max_unresolved) throw std::runtime_error("Unresolved light exceeds explicit global budget.");
        if (std::fabs((esc + unres) / area - 1) > o.max_balance)
            throw std::runtime_error("Orientation-weighted energy balance failed.");
        if (rep.histogram_relative_error > o.max_hist_err)
            throw std::runtime_error("Histogram mass differs from independent escaped-ray audit.");
        io::write_npy_f64(dir.staging() / "phi_cdf.npy", {o.cp + 1ull}, a.data(), a.size());
        io::write_npy_f64(dir.staging() / "theta_given_phi_cdf.npy", {o.cp, o.ct + 1ull}, t.data(), t.size());
        io::write_npy_f64(dir.staging() / "u_edges.npy", {o.ct + 1ull}, u.data(), u.size());
        write_metadata(dir.staging() / "metadata.json", o, plan, g, rep, per_ray_tol);
        dir.commit();
        std::cout.precision(17);
        std::cout << "saved=\"" << o.out << "\" g=" << rep.cdf.g_stored << " Csca_mm2=" << area
                  << " unresolved_fraction=" << unres / area << " histogram_relative_error=" << rep.histogram_relative_error
                  << " cdf_l1=" << rep.cdf.l1_error << " trace_s=" << rep.seconds_trace << " cdf_s=" << rep.seconds_cdf << '\n';
        return 0;
    } catch (const std::exception& e) {
        write_failure(dir.staging() / "failure.json", e.what(), rep);
        std::cerr << "Generation failed; retained " << dir.staging() << ": " << e.what() << '\n';
        return 2;
    }
}

} // namespace

int main(int argc, char** argv)
{
    try {
        if (argc == 2 && std::string_view(argv[1]) == "--help") {
            std::cout << "ice_generate_phase --out DIR --orientations CSV\n"
                         " --radius-mm R --length-mm L --ki X Y Z --ior N --wavelength-nm NM\n"
                         " --theta NT --phi NP [--cdf-theta CT --cdf-phi CP]\n"
                         " [--batch-size N --max-output-records N --max-internal-hits N --tail-tolerance E]\n"
                         " [--max-unresolved-fraction E --max-balance-error E --max-histogram-relative-error E]\n"
                         " [--cdf-max-l1 E --cdf-max-lost-mass E --max-coarsening-tv E]\n"
                         " [--device N --trace-precision fp32|fp64]   (B200 sm_100a; no CPU fallback)\n";
            return 0;
        }
        return run(parse(argc, argv));
    } catch (const std::exception& e) {
        std::cerr << "ice_generate_phase: " << e.what() << '\n';
        return 1;
    }
}
