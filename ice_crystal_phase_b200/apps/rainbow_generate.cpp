// rainbow_generate -- drop-in for the reference CLI of the same name (apps/generate_phase.cpp:
// 84-463) on the B200 C ABI (include/icp_b200.h): one water drop, traced and binned on the GPU
// into a (u, phi) record written in the reference's output contract.
//
// Same options, defaults, error messages and exit codes (0 on success; 1 with
// "rainbow_generate: <msg>" on any failure, before or after the GPU work; the record appears
// only through <out>.part -> <out>).  Differences, all announced in metadata.json:
//   * rays are sampled with the counter RNG uniformly over a disk that covers the drop
//     (--rays, --seed) instead of the reference's deterministic --grid vertex lattice, which is
//     accepted and recorded only;
//   * the optical model is the geometric R/T chain with Fresnel/Stokes splitting and up to
//     --max-internal-hits interactions (stage "incoherent", the default here).  The reference's
//     wave-optics patch stages (path, focal and its Table-II "diffraction") are rejected by name:
//     the library has their device stages from an outgoing-ray lattice on (icp_patch_build,
//     icp_patch_query, icp_patch_optics, icp_rainbow_diffraction, icp_stage_density), but not the
//     lattice trace and folded patches that a record of those stages needs;
//   * --diffraction analytic adds a separately reported Fraunhofer stage of the circle of equal
//     traced area (default none);
//   * --shape-coefficients c0,...,c7 replaces the Table-I shape of --radius-mm (which then only
//     sets the equal-volume radius);
//   * --trace-precision fp32|fp64 (default fp32, exact fixed-point power bookkeeping);
//   * --modules is accepted and ignored (the kernels are linked in).
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <locale>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

#include "icp_b200.h"
#include "icp_cli_options.hpp"
#include "icp_host_math.hpp"
#include "icp_record_io.hpp"

namespace {

namespace H = icp::host;
namespace io = icp::io;

enum class Material { Water, Constant };

struct Command {
    std::filesystem::path output;
    float radius_mm = 1.0f, wavelength_nm = 0.0f, interior_index = 0.0f;
    double wavelength_requested_nm = 0, constant_index = 0, temperature_c = 20.0, pressure_pa = 101325.0;
    double water_index = 0, water_density = 0;
    bool wavelength_given = false, index_given = false, state_given = false, sphere = false, allow_underresolved = false;
    Material material = Material::Water;
    uint32_t grid = 513, theta = 360, phi = 720, cdf_theta = 0, cdf_phi = 0;
    double inclination_deg = 20, max_l1 = 1e-10, max_lost = 1e-12, max_tv = 1, transition_contrast = 0;
    unsigned focal_offsets[4] = {0, 0, 0, 0};
    int device = 0;
    // extensions
    uint64_t rays = 10'000'000, seed = 12345;
    uint32_t max_hits = 1024, precision = ICP_FP32;
    // rays trapped by total internal reflection in a non-spherical drop keep bouncing past any
    // interaction limit; their residual is reported and bounded globally
    double tail = 1e-12, max_unresolved = 1e-4, max_balance = 1e-10, max_hist_err = 1e-10;
    bool analytic_diffraction = false, custom_shape = false;
    double coefficients[8] = {};
};

double number(std::string_view s)
{
    double x = 0;
    const auto r = std::from_chars(s.data(), s.data() + s.size(), x);
    if (r.ec != std::errc{} || r.ptr != s.data() + s.size() || !std::isfinite(x))
        throw std::invalid_argument("Invalid numeric option.");
    return x;
}
template <class T> T positive_integer(std::string_view s)
{
    T x = 0;
    const auto r = std::from_chars(s.data(), s.data() + s.size(), x);
    if (r.ec != std::errc{} || r.ptr != s.data() + s.size() || x == 0)
        throw std::invalid_argument("Invalid positive integer option.");
    return x;
}

std::string last_error()
{
    char buf[2048];
    icp_last_error(buf, sizeof buf);
    return buf;
}

void print_help()
{
    std::cout << "rainbow_generate --out DIRECTORY [--sphere]\n"
                 "  --radius-mm R --wavelength-nm L (required, vacuum nm) --grid VERTICES_PER_AXIS (recorded only)\n"
                 "  --inclination-deg A --query-theta T --query-phi P\n"
                 "  --stage incoherent (geometric R/T chain; path|focal|diffraction are not part of this build)\n"
                 "  --material water (default) --temperature-c T --pressure-pa P\n"
                 "  --material constant --ior N (explicit nondispersive reference)\n"
                 "  --cdf-max-l1 E --cdf-max-lost-mass E --device ORDINAL\n"
                 "  --cdf-theta T --cdf-phi P (integer divisors of query dimensions)\n"
                 "  --max-coarsening-tv E (quality policy, not a blur width)\n"
                 "  B200 extensions: --rays N (1e7) --seed S --max-internal-hits K (1024) --tail-tolerance E\n"
                 "  --trace-precision fp32|fp64 --diffraction none|analytic --shape-coefficients c0,...,c7\n"
                 "  --max-unresolved-fraction E (1e-4) --max-balance-error E --max-histogram-relative-error E\n";
}

// Flags, defaults and messages of apps/generate_phase.cpp:84-223: a repeated flag keeps its last
// value (except --wavelength-nm), every flag other than the three switches carries one value.
void focal_offsets(std::string_view value, unsigned out[4])
{
    size_t begin = 0;
    for (unsigned k = 0; k < 4; ++k) {
        const auto end = value.find(',', begin);
        if ((k < 3 && end == std::string_view::npos) || (k == 3 && end != std::string_view::npos))
            throw std::invalid_argument("Expected four focal offsets.");
        const auto part = value.substr(begin, end == std::string_view::npos ? std::string_view::npos : end - begin);
        const auto r = std::from_chars(part.data(), part.data() + part.size(), out[k]);
        if (r.ec != std::errc{} || r.ptr != part.data() + part.size() || out[k] > 3)
            throw std::invalid_argument("Focal offsets must be 0..3.");
        begin = end == std::string_view::npos ? value.size() : end + 1;
    }
}
unsigned shape_coefficients(std::string_view value, double out[8])
{
    unsigned k = 0;
    for (size_t begin = 0;;) {
        const auto end = value.find(',', begin);
        if (k >= 8) throw std::invalid_argument("At most eight shape coefficients.");
        out[k++] = number(value.substr(begin, end == std::string_view::npos ? std::string_view::npos : end - begin));
        if (end == std::string_view::npos) return k;
        begin = end + 1;
    }
}

bool parse(int argc, char** argv, Command& c)
{
    using V = icp::cli::Values;
    std::string stage = "incoherent";
    bool help = false;
    auto real = [](double& x) { return icp::cli::Flag{1, [&x](const V& v) { x = number(v[0]); }}; };
    auto count32 = [](uint32_t& x) { return icp::cli::Flag{1, [&x](const V& v) { x = positive_integer<uint32_t>(v[0]); }}; };
    auto refused = [](const char* why) { return icp::cli::Flag{1, [why](const V&) { throw std::invalid_argument(why); }}; };
    const icp::cli::Table table = {
        {"--sphere", {0, [&](const V&) { c.sphere = true; }}},
        {"--allow-underresolved", {0, [&](const V&) { c.allow_underresolved = true; }}},
        {"--help", {0, [&](const V&) { help = true; }, true}},
        {"--out", {1, [&](const V& v) { c.output = std::string(v[0]); }}},
        {"--modules", {1, [](const V&) {}}},
        {"--radius-mm", {1, [&](const V& v) { c.radius_mm = static_cast<float>(number(v[0])); }}},
        {"--wavelength-nm", {1, [&](const V& v) {
             if (c.wavelength_given) throw std::invalid_argument("Duplicate --wavelength-nm.");
             c.wavelength_requested_nm = number(v[0]);
             c.wavelength_given = true;
             if (!(c.wavelength_requested_nm > 0 && c.wavelength_requested_nm <= (std::numeric_limits<float>::max)()))
                 throw std::invalid_argument("Wavelength must be positive and representable by the solver.");
             c.wavelength_nm = static_cast<float>(c.wavelength_requested_nm);
             if (!(c.wavelength_nm > 0)) throw std::invalid_argument("Wavelength underflows solver precision.");
         }}},
        {"--material", {1, [&](const V& v) {
             if (v[0] == "water") c.material = Material::Water;
             else if (v[0] == "constant") c.material = Material::Constant;
             else throw std::invalid_argument("Material must be water or constant.");
         }}},
        {"--temperature-c", {1, [&](const V& v) { c.temperature_c = number(v[0]); c.state_given = true; }}},
        {"--pressure-pa", {1, [&](const V& v) { c.pressure_pa = number(v[0]); c.state_given = true; }}},
        {"--ior", {1, [&](const V& v) { c.constant_index = number(v[0]); c.index_given = true; }}},
        {"--grid", count32(c.grid)},
        {"--query-theta", count32(c.theta)},
        {"--query-phi", count32(c.phi)},
        {"--inclination-deg", real(c.inclination_deg)},
        {"--cdf-theta", count32(c.cdf_theta)},
        {"--cdf-phi", count32(c.cdf_phi)},
        {"--storage-gaussian-sigma-deg", refused("Global storage blur has been removed from rainbow_generate. Remove this option; only local Table-II diffraction and cell-mass aggregation are applied.")},
        {"--storage-gaussian-support", refused("Global storage blur has been removed from rainbow_generate. Remove this option; only local Table-II diffraction and cell-mass aggregation are applied.")},
        {"--max-coarsening-tv", real(c.max_tv)},
        {"--diffraction-sigma-deg", refused("Manual diffraction width is not supported by rainbow_generate. Remove this option; Table II is selected automatically.")},
        {"--transition-contrast", real(c.transition_contrast)},
        {"--cdf-max-l1", real(c.max_l1)},
        {"--cdf-max-lost-mass", real(c.max_lost)},
        {"--device", {1, [&](const V& v) {
             const auto r = std::from_chars(v[0].data(), v[0].data() + v[0].size(), c.device);
             if (r.ec != std::errc{} || r.ptr != v[0].data() + v[0].size() || c.device < 0)
                 throw std::invalid_argument("Invalid device ordinal.");
         }}},
        {"--stage", {1, [&](const V& v) {
             if (v[0] != "incoherent" && v[0] != "path" && v[0] != "focal" && v[0] != "diffraction")
                 throw std::invalid_argument("Unknown stage.");
             stage = std::string(v[0]);
         }}},
        {"--focal-offsets", {1, [&](const V& v) { focal_offsets(v[0], c.focal_offsets); }}},
        // extensions
        {"--rays", {1, [&](const V& v) { c.rays = positive_integer<uint64_t>(v[0]); }}},
        {"--seed", {1, [&](const V& v) {
             const auto r = std::from_chars(v[0].data(), v[0].data() + v[0].size(), c.seed);
             if (r.ec != std::errc{} || r.ptr != v[0].data() + v[0].size()) throw std::invalid_argument("Invalid seed.");
         }}},
        {"--max-internal-hits", count32(c.max_hits)},
        {"--tail-tolerance", real(c.tail)},
        {"--max-unresolved-fraction", real(c.max_unresolved)},
        {"--max-balance-error", real(c.max_balance)},
        {"--max-histogram-relative-error", real(c.max_hist_err)},
        {"--trace-precision", {1, [&](const V& v) {
             if (v[0] == "fp32") c.precision = ICP_FP32;
             else if (v[0] == "fp64") c.precision = ICP_FP64;
             else throw std::invalid_argument("--trace-precision must be fp32 or fp64.");
         }}},
        {"--diffraction", {1, [&](const V& v) {
             if (v[0] == "none") c.analytic_diffraction = false;
             else if (v[0] == "analytic") c.analytic_diffraction = true;
             else throw std::invalid_argument("--diffraction must be none or analytic.");
         }}},
        {"--shape-coefficients", {1, [&](const V& v) {
             shape_coefficients(v[0], c.coefficients);
             c.custom_shape = true;
         }}},
    };
    const icp::cli::Style style{false, true, nullptr, [](const std::string&) { return std::string("Missing option value."); }};
    icp::cli::apply(argc, argv, table, style);
    if (help) {
        print_help();
        return false;
    }
    if (c.output.empty()) throw std::invalid_argument("--out is required.");
    if (!c.wavelength_given) throw std::invalid_argument("--wavelength-nm is required; there is no implicit wavelength.");
    if (stage != "incoherent")
        throw std::invalid_argument("Stage " + stage + " is the reference's wave-optics patch model; its lattice trace and folded patches are not available here (the later stages are, through the library's icp_patch_* and icp_rainbow_* calls); use --stage incoherent (optionally with --diffraction analytic).");
    if (c.material == Material::Water) {
        if (c.index_given)
            throw std::invalid_argument("Do not specify --ior for water. It is evaluated from wavelength and state; use --material constant only for explicit reference calculations.");
        // evaluated at the wavelength the solver represents (binary32)
        if (icp_water_index(double(c.wavelength_nm), c.temperature_c, c.pressure_pa, &c.water_index, &c.water_density))
            throw std::invalid_argument(last_error());
        c.interior_index = static_cast<float>(c.water_index);
    } else {
        if (!c.index_given || !(c.constant_index > 0 && c.constant_index <= (std::numeric_limits<float>::max)()))
            throw std::invalid_argument("Constant material requires a finite positive --ior.");
        if (c.state_given) throw std::invalid_argument("Temperature/pressure do not define a constant-index material.");
        c.interior_index = static_cast<float>(c.constant_index);
        if (!(c.interior_index > 0)) throw std::invalid_argument("Index underflows solver precision.");
    }
    if (c.cdf_theta == 0) c.cdf_theta = c.theta;
    if (c.cdf_phi == 0) c.cdf_phi = c.phi;
    if (c.cdf_theta > c.theta || c.cdf_phi > c.phi || c.theta % c.cdf_theta || c.phi % c.cdf_phi)
        throw std::invalid_argument("CDF dimensions must divide the query dimensions without upsampling.");
    if (!(c.max_tv >= 0 && c.max_tv <= 1)) throw std::invalid_argument("Coarsening TV limit must lie in [0,1].");
    // RaindropSettings::make_config (include/rainbow/raindrop_settings.hpp:20-45)
    double tmp[8];
    if (icp_drop_shape(c.radius_mm, c.sphere ? 1 : 0, tmp, nullptr, nullptr))
        throw std::invalid_argument("radius_mm must be in (0,3]; no coefficient extrapolation is implemented.");
    if (!(c.wavelength_nm >= 380.0f && c.wavelength_nm <= 830.0f))
        throw std::invalid_argument("wavelength_nm must be in [380,830] for this implementation.");
    if (!(c.interior_index >= 1.0f && c.interior_index <= 2.0f))
        throw std::invalid_argument("interior_index must be in [1,2]; exterior_index is 1.");
    if (c.grid < 2 || uint64_t(c.grid) * c.grid > uint64_t(0xffffffffu) / 4)
        throw std::invalid_argument("Invalid grid dimensions or 32-bit path-major index overflow.");
    if (!c.custom_shape) std::memcpy(c.coefficients, tmp, sizeof tmp);
    else if (c.sphere) throw std::invalid_argument("--sphere and --shape-coefficients are exclusive.");
    if (!(H::finite(c.tail) && c.tail >= 0 && c.tail < 1)) throw std::invalid_argument("Invalid tail tolerance.");
    for (double t : {c.max_unresolved, c.max_balance, c.max_hist_err})
        if (!H::finite(t) || t < 0 || t >= 1) throw std::invalid_argument("Invalid quality tolerance.");
    if (!(c.max_l1 >= 0 && c.max_l1 <= 2 && c.max_lost >= 0 && c.max_lost <= 1))
        throw std::invalid_argument("Invalid CDF quality policy.");
    if (uint64_t(c.theta) * c.phi > 0xffffffffull) throw std::invalid_argument("Unsupported phase grid dimensions.");
    if (std::filesystem::exists(c.output)) throw std::runtime_error("Output already exists.");
    auto partial = c.output;
    partial += ".part";
    if (std::filesystem::exists(partial))
        throw std::runtime_error("Previous .part directory exists; inspect it before recomputing.");
    return true;
}

std::ofstream json_out(const std::filesystem::path& p)
{
    std::ofstream f(p, std::ios::binary | std::ios::trunc);
    if (!f) throw std::runtime_error("Cannot open metadata.json.");
    f.exceptions(std::ios::badbit | std::ios::failbit);
    f.imbue(std::locale::classic());
    f << std::setprecision(17);
    return f;
}

const char* kStatus[8] = {"exhausted", "tail_tolerance_reached", "interaction_limit", "ambiguous_boundary",
                          "invalid_input", "numerical_failure", "output_overflow", "replay_mismatch"};

// metadata.json: the keys of the reference writer (apps/generate_phase.cpp:233-394), with the
// patch-model fields replaced by this build's ray sampling, transport and histogram audits.
void write_metadata(const std::filesystem::path& path, const Command& c, const icp_drop_report& r, double area,
                    const float kf[3], const float e0f[3])
{
    auto f = json_out(path);
    const double* k = r.ki;
    const double* e = r.e0;
    const double* e1 = r.e1;
    const bool water = c.material == Material::Water;
    bool sphere = true;
    for (int n = 1; n < 8; ++n) sphere = sphere && c.coefficients[n] == 0;
    f << "{\n"
      << "  \"coordinate_contract_id\": \"rainbow.phase_cdf.coordinates.v1\",\n"
      << "  \"direction_convention\": \"physical_propagation\",\n"
      << "  \"particle_frame_handedness\": \"right\",\n"
      << "  \"particle_up_axis\": [0,1,0],\n"
      << "  \"shape_polar_axis\": [0,-1,0],\n"
      << "  \"sampling_frame_layout\": \"rows_xyz_columns_e0_e1_k\",\n"
      << "  \"sampling_frame_map\": \"local_column_to_particle_column\",\n"
      << "  \"theta_zero\": \"forward\",\n  \"theta_pi\": \"backward\",\n  \"azimuth_periodic\": true,\n"
      << "  \"inclination_definition\": \"ki=(cos(alpha),-sin(alpha),0); alpha=0 is +x; positive alpha points downward\",\n"
      << "  \"geometry\": {\n"
      << "    \"projected_area_mm2\": " << area << ",\n"
      << "    \"projected_area_m2\": " << area * 1e-6 << ",\n"
      << "    \"projected_area_method\": \"" << (sphere ? "analytic_sphere" : "convex_surface_integral_azimuth_analytic_gauss_legendre")
      << "\",\n"
      << "    \"projected_area_shape\": \"solver_shape_coefficients_promoted_to_fp64\",\n"
      << "    \"projected_area_converged\": true,\n"
      << "    \"projected_area_error_is_rigorous_bound\": false,\n"
      << "    \"convexity_verified\": true,\n"
      << "    \"convexity_method\": \"" << (sphere ? "analytic_sphere" : "dense_curvature_sampling") << "\",\n"
      << "    \"incident_axis_particle_frame\": [" << k[0] << ',' << k[1] << ',' << k[2] << "],\n"
      << "    \"sampled_disk_area_mm2\": " << r.sampled_area_mm2 << ",\n"
      << "    \"traced_hit_area_mm2\": " << r.incident_area_mm2 << "\n  },\n"
      << "  \"cross_sections\": {\n"
      << "    \"model\": \"geometric_nonabsorbing\",\n"
      << "    \"scattering_mm2\": " << area << ",\n    \"extinction_mm2\": " << area << ",\n"
      << "    \"absorption_mm2\": 0,\n"
      << "    \"scattering_m2\": " << area * 1e-6 << ",\n    \"extinction_m2\": " << area * 1e-6 << ",\n"
      << "    \"absorption_m2\": 0,\n"
      << "    \"assignment\": \"Csca=Cext=Aproj; Cabs=0 (transport model assumption)\",\n"
      << "    \"wave_scattering_cross_section_computed\": false\n  },\n"
      << "  \"material\": {\n"
      << "    \"model\": \"" << (water ? "water_iapws_r9_97" : "constant") << "\",\n"
      << "    \"wavelength_convention\": \"vacuum_nm\",\n"
      << "    \"wavelength_requested_nm\": " << c.wavelength_requested_nm << ",\n"
      << "    \"wavelength_evaluated_nm\": " << c.wavelength_nm << ",\n"
      << "    \"ambient_model\": \"unit_absolute_index_air_approximation\",\n"
      << "    \"absorption_model\": \"ignored_k_equals_zero\",\n"
      << "    \"interior_index_evaluated_fp64\": " << (water ? c.water_index : c.constant_index) << ",\n"
      << "    \"interior_index_solver_fp32\": " << c.interior_index << ",\n"
      << "    \"exterior_index_solver\": 1";
    if (water)
        f << ",\n    \"refractive_index_release\": \"IAPWS R9-97\",\n"
          << "    \"density_model\": \"Tanaka2001/Kell1975 at 1 atm with UNESCO-1981 secant bulk modulus\",\n"
          << "    \"temperature_kelvin\": " << c.temperature_c + 273.15 << ",\n"
          << "    \"pressure_pascal\": " << c.pressure_pa << ",\n"
          << "    \"density_kg_m3\": " << c.water_density;
    f << "\n  },\n  \"diffraction_policy\": {\n"
      << "    \"name\": \"" << (c.analytic_diffraction ? "fraunhofer_equal_area_circle_v1" : "none") << "\",\n"
      << "    \"computed\": " << (c.analytic_diffraction ? "true" : "false") << ",\n"
      << "    \"selected_output_includes_diffraction\": " << (c.analytic_diffraction ? "true" : "false") << ",\n"
      << "    \"primary_sigma_degrees\": null,\n    \"secondary_sigma_degrees\": null,\n"
      << "    \"power_mm2\": " << r.diffraction_area_mm2 << ",\n"
      << "    \"model\": \"Rayleigh encircled energy 1-J0^2-J1^2 of the circle of equal traced area, forward hemisphere, uniform in azimuth\",\n"
      << "    \"query_dtheta_degrees\": " << 180.0 / c.theta << ",\n"
      << "    \"query_dphi_degrees\": " << 360.0 / c.phi << "\n  },\n";
    f << "  \"schema\": \"rainbow.phase_cdf.numpy.v2\",\n  \"complete\": true,\n"
      << "  \"dtype\": \"<f8\",\n  \"order\": \"C\",\n"
      << "  \"theta_count\": " << c.cdf_theta << ",\n  \"phi_count\": " << c.cdf_phi << ",\n"
      << "  \"density_measure\": \"solid_angle_sr\",\n"
      << "  \"cell_model\": \"constant_density_per_spherical_cell\",\n"
      << "  \"coordinates\": \"u=(1-cos(theta))/2; v=(phi+pi)/(2*pi)\",\n"
      << "  \"theta_definition\": \"angle_between_incident_and_outgoing_propagation_directions\",\n"
      << "  \"cdf_axis_order\": [\"phi_cell\", \"theta_edge\"],\n"
      << "  \"phi_range_rad\": [" << -H::kPi << ',' << H::kPi << "],\n"
      << "  \"normalization\": \"integral_p_domega_equals_one\",\n"
      << "  \"input_polarization\": \"unpolarized\",\n"
      << "  \"incident_total_intensity\": 1,\n  \"single_scattering_albedo\": 1,\n"
      << "  \"collision_model\": \"geometric_projected_area\",\n"
      << "  \"projected_area_storage\": \"metadata.geometry.projected_area_mm2\",\n"
      << "  \"stage\": \"incoherent\",\n"
      << "  \"radius_mm\": " << c.radius_mm << ",\n"
      << "  \"wavelength_nm\": " << c.wavelength_nm << ",\n"
      << "  \"exterior_index\": 1,\n"
      << "  \"interior_index\": " << c.interior_index << ",\n"
      << "  \"force_sphere\": " << (c.sphere ? "true" : "false") << ",\n"
      << "  \"incident_grid\": [" << c.grid << ',' << c.grid << "],\n"
      << "  \"incident_grid_used\": false,\n"
      << "  \"query_frame_axis\": [" << kf[0] << ',' << kf[1] << ',' << kf[2] << "],\n"
      << "  \"query_frame_e0\": [" << e0f[0] << ',' << e0f[1] << ',' << e0f[2] << "],\n"
      << "  \"sampling_frame_columns\": [";
    for (unsigned i = 0; i < 3; ++i) f << (i ? "," : "") << '[' << e[i] << ',' << e1[i] << ',' << k[i] << ']';
    f << "],\n  \"shape_coefficients\": [";
    for (unsigned i = 0; i < 8; ++i) f << (i ? "," : "") << c.coefficients[i];
    f << "],\n  \"shape_source\": \"" << (c.custom_shape ? "command_line" : (c.sphere ? "sphere" : "Sadeghi2012_TableI"))
      << "\",\n  \"focal_quarter_turn_offsets\": [";
    for (unsigned i = 0; i < 4; ++i) f << (i ? "," : "") << c.focal_offsets[i];
    f << "],\n  \"diffraction_transition_contrast\": " << c.transition_contrast << ",\n"
      << "  \"generator_version\": \"icp_b200.rainbow.v1\",\n"
      << "  \"backend\": \"" << (c.precision == ICP_FP32 ? "b200_fused_trace_fp32" : "b200_fused_trace_fp64")
      << "_fixed_point_histogram_cooperative_cdf\",\n"
      << "  \"sampling\": {\"generator\": \"counter_splitmix64_open52_v1\",\"method\": \"uniform_disk_covering_silhouette\","
      << "\"rays\": " << c.rays << ",\"seed\": " << c.seed << ",\"missed_rays\": " << r.trace.missed
      << ",\"outgoing_samples\": " << r.trace.outputs << ",\"weight\": \"disk_area / rays * path_power\","
      << "\"trace_precision\": \"" << (c.precision == ICP_FP32 ? "fp32" : "fp64") << "\"},\n"
      << "  \"transport_audit\": {\"incident_mm2\": " << r.incident_area_mm2 << ",\"escaped_mm2\": " << r.escaped_area_mm2
      << ",\"unresolved_mm2\": " << r.unresolved_area_mm2
      << ",\"unresolved_fraction\": " << r.unresolved_area_mm2 / r.incident_area_mm2
      << ",\"maximum_balance_error\": " << r.trace.max_ray_balance
      << ",\"maximum_interface_balance_error\": " << r.trace.max_interface_balance
      << ",\"max_internal_hits\": " << c.max_hits << ",\"tail_tolerance_per_ray\": " << c.tail
      << ",\"max_unresolved_fraction\": " << c.max_unresolved << ",\"max_balance_error\": " << c.max_balance
      << ",\"internal_encounters\": " << r.trace.encounters << ",\"status_counts\": {";
    for (int i = 0; i < 8; ++i) f << (i ? "," : "") << io::json_quote(kStatus[i]) << ':' << r.trace.status_counts[i];
    f << "}},\n  \"histogram\": {\"theta_count\": " << c.theta << ",\"phi_count\": " << c.phi
      << ",\"mass_mm2\": " << r.histogram_mass_mm2 << ",\"relative_mass_audit_error\": " << r.histogram_relative_error
      << ",\"maximum_accepted_relative_mass_error\": " << c.max_hist_err
      << ",\"forward_axis_mass_mm2\": " << r.forward_mass_mm2 << ",\"backward_axis_mass_mm2\": " << r.backward_mass_mm2
      << ",\"boundary_snapped_samples\": " << r.trace.snapped
      << ",\"shared_memory_table_fallback_adds\": " << r.trace.fallback_adds << "},\n"
      << "  \"quality\": {\n    \"source_coverage_certified\": false,\n"
      << "    \"angular_convergence_certified\": false,\n"
      << "    \"missing_source_cells\": 0,\n"
      << "    \"invalid_values\": " << r.trace.invalid << ",\n"
      << "    \"incomplete_directions\": 0,\n    \"underresolved_directions\": 0,\n"
      << "    \"allow_underresolved\": " << (c.allow_underresolved ? "true" : "false") << ",\n"
      << "    \"cdf_l1_mass_error\": " << r.cdf.l1_error << ",\n"
      << "    \"cdf_maximum_cell_mass_error\": " << r.cdf.maximum_cell_error << ",\n"
      << "    \"cdf_lost_positive_cells\": " << r.cdf.lost_cells << ",\n"
      << "    \"cdf_lost_probability_mass\": " << r.cdf.lost_mass << ",\n"
      << "    \"maximum_accepted_l1_mass_error\": " << c.max_l1 << ",\n"
      << "    \"maximum_accepted_lost_probability_mass\": " << c.max_lost << "\n  },\n"
      << "  \"incident_inclination_degrees\": " << c.inclination_deg << ",\n"
      << "  \"query_grid\": [" << c.theta << ',' << c.phi << "],\n"
      << "  \"storage_processing\": {\n"
      << "    \"additional_filter\": \"none\",\n"
      << "    \"additional_filter_is_paper_diffraction\": false,\n"
      << "    \"sigma_degrees\": 0,\n"
      << "    \"aggregation\": \"nested_solid_angle_mass_preserving\",\n"
      << "    \"aggregation_integral_relative_change\": " << r.cdf.aggregation_relative_error << ",\n"
      << "    \"coarsening_tv\": " << r.cdf.coarsening_tv << ",\n"
      << "    \"maximum_accepted_coarsening_tv\": " << c.max_tv << "\n  },\n"
      << "  \"hg\": {\n    \"g\": " << r.cdf.g_stored << ",\n"
      << "    \"method\": \"first_moment_of_saved_cell_pdf\",\n"
      << "    \"target\": \"saved_cdf\",\n"
      << "    \"cosine_convention\": \"dot(incident_propagation,outgoing_propagation)\",\n"
      << "    \"axis_particle_frame\": [" << k[0] << ',' << k[1] << ',' << k[2] << "],\n"
      << "    \"g_source\": " << r.cdf.g_source << ",\n"
      << "    \"cdf_mass_check\": " << r.cdf.cdf_mass << "\n  },\n"
      << "  \"timing\": {\"trace_seconds\": " << r.seconds_trace << ",\"cdf_seconds\": " << r.seconds_cdf << "}\n}\n";
}

int run(const Command& c)
{
    double k[3], e0[3], e1[3];
    if (icp_drop_frame(c.inclination_deg, k, e0, e1)) throw std::invalid_argument(last_error());
    // the binary32 incident axis and frame vector the reference's solver holds
    const double a = c.inclination_deg * H::kPi / 180.0;
    float kf[3] = {static_cast<float>(std::cos(a)), static_cast<float>(-std::sin(a)), 0.0f};
    const float kn = std::sqrt(std::fmaf(kf[0], kf[0], std::fmaf(kf[1], kf[1], kf[2] * kf[2])));
    for (float& v : kf) v /= kn;
    const float e0f[3] = {static_cast<float>(e0[0]), static_cast<float>(e0[1]), static_cast<float>(e0[2])};
    // independent CPU projected area, validated before the GPU work
    double area = 0;
    if (icp_drop_projected_area(c.coefficients, double(c.radius_mm), k, &area)) throw std::invalid_argument(last_error());
    std::cout << std::setprecision(17) << "Material=" << (c.material == Material::Water ? "water_iapws_r9_97" : "constant")
              << " wavelength_vacuum_nm=" << c.wavelength_nm << " interior_index_solver=" << c.interior_index
              << " exterior_index=1; additional_storage_gaussian=none\n";
    icp_drop_record rec{};
    rec.radius_mm = c.radius_mm;
    std::memcpy(rec.coefficients, c.coefficients, sizeof rec.coefficients);
    rec.inclination_deg = c.inclination_deg;
    rec.exterior_index = 1.0;
    rec.interior_index = c.interior_index;
    rec.wavelength_nm = c.wavelength_nm;
    rec.tail_tolerance = c.tail;
    rec.balance_tolerance = c.max_balance;
    rec.nt = c.theta; rec.np = c.phi; rec.ct = c.cdf_theta; rec.cp = c.cdf_phi;
    rec.max_internal_hits = c.max_hits;
    rec.precision = c.precision;
    rec.rays = c.rays;
    rec.seed = c.seed;
    rec.diffraction = c.analytic_diffraction ? 1u : 0u;
    rec.policy = {c.max_l1, c.max_lost, c.max_tv};
    icp_context* ctx = nullptr;
    if (icp_context_create(c.device, &ctx)) throw std::runtime_error(last_error());
    std::vector<double> phi(c.cdf_phi + 1), theta((size_t)c.cdf_phi * (c.cdf_theta + 1)), u(c.cdf_theta + 1);
    icp_drop_report rep{};
    const int st = icp_drop_generate(ctx, &rec, phi.data(), theta.data(), u.data(), &rep);
    const std::string msg = st ? last_error() : std::string();
    icp_context_destroy(ctx);
    if (st) throw std::runtime_error(msg);
    // transport audits (the prism record's validate_composition, hex_phase/src/phase_generate.cpp:68-83)
    const double inc = rep.incident_area_mm2, esc = rep.escaped_area_mm2, unres = rep.unresolved_area_mm2;
    // exhausted, tail-terminated and interaction-limited rays are accepted (the last with their
    // residual counted as unresolved); any other status, a per-ray balance failure or an
    // unbinnable exit rejects the record
    bool failed = rep.trace.invalid != 0 || !(rep.trace.max_ray_balance <= c.max_balance);
    for (int i = 3; i < 8; ++i) failed = failed || rep.trace.status_counts[i] != 0;
    if (failed || !(inc > 0) || !(esc > 0) || !H::finite(unres) || unres < 0)
        throw std::runtime_error("Drop trace is NOT accepted. Inspect per-ray statuses and unresolved power; do not renormalize it away.");
    if (unres / inc > c.max_unresolved) throw std::runtime_error("Unresolved light exceeds explicit global budget.");
    if (std::fabs((esc + unres) / inc - 1) > c.max_balance) throw std::runtime_error("Energy balance failed.");
    if (rep.histogram_relative_error > c.max_hist_err)
        throw std::runtime_error("Histogram mass differs from independent escaped-ray audit.");
    io::StagingDirectory destination(c.output);
    io::write_npy_f64(destination.staging() / "phi_cdf.npy", {c.cdf_phi + 1ull}, phi.data(), phi.size());
    io::write_npy_f64(destination.staging() / "theta_given_phi_cdf.npy", {c.cdf_phi, c.cdf_theta + 1ull}, theta.data(),
                      theta.size());
    io::write_npy_f64(destination.staging() / "u_edges.npy", {c.cdf_theta + 1ull}, u.data(), u.size());
    write_metadata(destination.staging() / "metadata.json", c, rep, area, kf, e0f);
    destination.commit();
    std::cout << "Saved NumPy CDF dataset: " << c.output << "; elapsed_seconds=" << rep.seconds_trace + rep.seconds_cdf
              << "; CDF_L1_mass_error=" << rep.cdf.l1_error << "; lost_probability_mass=" << rep.cdf.lost_mass
              << "; saved_grid=" << c.cdf_theta << 'x' << c.cdf_phi << "; hg_g=" << rep.cdf.g_stored
              << "; projected_area_mm2=" << area << "; coarsening_TV=" << rep.cdf.coarsening_tv << '\n';
    return 0;
}

} // namespace

int main(int argc, char** argv)
{
    try {
        Command c;
        if (!parse(argc, argv, c)) return 0;
        return run(c);
    } catch (const std::exception& e) {
        std::cerr << "rainbow_generate: " << e.what() << '\n';
        return 1;
    }
}
