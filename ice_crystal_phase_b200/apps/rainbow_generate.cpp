// rainbow_generate -- drop-in for the reference CLI of the same name (apps/generate_phase.cpp:
// 84-463) on the B200 C ABI (include/icp_b200.h): one water drop, traced on the GPU into a
// (u, phi) record written in the reference's output contract.
//
// Same options, defaults, error messages and exit codes (0 on success; 1 with
// "rainbow_generate: <msg>" on any failure, before or after the GPU work; the record appears
// only through <out>.part -> <out>).  Two optical models:
//   * --stage path | focal | diffraction (the default, as in the reference), and incoherent with
//     --optics lattice: the reference's wave-optics patch model, every step on the device -- the
//     --grid x --grid incident lattice traced through the four path families
//     (icp_lattice_trace), its outgoing patches (icp_patch_build), the all-hit query of the
//     --query-theta x --query-phi directions (icp_patch_query), folded-patch records for the
//     NeedsRefinement patches (icp_folded_prepare), the per-direction optics with the focal
//     stage (icp_patch_optics_folded), the Table-II diffraction (icp_rainbow_diffraction), the
//     stage density and its gate (icp_stage_density) and the stored CDF (icp_phase_cdf_build);
//   * --stage incoherent (--optics rays, its default): the Monte-Carlo R/T chain -- rays sampled
//     with the counter RNG uniformly over a disk that covers the drop (--rays, --seed), Fresnel /
//     Stokes splitting with up to --max-internal-hits interactions, every exit binned; the
//     ray-model extensions below apply to it only.
// Extensions, all announced in metadata.json:
//   * --optics lattice|rays selects the model of --stage incoherent (path, focal and diffraction
//     are lattice stages);
//   * --diffraction analytic adds a separately reported Fraunhofer stage of the circle of equal
//     traced area to the ray model (default none);
//   * --shape-coefficients c0,...,c7 replaces the Table-I shape of --radius-mm (which then only
//     sets the equal-volume radius), for both models;
//   * --trace-precision fp32|fp64 (ray model; default fp32, exact fixed-point power bookkeeping);
//   * --modules is accepted and ignored (the kernels are linked in).
#include <charconv>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <locale>
#include <memory>
#include <sstream>
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
    double water_index = 0, water_density = 0, water_residual = 0, water_width = 0;
    std::string stage = "diffraction";
    bool lattice = true;           // the reference's patch model (false: the ray model)
    bool ray_options = false;      // a ray-model extension was given
    double table_sigma_deg = 0;    // Table-II primary width (focal / diffraction stages)
    bool wavelength_given = false, index_given = false, state_given = false, sphere = false, allow_underresolved = false;
    Material material = Material::Water;
    uint32_t grid = 513, theta = 360, phi = 720, cdf_theta = 0, cdf_phi = 0;
    double inclination_deg = 20, max_l1 = 1e-10, max_lost = 1e-12, max_tv = 1, transition_contrast = 0.25;
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
                 "  --stage diffraction|focal|incoherent|path\n"
                 "  --focal-offsets 0,0,0,0 --transition-contrast C (0.25) --allow-underresolved\n"
                 "  --material water (default) --temperature-c T --pressure-pa P\n"
                 "  --material constant --ior N (explicit nondispersive reference)\n"
                 "  --cdf-max-l1 E --cdf-max-lost-mass E --device ORDINAL\n"
                 "  --cdf-theta T --cdf-phi P (integer divisors of query dimensions)\n"
                 "  --max-coarsening-tv E (quality policy, not a blur width)\n"
                 "  B200 extensions: --shape-coefficients c0,...,c7\n"
                 "  --optics lattice|rays (model of --stage incoherent; default rays; the other stages are lattice)\n"
                 "  ray model: --rays N (1e7) --seed S --max-internal-hits K (1024) --tail-tolerance E\n"
                 "  --trace-precision fp32|fp64 --diffraction none|analytic\n"
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
    bool help = false, optics_given = false;
    auto real = [](double& x) { return icp::cli::Flag{1, [&x](const V& v) { x = number(v[0]); }}; };
    auto count32 = [](uint32_t& x) { return icp::cli::Flag{1, [&x](const V& v) { x = positive_integer<uint32_t>(v[0]); }}; };
    auto refused = [](const char* why) { return icp::cli::Flag{1, [why](const V&) { throw std::invalid_argument(why); }}; };
    auto ray = [&c](icp::cli::Flag f) {
        auto inner = f.set;
        f.set = [inner, &c](const V& v) {
            inner(v);
            c.ray_options = true;
        };
        return f;
    };
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
             c.stage = std::string(v[0]);
         }}},
        {"--optics", {1, [&](const V& v) {
             if (v[0] == "lattice") c.lattice = true;
             else if (v[0] == "rays") c.lattice = false;
             else throw std::invalid_argument("--optics must be lattice or rays.");
             optics_given = true;
         }}},
        {"--focal-offsets", {1, [&](const V& v) { focal_offsets(v[0], c.focal_offsets); }}},
        // extensions
        {"--rays", {1, [&](const V& v) { c.rays = positive_integer<uint64_t>(v[0]); c.ray_options = true; }}},
        {"--seed", {1, [&](const V& v) {
             const auto r = std::from_chars(v[0].data(), v[0].data() + v[0].size(), c.seed);
             if (r.ec != std::errc{} || r.ptr != v[0].data() + v[0].size()) throw std::invalid_argument("Invalid seed.");
             c.ray_options = true;
         }}},
        {"--max-internal-hits", ray(count32(c.max_hits))},
        {"--tail-tolerance", ray(real(c.tail))},
        {"--max-unresolved-fraction", ray(real(c.max_unresolved))},
        {"--max-balance-error", ray(real(c.max_balance))},
        {"--max-histogram-relative-error", ray(real(c.max_hist_err))},
        {"--trace-precision", {1, [&](const V& v) {
             if (v[0] == "fp32") c.precision = ICP_FP32;
             else if (v[0] == "fp64") c.precision = ICP_FP64;
             else throw std::invalid_argument("--trace-precision must be fp32 or fp64.");
             c.ray_options = true;
         }}},
        {"--diffraction", {1, [&](const V& v) {
             if (v[0] == "none") c.analytic_diffraction = false;
             else if (v[0] == "analytic") c.analytic_diffraction = true;
             else throw std::invalid_argument("--diffraction must be none or analytic.");
             c.ray_options = true;
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
    if (c.stage == "incoherent") {
        if (!optics_given) c.lattice = false;
    } else if (optics_given && !c.lattice)
        throw std::invalid_argument("--optics rays applies to --stage incoherent only; path, focal and diffraction are lattice stages.");
    if (c.lattice && c.ray_options)
        throw std::invalid_argument("--rays, --seed, --max-internal-hits, --tail-tolerance, --trace-precision, --diffraction and the ray audits apply to the ray model (--stage incoherent --optics rays).");
    if (c.material == Material::Water) {
        if (c.index_given)
            throw std::invalid_argument("Do not specify --ior for water. It is evaluated from wavelength and state; use --material constant only for explicit reference calculations.");
        // evaluated at the wavelength the solver represents (binary32)
        icp_water_optics w{};
        if (icp_water_state(double(c.wavelength_nm), c.temperature_c, c.pressure_pa, &w))
            throw std::invalid_argument(last_error());
        c.water_index = w.refractive_index;
        c.water_density = w.density_kg_m3;
        c.water_residual = w.density_pressure_residual_pascal;
        c.water_width = w.density_bracket_width_kg_m3;
        c.interior_index = static_cast<float>(c.water_index);
    } else {
        if (!c.index_given || !(c.constant_index > 0 && c.constant_index <= (std::numeric_limits<float>::max)()))
            throw std::invalid_argument("Constant material requires a finite positive --ior.");
        if (c.state_given) throw std::invalid_argument("Temperature/pressure do not define a constant-index material.");
        c.interior_index = static_cast<float>(c.constant_index);
        if (!(c.interior_index > 0)) throw std::invalid_argument("Index underflows solver precision.");
    }
    // Table II (focal and diffraction stages), as the reference checks it here
    if ((c.stage == "focal" || c.stage == "diffraction") && icp_rainbow_table_sigma(c.radius_mm, &c.table_sigma_deg))
        throw std::invalid_argument("Table II covers radius 0.1..1.0 mm only. No bandwidth extrapolation is performed. The existing focal path also computes diffraction; use incoherent/path for out-of-table reference runs.");
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
          << "    \"density_model\": \"IAPWS R6-95(2018) liquid pressure EOS inversion\",\n"
          << "    \"temperature_kelvin\": " << c.temperature_c + 273.15 << ",\n"
          << "    \"pressure_pascal\": " << c.pressure_pa << ",\n"
          << "    \"density_kg_m3\": " << c.water_density << ",\n"
          << "    \"density_pressure_residual_pascal\": " << c.water_residual << ",\n"
          << "    \"density_bracket_width_kg_m3\": " << c.water_width;
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

// ------------------------------------------------------------------ the lattice (patch) model
// Device memory owned by a context, released before it.
struct DeviceBuffer {
    icp_context* ctx;
    void* ptr = nullptr;
    DeviceBuffer(icp_context* c, size_t bytes) : ctx(c)
    {
        if (icp_device_alloc(c, bytes ? bytes : 1, &ptr)) throw std::runtime_error(last_error());
    }
    ~DeviceBuffer() { if (ptr) icp_device_free(ctx, ptr); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    template <class T> T* as() const { return static_cast<T*>(ptr); }
};
struct Context {
    icp_context* ctx = nullptr;
    explicit Context(int device) { if (icp_context_create(device, &ctx)) throw std::runtime_error(last_error()); }
    ~Context() { icp_context_destroy(ctx); }
};
void check(int status)
{
    if (status) throw std::runtime_error(last_error());
}

uint32_t stage_code(const std::string& s)
{
    if (s == "incoherent") return ICP_STAGE_INCOHERENT;
    if (s == "path") return ICP_STAGE_PATH;
    if (s == "focal") return ICP_STAGE_FOCAL;
    return ICP_STAGE_DIFFRACTION;
}

struct LatticeRecord {
    icp_raindrop_config cfg{};
    icp_lattice_stats trace{};
    uint32_t patch_count = 0;
    uint64_t patch_histogram[8] = {};
    uint64_t hits = 0;
    uint32_t folded_records = 0;
    icp_folded_stats folded{};
    uint64_t folded_hits = 0, pending_directions = 0, error_directions = 0, corrected_hits = 0;
    icp_diffraction_stats diffraction{};
    icp_density_report density{};
    icp_cdf_report cdf{};
    double seconds = 0;
};

// PatchOptics + PhaseCdf of one drop (apps/generate_phase.cpp:421-441) on the device.
void lattice_record(const Command& c, LatticeRecord& R, std::vector<double>& phi, std::vector<double>& theta)
{
    const auto t0 = std::chrono::steady_clock::now();
    const double a = c.inclination_deg * H::kPi / 180.0;
    const float k_in[3] = {static_cast<float>(std::cos(a)), static_cast<float>(-std::sin(a)), 0.0f};
    float coef[8];
    for (int i = 0; i < 8; ++i) coef[i] = static_cast<float>(c.coefficients[i]);
    check(icp_raindrop_config_make(c.radius_mm, c.sphere ? 1 : 0, c.custom_shape ? coef : nullptr, c.wavelength_nm,
                                   c.interior_index, k_in, c.grid, c.grid, &R.cfg));
    const icp_raindrop_config& cfg = R.cfg;
    const uint32_t W = cfg.grid_width, Hh = cfg.grid_height;
    const uint64_t vertices = 4ull * W * Hh, cells = 4ull * (W - 1) * (Hh - 1);
    const uint64_t n = uint64_t(c.theta) * c.phi;
    const uint32_t stage = stage_code(c.stage);
    const bool wave = stage == ICP_STAGE_FOCAL || stage == ICP_STAGE_DIFFRACTION;
    Context ctx(c.device);
    {
        // 1. the incident lattice through the four path families, with the trace validation
        DeviceBuffer dv(ctx.ctx, sizeof(icp_outgoing_vertex) * vertices), d2(ctx.ctx, sizeof(icp_field32) * vertices);
        check(icp_lattice_trace(ctx.ctx, &cfg, dv.as<icp_outgoing_vertex>(), d2.as<icp_field32>(), &R.trace));
        if (R.trace.incomplete)
            throw std::runtime_error("Trace contains failed vertices: incomplete=" + std::to_string(R.trace.incomplete) +
                                     ", first_problem=" + std::to_string(R.trace.first_problem));
        // 2. outgoing patches
        DeviceBuffer dp(ctx.ctx, sizeof(icp_outgoing_patch) * cells), db(ctx.ctx, sizeof(icp_patch_aabb) * cells);
        check(icp_patch_build(ctx.ctx, dv.as<icp_outgoing_vertex>(), W, Hh, cfg.grid_half_extent,
                              dp.as<icp_outgoing_patch>(), db.as<icp_patch_aabb>(), nullptr, &R.patch_count,
                              R.patch_histogram));
        // 3. query directions about the solver's incident axis and basis
        const float axis[3] = {cfg.incident_direction.x, cfg.incident_direction.y, cfg.incident_direction.z};
        const float e0[3] = {cfg.incident_basis_x.x, cfg.incident_basis_x.y, cfg.incident_basis_x.z};
        std::vector<float> dirs(3 * n);
        check(icp_query_directions(c.theta, c.phi, axis, e0, dirs.data()));
        DeviceBuffer dd(ctx.ctx, sizeof(float) * dirs.size());
        check(icp_memcpy_h2d(ctx.ctx, dd.ptr, dirs.data(), sizeof(float) * dirs.size()));
        // 4. all-hit query: counted and filled in one call when the hits fit a first guess of
        //    four per direction, else sized by that call and filled by a second
        DeviceBuffer doff(ctx.ctx, sizeof(uint64_t) * (n + 1)), dsum(ctx.ctx, sizeof(icp_query_summary) * n);
        const auto* vtx = dv.as<const icp_outgoing_vertex>();
        uint64_t capacity = 4 * n;
        auto dh = std::make_unique<DeviceBuffer>(ctx.ctx, sizeof(icp_query_hit) * capacity);
        int qs = icp_patch_query(ctx.ctx, vtx, uint32_t(vertices), dp.as<icp_outgoing_patch>(), db.as<icp_patch_aabb>(),
                                 R.patch_count, dd.as<icp_vec3f>(), uint32_t(n), doff.as<uint64_t>(),
                                 dsum.as<icp_query_summary>(), dh->as<icp_query_hit>(), capacity, &R.hits);
        if (qs == ICP_ERR_CAPACITY) {
            capacity = R.hits;
            dh.reset();
            dh = std::make_unique<DeviceBuffer>(ctx.ctx, sizeof(icp_query_hit) * capacity);
            qs = icp_patch_query(ctx.ctx, vtx, uint32_t(vertices), dp.as<icp_outgoing_patch>(), db.as<icp_patch_aabb>(),
                                 R.patch_count, dd.as<icp_vec3f>(), uint32_t(n), doff.as<uint64_t>(),
                                 dsum.as<icp_query_summary>(), dh->as<icp_query_hit>(), capacity, &R.hits);
        }
        check(qs);
        {
            std::vector<icp_query_summary> sums(n);
            check(icp_memcpy_d2h(ctx.ctx, sums.data(), dsum.ptr, sizeof(icp_query_summary) * n));
            uint64_t errors = 0;
            for (const auto& q : sums) errors += (q.flags & (1u | 2u | 4u | 256u)) != 0u;
            if (errors) throw std::runtime_error("Patch query has numerical failures.");
        }
        // 5. folded-patch records of the NeedsRefinement patches
        icp_focal_config fc{};
        fc.grid_width = W;
        fc.grid_height = Hh;
        fc.grid_half_extent = cfg.grid_half_extent;
        for (int i = 0; i < 4; ++i) fc.quarter_turn_offsets[i] = c.focal_offsets[i];
        const float kin[3] = {axis[0], axis[1], axis[2]};
        DeviceBuffer dfi(ctx.ctx, sizeof(uint32_t) * (R.patch_count ? R.patch_count : 1));
        int st = icp_folded_prepare(ctx.ctx, vtx, uint32_t(vertices), dp.as<icp_outgoing_patch>(), R.patch_count, kin,
                                    wave ? &fc : nullptr, nullptr, dfi.as<uint32_t>(), nullptr, 0, &R.folded_records,
                                    &R.folded);
        if (st && st != ICP_ERR_CAPACITY) check(st);
        DeviceBuffer dfr(ctx.ctx, sizeof(icp_folded_record) * (R.folded_records ? R.folded_records : 1));
        if (R.folded_records)
            check(icp_folded_prepare(ctx.ctx, vtx, uint32_t(vertices), dp.as<icp_outgoing_patch>(), R.patch_count, kin,
                                     wave ? &fc : nullptr, nullptr, dfi.as<uint32_t>(), dfr.as<icp_folded_record>(),
                                     R.folded_records, &R.folded_records, &R.folded));
        // 6. per-direction optics (with the focal stage for focal / diffraction)
        icp_optics_input in{};
        in.vertices = vtx;
        in.patches = dp.as<icp_outgoing_patch>();
        in.directions = dd.as<icp_vec3f>();
        in.offsets = doff.as<uint64_t>();
        in.summaries = dsum.as<icp_query_summary>();
        in.hits = dh->as<icp_query_hit>();
        in.second_input_fields = d2.as<icp_field32>();
        in.hit_storage_count = R.hits;
        in.vertex_count = uint32_t(vertices);
        in.patch_count = R.patch_count;
        in.direction_count = uint32_t(n);
        in.second_input_count = uint32_t(vertices);
        in.incident_direction = cfg.incident_direction;
        in.incident_basis_x = cfg.incident_basis_x;
        in.input_polarization = 1; // unpolarised: the two unit input states
        const icp_folded_view view{dfi.as<uint32_t>(), dfr.as<icp_folded_record>(), R.patch_count, R.folded_records};
        DeviceBuffer dres(ctx.ctx, sizeof(icp_optical_result) * n);
        DeviceBuffer dfoc(ctx.ctx, wave ? sizeof(icp_focal_sample) * n : 1);
        check(icp_patch_optics_folded(ctx.ctx, &in, dres.as<icp_optical_result>(), wave ? &fc : nullptr,
                                      wave ? dfoc.as<icp_focal_sample>() : nullptr, R.folded_records ? &view : nullptr));
        {
            std::vector<icp_optical_result> res(n);
            check(icp_memcpy_d2h(ctx.ctx, res.data(), dres.ptr, sizeof(icp_optical_result) * n));
            for (const auto& r : res) {
                R.folded_hits += r.folded_hits;
                R.pending_directions += (r.flags & (32u | 64u | 128u)) != 0u;
                R.error_directions += (r.flags & 31u) != 0u;
            }
        }
        // 7. the Table-II diffraction of the focal stage
        DeviceBuffer dtr(ctx.ctx, stage == ICP_STAGE_DIFFRACTION ? sizeof(uint32_t) * n : 1);
        DeviceBuffer ddr(ctx.ctx, stage == ICP_STAGE_DIFFRACTION ? sizeof(icp_diffraction_result) * n : 1);
        if (stage == ICP_STAGE_DIFFRACTION) {
            icp_diffraction_config dc{c.table_sigma_deg * H::kPi / 180.0, 4.0, c.transition_contrast, 3.0};
            check(icp_rainbow_diffraction(ctx.ctx, dfoc.as<icp_focal_sample>(), c.theta, c.phi, &dc, dtr.as<uint32_t>(),
                                          ddr.as<icp_diffraction_result>(), nullptr, &R.diffraction));
        }
        // 8. the stage's density and the CDF builder's input gate (src/phase_cdf.cpp:320-328)
        DeviceBuffer dden(ctx.ctx, sizeof(double) * n);
        check(icp_stage_density(ctx.ctx, stage, dres.as<icp_optical_result>(), wave ? dfoc.as<icp_focal_sample>() : nullptr,
                                stage == ICP_STAGE_DIFFRACTION ? ddr.as<icp_diffraction_result>() : nullptr, n,
                                dden.as<double>(), &R.density));
        const auto& d = R.density;
        if (d.invalid_values || d.incomplete || !(d.maximum > 0) || (!c.allow_underresolved && d.underresolved)) {
            std::ostringstream m;
            m.imbue(std::locale::classic());
            m << std::setprecision(17) << "CDF input rejected: max_intensity=" << d.maximum
              << ", invalid_values=" << d.invalid_values << ", incomplete=" << d.incomplete
              << ", underresolved=" << d.underresolved << ", first_problem=" << d.first_problem << "\n[cdf-input] stage="
              << c.stage << " directions=" << n << " allow_underresolved=" << c.allow_underresolved;
            throw std::runtime_error(m.str());
        }
        // 9. the stored CDF of the density (cell mass = density x solid angle)
        DeviceBuffer dphi(ctx.ctx, sizeof(double) * phi.size()), dth(ctx.ctx, sizeof(double) * theta.size());
        const icp_cdf_policy pol{c.max_l1, c.max_lost, c.max_tv};
        check(icp_phase_cdf_build(ctx.ctx, dden.as<double>(), ICP_CDF_DENSITY, c.theta, c.phi, 0.0, 0.0, c.cdf_theta,
                                  c.cdf_phi, &pol, dphi.as<double>(), dth.as<double>(), &R.cdf));
        check(icp_memcpy_d2h(ctx.ctx, phi.data(), dphi.ptr, sizeof(double) * phi.size()));
        check(icp_memcpy_d2h(ctx.ctx, theta.data(), dth.ptr, sizeof(double) * theta.size()));
    }
    R.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// metadata.json of a lattice record: the reference writer's keys (apps/generate_phase.cpp:233-394)
// with this build's trace, patch, folded and query counters.
void write_lattice_metadata(const std::filesystem::path& path, const Command& c, const LatticeRecord& R, double area,
                            const double k[3], const double e[3], const double e1[3])
{
    auto f = json_out(path);
    const icp_raindrop_config& g = R.cfg;
    const bool water = c.material == Material::Water;
    const bool paper = c.stage == "focal" || c.stage == "diffraction";
    bool sphere = true;
    for (int n = 1; n < 8; ++n) sphere = sphere && g.coefficients[n] == 0;
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
      << "    \"projected_area_method\": \""
      << (sphere ? "analytic_sphere" : "convex_surface_integral_azimuth_analytic_gauss_legendre") << "\",\n"
      << "    \"projected_area_shape\": \"solver_shape_coefficients_promoted_to_fp64\",\n"
      << "    \"projected_area_converged\": true,\n"
      << "    \"projected_area_error_is_rigorous_bound\": false,\n"
      << "    \"convexity_verified\": true,\n"
      << "    \"convexity_method\": \"" << (sphere ? "analytic_sphere" : "dense_curvature_sampling") << "\",\n"
      << "    \"incident_axis_particle_frame\": [" << k[0] << ',' << k[1] << ',' << k[2] << "]\n  },\n"
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
      << "    \"wavelength_evaluated_nm\": " << g.wavelength_nm << ",\n"
      << "    \"ambient_model\": \"unit_absolute_index_air_approximation\",\n"
      << "    \"absorption_model\": \"ignored_k_equals_zero\",\n"
      << "    \"interior_index_evaluated_fp64\": " << (water ? c.water_index : c.constant_index) << ",\n"
      << "    \"interior_index_solver_fp32\": " << g.interior_index << ",\n"
      << "    \"exterior_index_solver\": " << g.exterior_index;
    if (water)
        f << ",\n    \"refractive_index_release\": \"IAPWS R9-97\",\n"
          << "    \"density_model\": \"IAPWS R6-95(2018) liquid pressure EOS inversion\",\n"
          << "    \"temperature_kelvin\": " << c.temperature_c + 273.15 << ",\n"
          << "    \"pressure_pascal\": " << c.pressure_pa << ",\n"
          << "    \"density_kg_m3\": " << c.water_density << ",\n"
          << "    \"density_pressure_residual_pascal\": " << c.water_residual << ",\n"
          << "    \"density_bracket_width_kg_m3\": " << c.water_width;
    f << "\n  },\n  \"diffraction_policy\": {\n"
      << "    \"name\": \"Sadeghi2012_TableII_local_v1\",\n"
      << "    \"computed\": " << (paper ? "true" : "false") << ",\n"
      << "    \"selected_output_includes_diffraction\": " << (c.stage == "diffraction" ? "true" : "false") << ",\n"
      << "    \"primary_sigma_degrees\": ";
    if (paper) f << c.table_sigma_deg;
    else f << "null";
    f << ",\n    \"secondary_sigma_degrees\": ";
    if (paper) f << 2 * c.table_sigma_deg;
    else f << "null";
    f << ",\n"
      << "    \"bandwidth_source\": \"paper Table II; secondary sigma x2\",\n"
      << "    \"between_table_radii\": \"linear interpolation (project convention)\",\n"
      << "    \"outside_table_radii\": \"reject\",\n"
      << "    \"wavelength_scaling\": \"none; no rule specified in Table II\",\n"
      << "    \"support_sigma\": 4,\n"
      << "    \"support_and_transition_detection_are_project_conventions\": true,\n"
      << "    \"physical_sigma_depends_on_grid\": false,\n"
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
      << "  \"stage\": \"" << c.stage << "\",\n"
      << "  \"radius_mm\": " << g.radius_mm << ",\n"
      << "  \"wavelength_nm\": " << g.wavelength_nm << ",\n"
      << "  \"exterior_index\": " << g.exterior_index << ",\n"
      << "  \"interior_index\": " << g.interior_index << ",\n"
      << "  \"force_sphere\": " << (c.sphere ? "true" : "false") << ",\n"
      << "  \"incident_grid\": [" << g.grid_width << ',' << g.grid_height << "],\n"
      << "  \"incident_grid_half_extent\": " << g.grid_half_extent << ",\n"
      << "  \"reference_distances\": [" << g.reference_distance << ',' << g.outgoing_reference_distance << "],\n"
      << "  \"query_frame_axis\": [" << g.incident_direction.x << ',' << g.incident_direction.y << ','
      << g.incident_direction.z << "],\n"
      << "  \"query_frame_e0\": [" << g.incident_basis_x.x << ',' << g.incident_basis_x.y << ',' << g.incident_basis_x.z
      << "],\n"
      << "  \"sampling_frame_columns\": [";
    for (unsigned i = 0; i < 3; ++i) f << (i ? "," : "") << '[' << e[i] << ',' << e1[i] << ',' << k[i] << ']';
    f << "],\n  \"shape_coefficients\": [";
    for (unsigned i = 0; i < 8; ++i) f << (i ? "," : "") << g.coefficients[i];
    f << "],\n  \"shape_source\": \"" << (c.custom_shape ? "command_line" : (c.sphere ? "sphere" : "Sadeghi2012_TableI"))
      << "\",\n  \"focal_quarter_turn_offsets\": [";
    for (unsigned i = 0; i < 4; ++i) f << (i ? "," : "") << c.focal_offsets[i];
    f << "],\n  \"diffraction_primary_sigma_degrees_setting\": 0,\n"
      << "  \"diffraction_zero_setting_selects_Table_II\": true,\n"
      << "  \"diffraction_transition_contrast\": " << c.transition_contrast << ",\n"
      << "  \"folded_branch_model\": \"finite_branch_area_ratio_v1\",\n"
      << "  \"folded_relative_tolerance\": 1e-08,\n"
      << "  \"generator_version\": \"icp_b200.rainbow.lattice.v1\",\n"
      << "  \"backend\": \"b200_lattice_trace_patch_query_folded_optics_cooperative_cdf\",\n"
      << "  \"lattice\": {\"vertices\": " << uint64_t(g.grid_width) * g.grid_height
      << ",\"intersection_fallbacks\": " << R.trace.intersection_fallbacks << ",\"snell_fallbacks\": "
      << R.trace.snell_fallbacks << ",\"status_counts\": [";
    for (int fam = 0; fam < 4; ++fam) {
        f << (fam ? "," : "") << '[';
        for (int st = 0; st < 8; ++st) f << (st ? "," : "") << R.trace.status_counts[fam][st];
        f << ']';
    }
    f << "]},\n  \"patches\": {\"count\": " << R.patch_count << ",\"status_counts\": [";
    for (int st = 0; st < 8; ++st) f << (st ? "," : "") << R.patch_histogram[st];
    f << "],\"query_hits\": " << R.hits << ",\"folded_candidates\": " << R.folded.candidates
      << ",\"folded_prepared\": " << R.folded.prepared << ",\"folded_unresolved\": " << R.folded.unresolved
      << ",\"folded_branches\": " << R.folded.branch_count << ",\"folded_evaluated_hits\": " << R.folded_hits
      << ",\"folded_largest_estimated_relative_error\": " << R.folded.largest_estimated_relative_error
      << ",\"pending_directions\": " << R.pending_directions << ",\"error_directions\": " << R.error_directions << "},\n";
    if (c.stage == "diffraction")
        f << "  \"rainbow_transitions\": {\"primary\": " << R.diffraction.primary_transitions
          << ",\"secondary\": " << R.diffraction.secondary_transitions << ",\"unknown\": "
          << R.diffraction.unknown_transitions << ",\"filtered_directions\": " << R.diffraction.filtered_directions
          << ",\"underresolved_directions\": " << R.diffraction.underresolved_directions << "},\n";
    f << "  \"quality\": {\n    \"source_coverage_certified\": false,\n"
      << "    \"angular_convergence_certified\": false,\n"
      << "    \"missing_source_cells\": " << R.patch_histogram[4] << ",\n"
      << "    \"invalid_values\": " << R.density.invalid_values << ",\n"
      << "    \"incomplete_directions\": " << R.density.incomplete << ",\n"
      << "    \"underresolved_directions\": " << R.density.underresolved << ",\n"
      << "    \"allow_underresolved\": " << (c.allow_underresolved ? "true" : "false") << ",\n"
      << "    \"cdf_l1_mass_error\": " << R.cdf.l1_error << ",\n"
      << "    \"cdf_maximum_cell_mass_error\": " << R.cdf.maximum_cell_error << ",\n"
      << "    \"cdf_lost_positive_cells\": " << R.cdf.lost_cells << ",\n"
      << "    \"cdf_lost_probability_mass\": " << R.cdf.lost_mass << ",\n"
      << "    \"maximum_accepted_l1_mass_error\": " << c.max_l1 << ",\n"
      << "    \"maximum_accepted_lost_probability_mass\": " << c.max_lost << "\n  },\n"
      << "  \"incident_inclination_degrees\": " << c.inclination_deg << ",\n"
      << "  \"query_grid\": [" << c.theta << ',' << c.phi << "],\n"
      << "  \"storage_processing\": {\n"
      << "    \"additional_filter\": \"none\",\n"
      << "    \"additional_filter_is_paper_diffraction\": false,\n"
      << "    \"sigma_degrees\": 0,\n"
      << "    \"aggregation\": \"nested_solid_angle_mass_preserving\",\n"
      << "    \"aggregation_integral_relative_change\": " << R.cdf.aggregation_relative_error << ",\n"
      << "    \"coarsening_tv\": " << R.cdf.coarsening_tv << ",\n"
      << "    \"maximum_accepted_coarsening_tv\": " << c.max_tv << "\n  },\n"
      << "  \"hg\": {\n    \"g\": " << R.cdf.g_stored << ",\n"
      << "    \"method\": \"first_moment_of_saved_cell_pdf\",\n"
      << "    \"target\": \"saved_cdf\",\n"
      << "    \"cosine_convention\": \"dot(incident_propagation,outgoing_propagation)\",\n"
      << "    \"axis_particle_frame\": [" << k[0] << ',' << k[1] << ',' << k[2] << "],\n"
      << "    \"g_source\": " << R.cdf.g_source << ",\n"
      << "    \"cdf_mass_check\": " << R.cdf.cdf_mass << "\n  },\n"
      << "  \"timing\": {\"device_seconds\": " << R.seconds << "}\n}\n";
}

int run_lattice(const Command& c)
{
    double k[3], e0[3], e1[3];
    if (icp_drop_frame(c.inclination_deg, k, e0, e1)) throw std::invalid_argument(last_error());
    double area = 0;
    if (icp_drop_projected_area(c.coefficients, double(c.radius_mm), k, &area)) throw std::invalid_argument(last_error());
    std::cout << std::setprecision(17) << "Material=" << (c.material == Material::Water ? "water_iapws_r9_97" : "constant")
              << " wavelength_vacuum_nm=" << c.wavelength_nm << " interior_index_solver=" << c.interior_index
              << " exterior_index=1; additional_storage_gaussian=none\n";
    if (c.stage == "focal" || c.stage == "diffraction")
        std::cout << "Local diffraction sigma_primary_deg=" << c.table_sigma_deg
                  << " sigma_secondary_deg=" << 2 * c.table_sigma_deg << " query_step_theta_deg=" << 180.0 / c.theta
                  << " query_step_phi_deg=" << 360.0 / c.phi << " (phi arc step additionally varies with theta)\n";
    LatticeRecord R;
    std::vector<double> phi(c.cdf_phi + 1), theta((size_t)c.cdf_phi * (c.cdf_theta + 1)), u(c.cdf_theta + 1);
    lattice_record(c, R, phi, theta);
    check(icp_u_edges(c.cdf_theta, u.data()));
    io::StagingDirectory destination(c.output);
    io::write_npy_f64(destination.staging() / "phi_cdf.npy", {c.cdf_phi + 1ull}, phi.data(), phi.size());
    io::write_npy_f64(destination.staging() / "theta_given_phi_cdf.npy", {c.cdf_phi, c.cdf_theta + 1ull}, theta.data(),
                      theta.size());
    io::write_npy_f64(destination.staging() / "u_edges.npy", {c.cdf_theta + 1ull}, u.data(), u.size());
    write_lattice_metadata(destination.staging() / "metadata.json", c, R, area, k, e0, e1);
    destination.commit();
    std::cout << "Saved NumPy CDF dataset: " << c.output << "; elapsed_seconds=" << R.seconds
              << "; CDF_L1_mass_error=" << R.cdf.l1_error << "; lost_probability_mass=" << R.cdf.lost_mass
              << "; saved_grid=" << c.cdf_theta << 'x' << c.cdf_phi << "; hg_g=" << R.cdf.g_stored
              << "; projected_area_mm2=" << area << "; coarsening_TV=" << R.cdf.coarsening_tv << '\n';
    return 0;
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
        return c.lattice ? run_lattice(c) : run(c);
    } catch (const std::exception& e) {
        std::cerr << "rainbow_generate: " << e.what() << '\n';
        return 1;
    }
}
