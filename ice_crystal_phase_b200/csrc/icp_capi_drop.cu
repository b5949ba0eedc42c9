// icp_capi_drop.cu -- C ABI of the water-drop path (include/icp_b200.h, "water drops").
//
// Record flow (replaces rainbow_generate's OptiX trace -> patch build -> patch query ->
// patch optics -> PhaseCdf chain, apps/generate_phase.cpp:395-453): host FP64 inputs (shape,
// projected area, index, frame) -> one trace+bin launch of the drop geometry (rays sampled
// uniformly over a disk bounding the silhouette; misses carry no power) -> optional analytic
// diffraction rows -> the cooperative CDF build -> host arrays.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/icp_b200.h"
#include "../host/icp_drop_host.hpp"
#include "../host/icp_host_math.hpp"
#include "icp_internal.h"

using namespace icp;
namespace H = icp::host;

namespace {

thread_local char g_msg[1024];

int fail(int status, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_msg, sizeof g_msg, fmt, ap);
    va_end(ap);
    set_last_error(g_msg);
    return status;
}
int ok()
{
    set_last_error("");
    return ICP_OK;
}
#define ICP_CUDA(call)                                                                                  \
    do {                                                                                                \
        const cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return fail(ICP_ERR_DEVICE, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

} // namespace

bool icp::dropx::sphere_of(const double c[8])
{
    for (int n = 1; n < 8; ++n)
        if (c[n] != 0) return false;
    return true;
}

extern "C" int icp_water_index(double wavelength_nm, double temperature_c, double pressure_pa, double* index,
                               double* density)
{
    if (!index) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_water_index: null output");
    try {
        const auto s = H::water_optics(wavelength_nm, temperature_c, pressure_pa);
        *index = s.index;
        if (density) *density = s.density;
    } catch (const std::exception& e) {
        return fail(ICP_ERR_INVALID_ARGUMENT, "%s", e.what());
    }
    return ok();
}

extern "C" int icp_water_state(double wavelength_nm, double temperature_c, double pressure_pa, icp_water_optics* out)
{
    if (!out) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_water_state: null output");
    try {
        const auto s = H::water_optics(wavelength_nm, temperature_c, pressure_pa);
        *out = {s.temperature_k, s.pressure_pa, s.density, s.residual_pa, s.bracket_width, s.index};
    } catch (const std::exception& e) {
        return fail(ICP_ERR_INVALID_ARGUMENT, "%s", e.what());
    }
    return ok();
}

extern "C" int icp_drop_shape(double radius_mm, int sphere, double coefficients[8], double* inner, double* outer)
{
    if (!coefficients) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_drop_shape: null output");
    H::DropShapeHost s;
    if (!H::drop_shape_from_radius((float)radius_mm, sphere != 0, s))
        return fail(ICP_ERR_INVALID_ARGUMENT, "radius_mm must be in (0,3]; no coefficient extrapolation is implemented.");
    for (int n = 0; n < 8; ++n) coefficients[n] = s.c[n];
    if (inner) *inner = s.inner;
    if (outer) *outer = s.outer;
    return ok();
}

extern "C" int icp_drop_projected_area(const double coefficients[8], double radius_mm, const double k[3], double* area)
{
    if (!coefficients || !k || !area) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_drop_projected_area: null argument");
    try {
        *area = H::drop_projected_area(coefficients, radius_mm, k).area_mm2;
    } catch (const std::exception& e) {
        return fail(ICP_ERR_INVALID_ARGUMENT, "%s", e.what());
    }
    return ok();
}

extern "C" int icp_drop_frame(double inclination_deg, double k[3], double e0[3], double e1[3])
{
    if (!k || !e0 || !e1 || !H::finite(inclination_deg)) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_drop_frame: bad argument");
    const auto F = H::drop_frame(inclination_deg);
    for (int i = 0; i < 3; ++i) {
        k[i] = F.k[i];
        e0[i] = F.e0[i];
        e1[i] = F.e1[i];
    }
    return ok();
}

extern "C" int icp_drop_diffraction_rows(const double* u_edges, uint32_t nt, double area_mm2, double wavelength_nm,
                                         double* rows)
{
    if (!u_edges || !rows || !nt) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_drop_diffraction_rows: bad argument");
    if (!(area_mm2 > 0) || !H::finite(area_mm2) || !(wavelength_nm > 0) || !H::finite(wavelength_nm))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Diffraction needs a positive area and wavelength.");
    for (uint32_t i = 0; i < nt; ++i)
        if (!(u_edges[i + 1] > u_edges[i])) return fail(ICP_ERR_INVALID_ARGUMENT, "u edges must increase.");
    if (u_edges[0] != 0 || u_edges[nt] != 1) return fail(ICP_ERR_INVALID_ARGUMENT, "u edges must span [0, 1].");
    const std::vector<double> e(u_edges, u_edges + nt + 1);
    const auto r = H::diffraction_rows(e, area_mm2, wavelength_nm);
    std::memcpy(rows, r.data(), sizeof(double) * nt);
    return ok();
}

namespace icp::dropx {

// Bounding radius of the sampling disk and the conservative outer radius (units of a).
void drop_bounds(const double c[8], double& r_center, double& r_out)
{
    r_center = 1 + c[0];
    double s = 0;
    for (int n = 1; n < 8; ++n) s += std::fabs(c[n]);
    r_out = (1 + c[0] + s) * (1 + 1e-6) + 1e-6;
}

int validate_record(const icp_drop_record* r)
{
    if (!(r->radius_mm > 0) || !H::finite(r->radius_mm)) return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid drop radius.");
    for (int n = 0; n < 8; ++n)
        if (!H::finite(r->coefficients[n])) return fail(ICP_ERR_INVALID_ARGUMENT, "Nonfinite shape coefficient.");
    if (!sphere_of(r->coefficients) && !H::drop_convex(r->coefficients))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Drop shape is not strictly convex.");
    if (1 + r->coefficients[0] <= 0) return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid sphere radius.");
    if (!(r->exterior_index > 0 && r->interior_index > 0 && H::finite(r->exterior_index) && H::finite(r->interior_index)))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid refractive indices.");
    if (!(H::finite(r->tail_tolerance) && r->tail_tolerance >= 0 && r->tail_tolerance < 1))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid tail tolerance.");
    if (!r->max_internal_hits || !r->rays) return fail(ICP_ERR_INVALID_ARGUMENT, "Ray count and hit limit must be positive.");
    if (r->precision > 1) return fail(ICP_ERR_INVALID_ARGUMENT, "Unknown precision.");
    return ICP_OK;
}

} // namespace icp::dropx

using namespace icp::dropx;

extern "C" int icp_drop_sampling_area(const double coefficients[8], double radius_mm, double* area_mm2)
{
    if (!coefficients || !area_mm2 || !(radius_mm > 0) || !H::finite(radius_mm))
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_drop_sampling_area: bad argument");
    double r_center, r_out;
    drop_bounds(coefficients, r_center, r_out);
    const double disk = sphere_of(coefficients) ? r_center : r_out;
    *area_mm2 = H::kPi * disk * disk * radius_mm * radius_mm;
    return ok();
}

namespace icp::dropx {

// Kernel description of one drop record (shared by the single-record and batched launches).
HexLaunch drop_launch(const icp_drop_record* r, const icp_grid* g, const double* d_edges, const float* edges_f,
                      double* d_mass, void* d_stats, double area_weight, uint32_t slots)
{
    const auto F = H::drop_frame(r->inclination_deg);
    HexLaunch L{};
    L.geometry = 1;
    std::memcpy(L.coeff, r->coefficients, sizeof L.coeff);
    drop_bounds(r->coefficients, L.r_center, L.r_out);
    L.sphere = sphere_of(r->coefficients) ? 1u : 0u;
    L.disk = L.sphere ? L.r_center : L.r_out;
    L.back = 2 * L.r_out + 1;
    for (int i = 0; i < 3; ++i) {
        L.k[i] = F.k[i];
        L.ke0[i] = F.e0[i];
        L.e1[i] = F.e1[i];
        L.ki[i] = g->ki[i];
        L.e0[i] = g->e0[i];
        L.e1g[i] = g->e1[i];
    }
    L.rot[0] = L.rot[4] = L.rot[8] = 1.0;
    L.n_ext = r->exterior_index;
    L.n_int = r->interior_index;
    L.tail = r->tail_tolerance;
    L.bal_tol = r->balance_tolerance;
    L.seed = r->seed;
    L.total = r->rays;
    L.first = 0;
    L.count = r->rays;
    L.max_hits = r->max_internal_hits;
    L.batch_size = 1u << 20;
    L.batch_out = nullptr;
    L.nt = g->nt;
    L.np = g->np;
    L.edges_d = d_edges;
    L.edges_f = edges_f;
    L.mass = d_mass;
    L.to_mass = area_weight * 0x1p-44;
    L.stats = d_stats;
    L.hash_slots = slots;
    return L;
}

// Drop exits spread continuously over the sphere, so a shared table of a few thousand cells
// saturates within one block and only adds probes: by default exits go straight to the FP64
// histogram (fire-and-forget L2 reductions).  A table can still be requested.
int table_slots(const icp_tuning& t, uint32_t& slots)
{
    slots = 0u;
    if (t.hash_slots) slots = t.hash_slots == 1 ? 0u : t.hash_slots;
    if (slots & (slots - 1)) return fail(ICP_ERR_INVALID_ARGUMENT, "hash_slots must be a power of two");
    return ICP_OK;
}

// Enqueues the trace of rays [first, first+count) into d_mass / d_stats (no synchronisation).
int drop_trace_enqueue(icp_context* c, const icp_drop_record* r, uint64_t first, uint64_t count, double area_weight,
                       const icp_grid* g, const double* d_edges, double* d_mass, void* d_stats)
{
    const bool f32 = r->precision == ICP_FP32;
    const uint32_t max_threads = f32 ? drop_trace_threads_f32() : drop_trace_threads_f64();
    const uint32_t threads = r->tuning.block_threads ? r->tuning.block_threads : max_threads;
    if (threads < 64 || threads > max_threads || threads % 32)
        return fail(ICP_ERR_INVALID_ARGUMENT, "block_threads must be 64..%u, multiple of 32", max_threads);
    uint32_t slots;
    if (const int e = table_slots(r->tuning, slots)) return e;
    int per_sm = f32 ? drop_blocks_per_sm_f32(slots, g->nt, threads) : drop_blocks_per_sm_f64(slots, g->nt, threads);
    if (per_sm <= 0) return fail(ICP_ERR_DEVICE, "drop trace kernel cannot be resident");
    if (r->tuning.blocks_per_sm) per_sm = std::min<int>(per_sm, (int)r->tuning.blocks_per_sm);
    const uint32_t wpb = threads / 32;
    uint64_t blocks = (uint64_t)per_sm * c->sms;
    blocks = std::max<uint64_t>(1, std::min<uint64_t>(blocks, (count + 64ull * wpb - 1) / (64ull * wpb)));
    const uint64_t piece = blocks * wpb * lane_rays_max(r->max_internal_hits);
    if (f32)
        if (const int e = ensure_float_edges(c, d_edges, g->nt)) return e;
    HexLaunch L = drop_launch(r, g, d_edges, (const float*)c->edges_f.ptr, d_mass, d_stats, area_weight, slots);
    L.block_threads = threads;
    L.blocks = (uint32_t)blocks;
    for (uint64_t off = 0; off < count; off += piece) {
        L.first = first + off;
        L.count = std::min<uint64_t>(piece, count - off);
        const int e = f32 ? launch_drop_f32(L, c->stream) : launch_drop_f64(L, c->stream);
        count_launch();
        if (e) return fail(ICP_ERR_DEVICE, "drop trace launch failed: %s", cudaGetErrorString((cudaError_t)e));
    }
    return ICP_OK;
}

int grid_of(const icp_drop_record* r, icp_grid& g)
{
    const auto F = H::drop_frame(r->inclination_deg);
    g = icp_grid{};
    g.nt = r->nt;
    g.np = r->np;
    for (int i = 0; i < 3; ++i) {
        g.ki[i] = F.k[i];
        g.e0[i] = F.e0[i];
        g.e1[i] = F.e1[i];
    }
    return ICP_OK;
}

int validate_grid(const icp_drop_record* r)
{
    if (!r->nt || !r->np || (uint64_t)r->nt * r->np > 0xffffffffull || !r->ct || !r->cp || r->ct > r->nt ||
        r->cp > r->np || r->nt % r->ct || r->np % r->cp)
        return fail(ICP_ERR_INVALID_ARGUMENT, "CDF dimensions must divide the query dimensions without upsampling.");
    if (r->diffraction && !(r->wavelength_nm > 0 && H::finite(r->wavelength_nm)))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Diffraction needs a wavelength.");
    const icp_cdf_policy& p = r->policy;
    if (!(H::finite(p.max_l1_error) && p.max_l1_error >= 0 && p.max_l1_error <= 2 && H::finite(p.max_lost_mass) &&
          p.max_lost_mass >= 0 && p.max_lost_mass <= 1 && H::finite(p.max_coarsening_tv) && p.max_coarsening_tv >= 0 &&
          p.max_coarsening_tv <= 1))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid CDF quality policy.");
    return ICP_OK;
}

// Host part of a record's report from its trace counters, CDF report and diffraction power.
int finish_report(const icp_drop_record* r, const unsigned char* raw_stats, const CdfDeviceReport& cdf, double power,
                  double weight, icp_drop_report* rep)
{
    icp_trace_stats& T = rep->trace;
    T = icp_trace_stats{};
    stats_accumulate(raw_stats, &T);
    const uint64_t hits = T.rays - T.missed;
    rep->incident_area_mm2 = weight * double(hits);
    rep->escaped_area_mm2 = weight * T.escaped;
    rep->unresolved_area_mm2 = weight * T.unresolved;
    rep->forward_mass_mm2 = weight * T.forward_pole;
    rep->backward_mass_mm2 = weight * T.backward_pole;
    rep->point_axial_mm2 = weight * T.point_axial;
    rep->diffraction_area_mm2 = r->diffraction ? power : 0.0;
    if (!(hits > 0)) return fail(ICP_ERR_AUDIT, "No sampled ray hit the drop.");
    const int st = cdf_finish(cdf, r->policy, &rep->cdf);
    rep->histogram_mass_mm2 = rep->cdf.fine_mass;
    const double expected = rep->escaped_area_mm2 + rep->diffraction_area_mm2;
    rep->histogram_relative_error = std::fabs(rep->histogram_mass_mm2 / expected - 1);
    return st;
}

double projected_area_of(const icp_drop_record* r, int& status)
{
    status = ICP_OK;
    try {
        const auto F = H::drop_frame(r->inclination_deg);
        return H::drop_projected_area(r->coefficients, r->radius_mm, F.k).area_mm2;
    } catch (const std::exception& e) {
        status = fail(ICP_ERR_INVALID_ARGUMENT, "%s", e.what());
        return 0;
    }
}

} // namespace icp::dropx

extern "C" int icp_drop_trace_bin(icp_context* c, const icp_drop_record* r, uint64_t first, uint64_t count,
                                  double area_weight, const icp_grid* g, const double* d_edges, double* d_mass,
                                  icp_trace_stats* stats)
{
    if (!c || !r || !g || !d_edges || !d_mass || !stats) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_drop_trace_bin: null argument");
    if (const int v = validate_record(r)) return v;
    if (first >= r->rays || count > r->rays - first) return fail(ICP_ERR_INVALID_ARGUMENT, "Batch is outside the ray range.");
    if (!(area_weight > 0) || !H::finite(area_weight)) return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid area weight.");
    if (count == 0) return ok();
    ICP_CUDA(cudaSetDevice(c->device));
    ICP_CUDA(c->stats.ensure(hex_stats_bytes()));
    ICP_CUDA(cudaMemsetAsync(c->stats.ptr, 0, hex_stats_bytes(), c->stream));
    if (const int e = drop_trace_enqueue(c, r, first, count, area_weight, g, d_edges, d_mass, c->stats.ptr)) return e;
    std::vector<unsigned char> raw(hex_stats_bytes());
    ICP_CUDA(cudaMemcpyAsync(raw.data(), c->stats.ptr, raw.size(), cudaMemcpyDeviceToHost, c->stream));
    ICP_CUDA(cudaStreamSynchronize(c->stream));
    stats_accumulate(raw.data(), stats);
    return ok();
}

namespace {

// One record: trace + bin, diffraction rows and the CDF enqueued back to back, one
// synchronisation.  host = true: phi/theta/u are host arrays (the CDF goes through context
// scratch and is copied back); host = false: phi/theta/u are caller device arrays written in
// place (u may be null).
int drop_record(icp_context* c, const icp_drop_record* r, double* phi_out, double* theta_out, double* u_out, bool host,
                icp_drop_report* rep)
{
    std::memset(rep, 0, sizeof *rep);
    if (const int v = validate_record(r)) return v;
    if (const int v = validate_grid(r)) return v;
    ICP_CUDA(cudaSetDevice(c->device));
    icp_grid g;
    grid_of(r, g);
    for (int i = 0; i < 3; ++i) {
        rep->ki[i] = g.ki[i];
        rep->e0[i] = g.e0[i];
        rep->e1[i] = g.e1[i];
    }
    double disk_area = 0;
    if (const int e = icp_drop_sampling_area(r->coefficients, r->radius_mm, &disk_area)) return e;
    rep->sampled_area_mm2 = disk_area;
    const double weight = disk_area / double(r->rays);
    std::vector<double> edges;
    if (!H::u_edges(r->nt, edges)) return fail(ICP_ERR_INVALID_ARGUMENT, "Angular cells cannot be represented in binary64.");
    const uint64_t cells = (uint64_t)r->nt * r->np;
    const size_t sb = hex_stats_bytes();
    ICP_CUDA(c->rec_edges.ensure(sizeof(double) * (r->nt + 1)));
    ICP_CUDA(c->rec_mass.ensure(sizeof(double) * cells));
    ICP_CUDA(c->stats.ensure(sb));
    ICP_CUDA(c->rows.ensure(sizeof(double) * (r->nt + 1)));
    ICP_CUDA(c->dargs.ensure(sizeof(DiffractionArgs)));
    ICP_CUDA(c->cdf_report.ensure_zeroed(sizeof(CdfDeviceReport), c->stream));
    ICP_CUDA(c->cdf_sync.ensure_zeroed(2 * sizeof(unsigned), c->stream));
    if (host) {
        ICP_CUDA(c->rec_phi.ensure(sizeof(double) * (r->cp + 1)));
        ICP_CUDA(c->rec_theta.ensure(sizeof(double) * (size_t)r->cp * (r->ct + 1)));
    }
    double* d_phi = host ? (double*)c->rec_phi.ptr : phi_out;
    double* d_theta = host ? (double*)c->rec_theta.ptr : theta_out;
    double* d_mass = (double*)c->rec_mass.ptr;
    double* d_rows = (double*)c->rows.ptr;
    ICP_CUDA(cudaEventRecord(c->ev0, c->stream));
    ICP_CUDA(cudaMemcpyAsync(c->rec_edges.ptr, edges.data(), sizeof(double) * (r->nt + 1), cudaMemcpyHostToDevice, c->stream));
    ICP_CUDA(cudaMemsetAsync(d_mass, 0, sizeof(double) * cells, c->stream));
    ICP_CUDA(cudaMemsetAsync(c->stats.ptr, 0, sb, c->stream));
    const double* d_edges = (const double*)c->rec_edges.ptr;
    if (const int e = drop_trace_enqueue(c, r, 0, r->rays, weight, &g, d_edges, d_mass, c->stats.ptr)) return e;
    if (r->diffraction) {
        DiffractionArgs a{};
        a.edges = d_edges;
        a.rays = (const unsigned long long*)c->stats.ptr + devstats_rays_word();
        a.missed_offset = devstats_missed_word() - devstats_rays_word();
        a.row_add = d_rows;
        a.power = d_rows + r->nt;
        a.weight = weight;
        a.wavelength_nm = r->wavelength_nm;
        a.nt = r->nt;
        a.np = r->np;
        ICP_CUDA(cudaMemcpyAsync(c->dargs.ptr, &a, sizeof a, cudaMemcpyHostToDevice, c->stream));
        const int e = launch_diffraction_rows((const DiffractionArgs*)c->dargs.ptr, 1, r->nt, c->stream);
        count_launch();
        if (e) return fail(ICP_ERR_DEVICE, "diffraction launch failed: %s", cudaGetErrorString((cudaError_t)e));
    }
    ICP_CUDA(cudaEventRecord(c->ev1, c->stream));
    if (const int e = cdf_enqueue(c, d_mass, r->nt, r->np, r->ct, r->cp, d_edges, 0.0, 0.0,
                                  (const unsigned long long*)c->stats.ptr + devstats_fwd_word(), weight,
                                  r->diffraction ? d_rows : nullptr, d_phi, d_theta,
                                  (CdfDeviceReport*)c->cdf_report.ptr, (unsigned*)c->cdf_sync.ptr))
        return e;
    ICP_CUDA(cudaEventRecord(c->ev2, c->stream));
    std::vector<unsigned char> raw(sb);
    CdfDeviceReport cdf{};
    double power = 0;
    ICP_CUDA(cudaMemcpyAsync(raw.data(), c->stats.ptr, sb, cudaMemcpyDeviceToHost, c->stream));
    ICP_CUDA(cudaMemcpyAsync(&cdf, c->cdf_report.ptr, sizeof cdf, cudaMemcpyDeviceToHost, c->stream));
    if (r->diffraction) ICP_CUDA(cudaMemcpyAsync(&power, d_rows + r->nt, sizeof power, cudaMemcpyDeviceToHost, c->stream));
    const uint32_t dt = r->nt / r->ct;
    std::vector<double> coarse(r->ct + 1);
    for (uint32_t i = 0; i <= r->ct; ++i) coarse[i] = edges[(size_t)i * dt];
    if (host) {
        ICP_CUDA(cudaMemcpyAsync(phi_out, d_phi, sizeof(double) * (r->cp + 1), cudaMemcpyDeviceToHost, c->stream));
        ICP_CUDA(cudaMemcpyAsync(theta_out, d_theta, sizeof(double) * (size_t)r->cp * (r->ct + 1),
                                 cudaMemcpyDeviceToHost, c->stream));
        std::memcpy(u_out, coarse.data(), sizeof(double) * (r->ct + 1));
    } else if (u_out) {
        ICP_CUDA(cudaMemcpyAsync(u_out, coarse.data(), sizeof(double) * (r->ct + 1), cudaMemcpyHostToDevice, c->stream));
    }
    // the projected area (CPU, binary64) overlaps the device work
    int area_status = ICP_OK;
    rep->projected_area_mm2 = projected_area_of(r, area_status);
    ICP_CUDA(cudaStreamSynchronize(c->stream));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    rep->seconds_trace = ms * 1e-3;
    cudaEventElapsedTime(&ms, c->ev1, c->ev2);
    rep->seconds_cdf = ms * 1e-3;
    if (cdf.timeout)
        if (const int e = cdf_clear(c, c->cdf_report.ptr, c->cdf_sync.ptr, 1)) return e;
    if (area_status) return area_status;
    const int st = finish_report(r, raw.data(), cdf, power, weight, rep);
    return st == ICP_OK ? ok() : st;
}

} // namespace

extern "C" int icp_drop_generate(icp_context* c, const icp_drop_record* r, double* h_phi, double* h_theta, double* h_u,
                                 icp_drop_report* rep)
{
    if (!c || !r || !h_phi || !h_theta || !h_u || !rep) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_drop_generate: null argument");
    return drop_record(c, r, h_phi, h_theta, h_u, true, rep);
}

extern "C" int icp_drop_generate_device(icp_context* c, const icp_drop_record* r, double* d_phi, double* d_theta,
                                        double* d_u, icp_drop_report* rep)
{
    if (!c || !r || !d_phi || !d_theta || !rep)
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_drop_generate_device: null argument");
    return drop_record(c, r, d_phi, d_theta, d_u, false, rep);
}
