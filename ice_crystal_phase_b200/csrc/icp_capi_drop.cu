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

// Adds rows[i] / np to every cell of row i (analytic diffraction stage).
__global__ void add_rows(double* mass, const double* rows, uint32_t nt, uint32_t np)
{
    const uint64_t n = (uint64_t)nt * np;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
        mass[k] += rows[k / np] / np;
}

bool sphere_of(const double c[8])
{
    for (int n = 1; n < 8; ++n)
        if (c[n] != 0) return false;
    return true;
}

} // namespace

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

namespace {

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

} // namespace

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
    const auto F = H::drop_frame(r->inclination_deg);
    const bool f32 = r->precision == ICP_FP32;
    const uint32_t threads = r->tuning.block_threads ? r->tuning.block_threads : 256u;
    if (threads < 64 || threads > 256 || threads % 32) return fail(ICP_ERR_INVALID_ARGUMENT, "block_threads must be 64..256, multiple of 32");
    uint32_t slots = 4096u;
    if (r->tuning.hash_slots) slots = r->tuning.hash_slots == 1 ? 0u : r->tuning.hash_slots;
    if (slots & (slots - 1)) return fail(ICP_ERR_INVALID_ARGUMENT, "hash_slots must be a power of two");
    int per_sm = f32 ? drop_blocks_per_sm_f32(slots, g->nt, threads) : drop_blocks_per_sm_f64(slots, g->nt, threads);
    if (per_sm <= 0) return fail(ICP_ERR_DEVICE, "drop trace kernel cannot be resident");
    if (r->tuning.blocks_per_sm) per_sm = std::min<int>(per_sm, (int)r->tuning.blocks_per_sm);
    const uint32_t wpb = threads / 32;
    uint64_t blocks = (uint64_t)per_sm * c->sms;
    blocks = std::max<uint64_t>(1, std::min<uint64_t>(blocks, (count + 64ull * wpb - 1) / (64ull * wpb)));
    const uint64_t piece = blocks * wpb * 65536ull;
    ICP_CUDA(c->stats.ensure(hex_stats_bytes()));
    ICP_CUDA(cudaMemsetAsync(c->stats.ptr, 0, hex_stats_bytes(), c->stream));
    if (f32)
        if (const int e = ensure_float_edges(c, d_edges, g->nt)) return e;
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
    L.max_hits = r->max_internal_hits;
    L.batch_size = 1u << 20;
    L.batch_out = nullptr;
    L.nt = g->nt;
    L.np = g->np;
    L.edges_d = d_edges;
    L.edges_f = (const float*)c->edges_f.ptr;
    L.mass = d_mass;
    L.to_mass = area_weight * 0x1p-44;
    L.stats = c->stats.ptr;
    L.hash_slots = slots;
    L.block_threads = threads;
    L.blocks = (uint32_t)blocks;
    for (uint64_t off = 0; off < count; off += piece) {
        L.first = first + off;
        L.count = std::min<uint64_t>(piece, count - off);
        const int e = f32 ? launch_drop_f32(L, c->stream) : launch_drop_f64(L, c->stream);
        count_launch();
        if (e) return fail(ICP_ERR_DEVICE, "drop trace launch failed: %s", cudaGetErrorString((cudaError_t)e));
    }
    std::vector<unsigned char> raw(hex_stats_bytes());
    ICP_CUDA(cudaMemcpyAsync(raw.data(), c->stats.ptr, raw.size(), cudaMemcpyDeviceToHost, c->stream));
    ICP_CUDA(cudaStreamSynchronize(c->stream));
    stats_accumulate(raw.data(), stats);
    return ok();
}

extern "C" int icp_drop_generate(icp_context* c, const icp_drop_record* r, double* h_phi, double* h_theta, double* h_u,
                                 icp_drop_report* rep)
{
    if (!c || !r || !h_phi || !h_theta || !h_u || !rep) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_drop_generate: null argument");
    std::memset(rep, 0, sizeof *rep);
    if (const int v = validate_record(r)) return v;
    if (!r->nt || !r->np || (uint64_t)r->nt * r->np > 0xffffffffull || !r->ct || !r->cp || r->ct > r->nt ||
        r->cp > r->np || r->nt % r->ct || r->np % r->cp)
        return fail(ICP_ERR_INVALID_ARGUMENT, "CDF dimensions must divide the query dimensions without upsampling.");
    if (r->diffraction && !(r->wavelength_nm > 0)) return fail(ICP_ERR_INVALID_ARGUMENT, "Diffraction needs a wavelength.");
    ICP_CUDA(cudaSetDevice(c->device));
    const auto F = H::drop_frame(r->inclination_deg);
    icp_grid g{};
    g.nt = r->nt;
    g.np = r->np;
    for (int i = 0; i < 3; ++i) {
        g.ki[i] = F.k[i];
        g.e0[i] = F.e0[i];
        g.e1[i] = F.e1[i];
        rep->ki[i] = F.k[i];
        rep->e0[i] = F.e0[i];
        rep->e1[i] = F.e1[i];
    }
    double area = 0;
    try {
        area = H::drop_projected_area(r->coefficients, r->radius_mm, F.k).area_mm2;
    } catch (const std::exception& e) {
        return fail(ICP_ERR_INVALID_ARGUMENT, "%s", e.what());
    }
    rep->projected_area_mm2 = area;
    double disk_area = 0;
    if (const int e = icp_drop_sampling_area(r->coefficients, r->radius_mm, &disk_area)) return e;
    rep->sampled_area_mm2 = disk_area;
    const double weight = disk_area / double(r->rays);
    std::vector<double> edges;
    if (!H::u_edges(r->nt, edges)) return fail(ICP_ERR_INVALID_ARGUMENT, "Angular cells cannot be represented in binary64.");
    const uint64_t cells = (uint64_t)r->nt * r->np;
    ICP_CUDA(c->rec_edges.ensure(sizeof(double) * (r->nt + 1)));
    ICP_CUDA(c->rec_mass.ensure(sizeof(double) * cells));
    ICP_CUDA(c->rec_phi.ensure(sizeof(double) * (r->cp + 1)));
    ICP_CUDA(c->rec_theta.ensure(sizeof(double) * (size_t)r->cp * (r->ct + 1)));
    ICP_CUDA(cudaMemcpyAsync(c->rec_edges.ptr, edges.data(), sizeof(double) * (r->nt + 1), cudaMemcpyHostToDevice, c->stream));
    ICP_CUDA(cudaMemsetAsync(c->rec_mass.ptr, 0, sizeof(double) * cells, c->stream));
    ICP_CUDA(cudaEventRecord(c->ev0, c->stream));
    icp_trace_stats& T = rep->trace;
    if (const int e = icp_drop_trace_bin(c, r, 0, r->rays, weight, &g, (const double*)c->rec_edges.ptr,
                                         (double*)c->rec_mass.ptr, &T))
        return e;
    const uint64_t hits = T.rays - T.missed;
    rep->incident_area_mm2 = weight * double(hits);
    rep->escaped_area_mm2 = weight * T.escaped;
    rep->unresolved_area_mm2 = weight * T.unresolved;
    rep->forward_mass_mm2 = weight * T.forward_pole;
    rep->backward_mass_mm2 = weight * T.backward_pole;
    rep->point_axial_mm2 = weight * T.point_axial;
    if (r->diffraction) {
        // separately reported stage: Fraunhofer lobe carrying as much power as the geometric part
        const auto rows = H::diffraction_rows(edges, rep->incident_area_mm2, r->wavelength_nm);
        for (double v : rows) rep->diffraction_area_mm2 += v;
        ICP_CUDA(c->rows.ensure(sizeof(double) * r->nt));
        ICP_CUDA(cudaMemcpyAsync(c->rows.ptr, rows.data(), sizeof(double) * r->nt, cudaMemcpyHostToDevice, c->stream));
        add_rows<<<(unsigned)std::min<uint64_t>(4096, (cells + 255) / 256), 256, 0, c->stream>>>(
            (double*)c->rec_mass.ptr, (const double*)c->rows.ptr, r->nt, r->np);
        count_launch();
        ICP_CUDA(cudaGetLastError());
    }
    ICP_CUDA(cudaEventRecord(c->ev1, c->stream));
    ICP_CUDA(cudaEventSynchronize(c->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    rep->seconds_trace = ms * 1e-3;
    if (!(hits > 0)) return fail(ICP_ERR_AUDIT, "No sampled ray hit the drop.");
    ICP_CUDA(cudaEventRecord(c->ev0, c->stream));
    const int cr = icp_phase_cdf_build(c, (const double*)c->rec_mass.ptr, ICP_CDF_MASS, r->nt, r->np,
                                       rep->forward_mass_mm2, rep->backward_mass_mm2, r->ct, r->cp, &r->policy,
                                       (double*)c->rec_phi.ptr, (double*)c->rec_theta.ptr, &rep->cdf);
    ICP_CUDA(cudaEventRecord(c->ev1, c->stream));
    rep->histogram_mass_mm2 = rep->cdf.fine_mass;
    if (cr != ICP_OK) return cr;
    ICP_CUDA(cudaMemcpyAsync(h_phi, c->rec_phi.ptr, sizeof(double) * (r->cp + 1), cudaMemcpyDeviceToHost, c->stream));
    ICP_CUDA(cudaMemcpyAsync(h_theta, c->rec_theta.ptr, sizeof(double) * (size_t)r->cp * (r->ct + 1),
                             cudaMemcpyDeviceToHost, c->stream));
    ICP_CUDA(cudaStreamSynchronize(c->stream));
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    rep->seconds_cdf = ms * 1e-3;
    const uint32_t dt = r->nt / r->ct;
    for (uint32_t i = 0; i <= r->ct; ++i) h_u[i] = edges[(size_t)i * dt];
    const double expected = rep->escaped_area_mm2 + rep->diffraction_area_mm2;
    rep->histogram_relative_error = std::fabs(rep->histogram_mass_mm2 / expected - 1);
    return ok();
}
