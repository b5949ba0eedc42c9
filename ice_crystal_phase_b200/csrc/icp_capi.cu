// icp_capi.cu -- implementation of the C ABI declared in include/icp_b200.h.
//
// The context owns one CUDA stream and reusable device scratch (u edges, statistics,
// CDF partials and counters).  Every entry point validates its arguments, enqueues on the
// context stream and synchronises before returning, as the reference stage owners do
// (hex_trace/src/hex_trace_cuda.cpp:127-174, hex_phase/src/phase_cuda.cpp:334-375,
// src/phase_cdf.cpp:211-223).  Errors are reported as status codes with a per-thread
// message (icp_last_error); nothing throws across the ABI.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/icp_b200.h"
#include "../host/icp_ice_optics.hpp"
#include "../host/icp_host_math.hpp"
#include "icp_internal.h"


using namespace icp;
namespace H = icp::host;

namespace {

thread_local std::string g_error;
std::atomic<unsigned long long> g_launches{0};

int fail(int status, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_error = buf;
    return status;
}
int ok()
{
    g_error.clear();
    return ICP_OK;
}

#define ICP_CUDA(call)                                                                                  \
    do {                                                                                                \
        const cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                          \
            return fail(ICP_ERR_DEVICE, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                        __LINE__);                                                                      \
    } while (0)

__global__ void edges_to_float(const double* in, float* out, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)in[i];
}

} // namespace

namespace icp {
void set_last_error(const char* message) { g_error = message; }
void count_launch() { ++g_launches; }
} // namespace icp

extern "C" {

uint32_t icp_abi_version(void) { return ICP_ABI_VERSION; }

unsigned long long icp_kernel_launches(void) { return g_launches.load(); }

size_t icp_last_error(char* buffer, size_t n)
{
    if (buffer && n) {
        const size_t m = std::min(n - 1, g_error.size());
        std::memcpy(buffer, g_error.data(), m);
        buffer[m] = '\0';
    }
    return g_error.size();
}

int icp_context_create(int device, icp_context** out)
{
    if (!out) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_context_create: null output pointer");
    *out = nullptr;
    int count = 0;
    ICP_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count)
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_context_create: device %d outside [0,%d)", device, count);
    ICP_CUDA(cudaSetDevice(device));
    int major = 0;
    ICP_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    if (major < 10)
        return fail(ICP_ERR_DEVICE, "icp_context_create: device %d is compute capability %d.x; this library targets sm_100a",
                    device, major);
    auto* c = new icp_context();
    c->device = device;
    cudaError_t e = cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess && c->sms <= 0) e = cudaErrorInvalidDevice;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev2);
    if (e != cudaSuccess) {
        icp_context_destroy(c);
        return fail(ICP_ERR_DEVICE, "icp_context_create: %s", cudaGetErrorString(e));
    }
    *out = c;
    return ok();
}

int icp_context_destroy(icp_context* c)
{
    if (!c) return ok();
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    Scratch* all[] = {&c->stats,      &c->edges_f,    &c->cdf_partial,  &c->cdf_report,  &c->cdf_sync,
                      &c->cdf_colsum, &c->rec_edges,  &c->rec_mass,     &c->rec_phi,     &c->rec_theta,
                      &c->rec_batch,  &c->rows,       &c->dargs,        &c->b_table,     &c->b_chunks,
                      &c->b_queue,    &c->b_stats,    &c->b_mass,       &c->b_rows,      &c->b_dargs,
                      &c->b_reports,  &c->b_sync,     &c->b_phi,        &c->b_theta,     &c->mlp_error,
                      &c->cdfb_partial, &c->cdfb_colsum, &c->cdfb_recs, &c->atlas_trace, &c->atlas_coupling,
                      &c->rainbow,    &c->patches,
                      &c->query,      &c->query_list, &c->stage_audit, &c->cdf_edges, &c->lattice, &c->folded, &c->atlas_list};
    for (Scratch* s : all) s->release();
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->ev2) cudaEventDestroy(c->ev2);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return ok();
}

int icp_context_set_wait_limit(icp_context* c, uint32_t limit)
{
    if (!c) return fail(ICP_ERR_INVALID_ARGUMENT, "null context");
    c->wait_limit = limit;
    return ok();
}

int icp_context_synchronize(icp_context* c)
{
    if (!c) return fail(ICP_ERR_INVALID_ARGUMENT, "null context");
    ICP_CUDA(cudaSetDevice(c->device));
    ICP_CUDA(cudaStreamSynchronize(c->stream));
    return ok();
}

void* icp_context_stream(icp_context* c) { return c ? (void*)c->stream : nullptr; }

int icp_device_alloc(icp_context* c, size_t bytes, void** out)
{
    if (!c || !out) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_device_alloc: null argument");
    ICP_CUDA(cudaSetDevice(c->device));
    const cudaError_t e = cudaMalloc(out, bytes ? bytes : 1);
    if (e != cudaSuccess) {
        cudaGetLastError(); // a refused allocation leaves the context usable: clear the error
        *out = nullptr;
        return fail(ICP_ERR_DEVICE, "icp_device_alloc: cudaMalloc of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    return ok();
}
int icp_device_free(icp_context* c, void* ptr)
{
    if (!c) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_device_free: null context");
    ICP_CUDA(cudaSetDevice(c->device));
    ICP_CUDA(cudaStreamSynchronize(c->stream));
    ICP_CUDA(cudaFree(ptr));
    return ok();
}
int icp_memcpy_h2d(icp_context* c, void* dst, const void* src, size_t bytes)
{
    if (!c) return fail(ICP_ERR_INVALID_ARGUMENT, "null context");
    ICP_CUDA(cudaSetDevice(c->device));
    ICP_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
    ICP_CUDA(cudaStreamSynchronize(c->stream));
    return ok();
}
int icp_memcpy_d2h(icp_context* c, void* dst, const void* src, size_t bytes)
{
    if (!c) return fail(ICP_ERR_INVALID_ARGUMENT, "null context");
    ICP_CUDA(cudaSetDevice(c->device));
    ICP_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
    ICP_CUDA(cudaStreamSynchronize(c->stream));
    return ok();
}
int icp_memset_d(icp_context* c, void* dst, int value, size_t bytes)
{
    if (!c) return fail(ICP_ERR_INVALID_ARGUMENT, "null context");
    ICP_CUDA(cudaSetDevice(c->device));
    ICP_CUDA(cudaMemsetAsync(dst, value, bytes, c->stream));
    ICP_CUDA(cudaStreamSynchronize(c->stream));
    return ok();
}

int icp_ice_index(double wavelength_nm, icp_ice_state* out)
{
    if (!out) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_ice_index: null argument");
    std::memset(out, 0, sizeof *out);
    if (!std::isfinite(wavelength_nm) || wavelength_nm < 200.0 || wavelength_nm > 1100.0)
        return fail(ICP_ERR_INVALID_ARGUMENT,
                    "Warren-Brandt 2008 ice: supported vacuum wavelengths are 200..1100 nm; no extrapolation.");
    H::IceIndex v{};
    if (!H::ice_index_wb2008(wavelength_nm, v)) return fail(ICP_ERR_AUDIT, "Invalid ice optical state.");
    out->wavelength_nm = wavelength_nm;
    out->n = v.n;
    out->kappa = v.kappa;
    out->lower_nm = v.lower_nm;
    out->upper_nm = v.upper_nm;
    out->log_wavelength_fraction = v.fraction;
    return ok();
}

int icp_u_edges(uint32_t nt, double* out)
{
    if (!out || nt == 0) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_u_edges: theta_count must be positive");
    std::vector<double> e;
    if (!H::u_edges(nt, e)) return fail(ICP_ERR_INVALID_ARGUMENT, "Angular cells cannot be represented in binary64.");
    std::memcpy(out, e.data(), e.size() * sizeof(double));
    return ok();
}

} // extern "C"

namespace {

bool grid_valid(const icp_grid* g)
{
    if (!g || !g->nt || !g->np || (uint64_t)g->nt * g->np > 0xffffffffull) return false;
    const H::V k{g->ki[0], g->ki[1], g->ki[2]};
    const H::Frame f{{g->e0[0], g->e0[1], g->e0[2]}, {g->e1[0], g->e1[1], g->e1[2]}};
    return H::frame_valid(f, k);
}

struct NodeSetup {
    H::V k;
    H::Frame kf;
    H::FaceTable faces;
};

int node_setup(const icp_hex_node* n, const icp_grid* g, NodeSetup& s)
{
    if (!H::rotation_valid(n->rotation)) return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid orientation rotation.");
    const H::V gk{g->ki[0], g->ki[1], g->ki[2]};
    if (!H::normalize(H::rotate_inverse(n->rotation, gk), s.k) || !H::make_frame(s.k, s.kf))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Incident direction must be finite and nonzero.");
    const double R = n->circumradius_mm, L = n->length_mm;
    const double half = 0.5 * (L / R);
    if (!(H::finite(R) && H::finite(L) && R > 0 && L > 0 && H::finite(half) && half > 0 && R * R > 0 && R * L > 0))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid hex prism geometry.");
    s.faces = H::prism_faces(R, L, s.k);
    if (!(s.faces.area > 0) || !H::finite(s.faces.area)) return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid projected area.");
    return ICP_OK;
}

} // namespace

extern "C" int icp_hex_node_area(const icp_hex_node* node, const icp_grid* grid, double* area)
{
    if (!node || !grid || !area) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_hex_node_area: null argument");
    if (!grid_valid(grid)) return fail(ICP_ERR_INVALID_ARGUMENT, "Malformed phase grid.");
    NodeSetup s;
    if (const int r = node_setup(node, grid, s)) return r;
    *area = s.faces.area;
    return ok();
}

int icp::ensure_float_edges(icp_context* c, const double* d_edges, uint32_t nt)
{
    ICP_CUDA(c->edges_f.ensure(sizeof(float) * (nt + 1)));
    edges_to_float<<<(nt + 1 + 255) / 256, 256, 0, c->stream>>>(d_edges, (float*)c->edges_f.ptr, nt + 1);
    ++g_launches;
    ICP_CUDA(cudaGetLastError());
    return ICP_OK;
}

void icp::stats_accumulate(const unsigned char* raw, icp_trace_stats* out)
{
    // DevStats layout (icp_hex_kernel.cuh)
    struct Raw {
        unsigned long long esc[2], unres[2], fwd[2], bwd[2];
        double axial;
        unsigned long long max_bal_bits, max_iface_bits;
        unsigned long long rays, outputs, status[8], rejected, snapped, near_edge, fallback, invalid;
        unsigned long long encounters, missed, gauge_evals;
    } r;
    std::memcpy(&r, raw, sizeof r);
    auto fx = [](const unsigned long long* v) { return (std::ldexp((double)v[1], 64) + (double)v[0]) * 0x1p-44; };
    out->escaped += fx(r.esc);
    out->unresolved += fx(r.unres);
    out->forward_pole += fx(r.fwd);
    out->backward_pole += fx(r.bwd);
    out->point_axial += r.axial;
    double mb, mi;
    std::memcpy(&mb, &r.max_bal_bits, 8);
    std::memcpy(&mi, &r.max_iface_bits, 8);
    out->max_ray_balance = std::max(out->max_ray_balance, mb);
    out->max_interface_balance = std::max(out->max_interface_balance, mi);
    out->rays += r.rays;
    out->outputs += r.outputs;
    for (int i = 0; i < 8; ++i) out->status_counts[i] += r.status[i];
    out->rejected_rays += r.rejected;
    out->snapped += r.snapped;
    out->near_edge += r.near_edge;
    out->fallback_adds += r.fallback;
    out->invalid += r.invalid;
    out->encounters += r.encounters;
    out->missed += r.missed;
    out->gauge_evals += r.gauge_evals;
}

namespace {

__global__ void max_u32(const uint32_t* v, uint64_t n, unsigned long long* out)
{
    unsigned long long m = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        m = v[i] > m ? v[i] : m;
    for (int o = 16; o; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, m, o);
        m = t > m ? t : m;
    }
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

} // namespace

extern "C" int icp_hex_trace_bin(icp_context* c, const icp_hex_node* n, const icp_grid* g, const double* d_edges,
                                 double* d_mass, icp_trace_stats* stats, uint32_t* d_batch_out, const icp_tuning* tune)
{
    if (!c || !n || !g || !d_edges || !d_mass || !stats) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_hex_trace_bin: null argument");
    if (!grid_valid(g)) return fail(ICP_ERR_INVALID_ARGUMENT, "Malformed phase grid.");
    NodeSetup s;
    if (const int r = node_setup(n, g, s)) return r;
    if (!(n->exterior_index > 0 && n->interior_index > 0 && H::finite(n->exterior_index) && H::finite(n->interior_index)))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid refractive indices.");
    if (!(H::finite(n->tail_tolerance) && n->tail_tolerance >= 0 && n->tail_tolerance < 1))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid tail tolerance.");
    if (!n->total_samples || !n->max_internal_hits || !n->batch_size)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Sample count, hit limit and batch size must be positive.");
    if (n->sample_count == 0) return ok();
    if (n->first_sample >= n->total_samples || n->sample_count > n->total_samples - n->first_sample)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Batch is outside the global incident-sample range.");
    if (!(n->area_weight > 0) || !H::finite(n->area_weight))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid orientation / area weight.");
    if (n->precision != ICP_FP32 && n->precision != ICP_FP64) return fail(ICP_ERR_INVALID_ARGUMENT, "Unknown precision.");
    ICP_CUDA(cudaSetDevice(c->device));

    uint32_t threads = tune && tune->block_threads ? tune->block_threads : 256u;
    if (threads < 64 || threads > 256 || threads % 32) return fail(ICP_ERR_INVALID_ARGUMENT, "block_threads must be 64..256, multiple of 32");
    uint32_t slots = 4096u;
    if (tune && tune->hash_slots) slots = tune->hash_slots == 1 ? 0u : tune->hash_slots;
    if (slots & (slots - 1)) return fail(ICP_ERR_INVALID_ARGUMENT, "hash_slots must be a power of two");
    const bool f32 = n->precision == ICP_FP32;
    int per_sm = f32 ? hex_blocks_per_sm_f32(slots, g->nt, threads) : hex_blocks_per_sm_f64(slots, g->nt, threads);
    if (per_sm <= 0) return fail(ICP_ERR_DEVICE, "hex trace kernel cannot be resident with %u threads / %u slots", threads, slots);
    if (tune && tune->blocks_per_sm) per_sm = std::min<int>(per_sm, (int)tune->blocks_per_sm);
    const uint32_t warps_per_block = threads / 32;
    // at least 64 rays per warp when the range is small; at most 2^16 per warp per launch
    uint64_t blocks = (uint64_t)per_sm * c->sms;
    blocks = std::max<uint64_t>(1, std::min<uint64_t>(blocks, (n->sample_count + 64ull * warps_per_block - 1) / (64ull * warps_per_block)));
    const uint64_t piece = blocks * warps_per_block * lane_rays_max(n->max_internal_hits);

    ICP_CUDA(c->stats.ensure(hex_stats_bytes()));
    ICP_CUDA(cudaMemsetAsync(c->stats.ptr, 0, hex_stats_bytes(), c->stream));
    if (f32)
        if (const int r = ensure_float_edges(c, d_edges, g->nt)) return r;

    HexLaunch L{};
    L.half_len = 0.5 * (n->length_mm / n->circumradius_mm);
    L.k[0] = s.k.x; L.k[1] = s.k.y; L.k[2] = s.k.z;
    L.ke0[0] = s.kf.e0.x; L.ke0[1] = s.kf.e0.y; L.ke0[2] = s.kf.e0.z;
    for (int f = 0; f < 8; ++f) L.cum[f] = s.faces.cum[f];
    L.face_mask = s.faces.mask;
    L.area = s.faces.area;
    L.n_ext = n->exterior_index;
    L.n_int = n->interior_index;
    L.tail = n->tail_tolerance;
    L.bal_tol = n->balance_tolerance;
    L.seed = n->seed;
    L.total = n->total_samples;
    L.max_hits = n->max_internal_hits;
    L.batch_size = n->batch_size;
    L.batch_out = d_batch_out;
    std::memcpy(L.rot, n->rotation, sizeof L.rot);
    std::memcpy(L.ki, g->ki, sizeof L.ki);
    std::memcpy(L.e0, g->e0, sizeof L.e0);
    std::memcpy(L.e1g, g->e1, sizeof L.e1g);
    L.nt = g->nt;
    L.np = g->np;
    L.edges_d = d_edges;
    L.edges_f = (const float*)c->edges_f.ptr;
    L.mass = d_mass;
    L.to_mass = n->area_weight * 0x1p-44;
    L.stats = c->stats.ptr;
    L.hash_slots = slots;
    L.block_threads = threads;
    L.blocks = (uint32_t)blocks;
    for (uint64_t off = 0; off < n->sample_count; off += piece) {
        L.first = n->first_sample + off;
        L.count = std::min<uint64_t>(piece, n->sample_count - off);
        const int e = f32 ? launch_hex_f32(L, c->stream) : launch_hex_f64(L, c->stream);
        ++g_launches;
        if (e) return fail(ICP_ERR_DEVICE, "hex trace launch failed: %s", cudaGetErrorString((cudaError_t)e));
    }
    std::vector<unsigned char> raw(hex_stats_bytes());
    ICP_CUDA(cudaMemcpyAsync(raw.data(), c->stats.ptr, raw.size(), cudaMemcpyDeviceToHost, c->stream));
    ICP_CUDA(cudaStreamSynchronize(c->stream));
    stats_accumulate(raw.data(), stats);
    return ok();
}

namespace {

int cdf_launch_common(icp_context* c, CdfLaunch& L, uint32_t ct, uint32_t cp)
{
    const bool tma_ok = L.nt == ct && L.np == cp && L.np % 2 == 0 && ((uintptr_t)L.values % 16) == 0;
    CdfShape sh{};
    if (const int r = icp::cdf_shape(c, L.nt, L.np, ct, cp, tma_ok, sh)) return r;
    const uint32_t blocks = (cp + sh.cw - 1) / sh.cw;
    ICP_CUDA(c->cdf_partial.ensure(cdf_partial_bytes() * blocks));
    ICP_CUDA(c->cdf_colsum.ensure(sizeof(double) * cp));
    L.colsum = (double*)c->cdf_colsum.ptr;
    L.partial = c->cdf_partial.ptr;
    L.spin_limit = c->wait_limit;
    const int e = launch_cdf_build(L, sh, c->stream);
    ++g_launches;
    if (e) return fail(ICP_ERR_DEVICE, "CDF launch failed: %s", cudaGetErrorString((cudaError_t)e));
    return ICP_OK;
}

// Density input (kind 1) with host pole additions: the public entry's path.
int cdf_enqueue_kind(icp_context* c, const double* d_values, uint32_t kind, uint32_t nt, uint32_t np, uint32_t ct,
                     uint32_t cp, const double* d_edges, double fa, double ba, double* d_phi, double* d_theta)
{
    CdfLaunch L{};
    L.values = d_values;
    L.edges = d_edges;
    L.phi = d_phi;
    L.theta = d_theta;
    L.report = (CdfDeviceReport*)c->cdf_report.ptr;
    L.sync = (unsigned*)c->cdf_sync.ptr;
    L.kind = kind;
    L.nt = nt; L.np = np; L.ct = ct; L.cp = cp;
    L.fwd_add = fa;
    L.bwd_add = ba;
    return cdf_launch_common(c, L, ct, cp);
}

// Arguments of icp_phase_cdf_enqueue / icp_phase_cdf_build (the reference's PhaseCdf::build
// input checks, src/phase_cdf.cpp:285-310, and the host's pole split).
int cdf_check_args(const icp_context* c, const double* d_values, uint32_t kind, uint32_t nt, uint32_t np, double fwd,
                   double bwd, uint32_t ct, uint32_t cp, const double* d_phi, const double* d_theta, double& fa,
                   double& ba)
{
    if (!c || !d_values || !d_phi || !d_theta) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_phase_cdf_build: null argument");
    if (kind > 1) return fail(ICP_ERR_INVALID_ARGUMENT, "Unknown CDF input kind.");
    if (!nt || !np || (uint64_t)nt * np > 0xffffffffull)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Unsupported phase grid dimensions.");
    if (!ct || !cp || ct > nt || cp > np || nt % ct || np % cp)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Storage dimensions must divide histogram dimensions.");
    if (!(fwd >= 0) || !(bwd >= 0) || !H::finite(fwd) || !H::finite(bwd))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid pole masses.");
    fa = fwd / np;
    ba = bwd / np;
    if ((fwd > 0 && !(fa > 0)) || (bwd > 0 && !(ba > 0))) return fail(ICP_ERR_AUDIT, "Pole weight underflow.");
    return ICP_OK;
}

bool policy_ok(const icp_cdf_policy& p)
{
    return H::finite(p.max_l1_error) && p.max_l1_error >= 0 && p.max_l1_error <= 2 && H::finite(p.max_lost_mass) &&
           p.max_lost_mass >= 0 && p.max_lost_mass <= 1 && H::finite(p.max_coarsening_tv) &&
           p.max_coarsening_tv >= 0 && p.max_coarsening_tv <= 1;
}

} // namespace

int icp::cdf_clear(icp_context* c, void* d_reports, void* d_sync, uint32_t records)
{
    ICP_CUDA(cudaMemsetAsync(d_sync, 0, 2 * sizeof(unsigned) * records, c->stream));
    ICP_CUDA(cudaMemsetAsync(d_reports, 0, sizeof(CdfDeviceReport) * records, c->stream));
    ICP_CUDA(cudaStreamSynchronize(c->stream));
    return ICP_OK;
}

int icp::cdf_enqueue(icp_context* c, const double* d_values, uint32_t nt, uint32_t np, uint32_t ct, uint32_t cp,
                     const double* d_edges, double fwd_add, double bwd_add, const unsigned long long* pole_fx,
                     double pole_weight, const double* row_add, double* d_phi, double* d_theta,
                     CdfDeviceReport* d_report, unsigned* d_sync)
{
    CdfLaunch L{};
    L.values = d_values;
    L.edges = d_edges;
    L.phi = d_phi;
    L.theta = d_theta;
    L.report = d_report;
    L.sync = d_sync;
    L.kind = 0;
    L.nt = nt; L.np = np; L.ct = ct; L.cp = cp;
    L.fwd_add = fwd_add;
    L.bwd_add = bwd_add;
    L.pole_fx = pole_fx;
    L.pole_weight = pole_weight;
    L.row_add = row_add;
    return cdf_launch_common(c, L, ct, cp);
}

int icp::cdf_enqueue_batch(icp_context* c, const CdfBatchInput* in, uint32_t count, uint32_t nt, uint32_t np,
                           uint32_t ct, uint32_t cp, const double* d_edges, CdfDeviceReport* d_reports, unsigned* d_sync)
{
    if (!count) return ICP_OK;
    ICP_CUDA(cudaMemsetAsync(d_sync, 0, 2 * sizeof(unsigned) * count, c->stream));
    ICP_CUDA(cudaMemsetAsync(d_reports, 0, sizeof(CdfDeviceReport) * count, c->stream));
    // 2 strips per record, as many records per launch as stay co-resident (the chains of a
    // strip's columns run side by side, so wider strips cost little and let more records share
    // one launch)
    CdfShape sh{};
    const bool fits = cdf_choose_shape(c->device, c->sms, nt, np, ct, cp, false, std::max(1u, (cp + 1u) / 2u),
                                       0xffffffffu, sh) == 0;
    const uint32_t strips = fits ? (cp + sh.cw - 1) / sh.cw : 0u;
    const uint32_t per = fits ? (uint32_t)std::max(0, cdf_max_coresident_blocks(sh.smem, c->device)) / strips : 0u;
    if (!per) {
        // a record's strips alone do not fit: one launch per record, with its own strip width
        for (uint32_t r = 0; r < count; ++r)
            if (const int e = cdf_enqueue(c, in[r].values, nt, np, ct, cp, d_edges, in[r].fwd_add, in[r].bwd_add,
                                          in[r].pole_fx, in[r].pole_weight, in[r].row_add, in[r].phi, in[r].theta,
                                          d_reports + r, d_sync + 2 * r))
                return e;
        return ICP_OK;
    }
    const size_t pb = cdf_partial_bytes() * strips;
    ICP_CUDA(c->cdfb_partial.ensure(pb * count));
    ICP_CUDA(c->cdfb_colsum.ensure(sizeof(double) * cp * count));
    ICP_CUDA(c->cdfb_recs.ensure(sizeof(CdfBatchRecord) * count));
    std::vector<CdfBatchRecord> recs(count);
    for (uint32_t r = 0; r < count; ++r) {
        CdfBatchRecord& b = recs[r];
        b.values = in[r].values;
        b.phi = in[r].phi;
        b.theta = in[r].theta;
        b.colsum = (double*)c->cdfb_colsum.ptr + (size_t)cp * r;
        b.partial = (unsigned char*)c->cdfb_partial.ptr + pb * r;
        b.report = d_reports + r;
        b.sync = d_sync + 2 * r;
        b.row_add = in[r].row_add;
        b.pole_fx = in[r].pole_fx;
        b.pole_weight = in[r].pole_weight;
        b.fwd_add = in[r].fwd_add;
        b.bwd_add = in[r].bwd_add;
    }
    ICP_CUDA(cudaMemcpyAsync(c->cdfb_recs.ptr, recs.data(), sizeof(CdfBatchRecord) * count, cudaMemcpyHostToDevice,
                             c->stream));
    CdfLaunch L{};
    L.edges = d_edges;
    L.kind = 0;
    L.nt = nt;
    L.np = np;
    L.ct = ct;
    L.cp = cp;
    L.spin_limit = c->wait_limit;
    for (uint32_t r0 = 0; r0 < count; r0 += per) {
        const uint32_t n = std::min(per, count - r0);
        const int e = launch_cdf_build_batch(L, sh, (const CdfBatchRecord*)c->cdfb_recs.ptr + r0, n, c->stream);
        ++g_launches;
        if (e) return fail(ICP_ERR_DEVICE, "batched CDF launch failed: %s", cudaGetErrorString((cudaError_t)e));
    }
    return ICP_OK;
}

int icp::cdf_shape(icp_context* c, uint32_t nt, uint32_t np, uint32_t ct, uint32_t cp, bool tma_ok, CdfShape& s)
{
    for (const auto& k : c->cdf_shapes)
        if (k.nt == nt && k.np == np && k.ct == ct && k.cp == cp && k.tma_ok == (uint32_t)tma_ok) {
            s = k.shape;
            return ICP_OK;
        }
    if (cdf_choose_shape(c->device, c->sms, nt, np, ct, cp, tma_ok, 1u, 0xffffffffu, s))
        return fail(ICP_ERR_CAPACITY, "CDF strip for %u theta rows does not fit shared memory with a co-resident grid", ct);
    c->cdf_shapes.push_back({nt, np, ct, cp, (uint32_t)tma_ok, s});
    return ICP_OK;
}

extern "C" int icp_phase_cdf_enqueue(icp_context* c, const double* d_values, uint32_t kind, uint32_t nt, uint32_t np,
                                     double fwd, double bwd, uint32_t ct, uint32_t cp, double* d_phi, double* d_theta)
{
    double fa = 0, ba = 0;
    if (const int e = cdf_check_args(c, d_values, kind, nt, np, fwd, bwd, ct, cp, d_phi, d_theta, fa, ba)) return e;
    ICP_CUDA(cudaSetDevice(c->device));
    if (c->cdf_edges_nt != nt) {
        std::vector<double> edges;
        if (!H::u_edges(nt, edges))
            return fail(ICP_ERR_INVALID_ARGUMENT, "Angular cells cannot be represented in binary64.");
        ICP_CUDA(c->cdf_edges.ensure(sizeof(double) * (nt + 1)));
        ICP_CUDA(cudaMemcpyAsync(c->cdf_edges.ptr, edges.data(), sizeof(double) * (nt + 1), cudaMemcpyHostToDevice,
                                 c->stream));
        ICP_CUDA(cudaStreamSynchronize(c->stream)); // the host vector goes out of scope
        c->cdf_edges_nt = nt;
    }
    ICP_CUDA(c->cdf_report.ensure_zeroed(sizeof(CdfDeviceReport), c->stream));
    ICP_CUDA(c->cdf_sync.ensure_zeroed(2 * sizeof(unsigned), c->stream));
    const double* d_edges = (const double*)c->cdf_edges.ptr;
    if (kind == 1) {
        // density input: the kernel's mass conversion (kind 1) is only reached through here
        if (const int e = cdf_enqueue_kind(c, d_values, kind, nt, np, ct, cp, d_edges, fa, ba, d_phi, d_theta)) return e;
    } else if (const int e = cdf_enqueue(c, d_values, nt, np, ct, cp, d_edges, fa, ba, nullptr, 0.0, nullptr, d_phi,
                                         d_theta, (CdfDeviceReport*)c->cdf_report.ptr, (unsigned*)c->cdf_sync.ptr))
        return e;
    return ok();
}

extern "C" int icp_phase_cdf_result(icp_context* c, const icp_cdf_policy* policy, icp_cdf_report* report)
{
    if (!c || !policy || !report) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_phase_cdf_result: null argument");
    std::memset(report, 0, sizeof *report);
    if (!policy_ok(*policy)) return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid CDF quality policy.");
    if (!c->cdf_report.ptr) return fail(ICP_ERR_STATE, "icp_phase_cdf_result: no CDF build was enqueued");
    ICP_CUDA(cudaSetDevice(c->device));
    CdfDeviceReport r{};
    ICP_CUDA(cudaMemcpyAsync(&r, c->cdf_report.ptr, sizeof r, cudaMemcpyDeviceToHost, c->stream));
    ICP_CUDA(cudaStreamSynchronize(c->stream));
    if (r.timeout)
        if (const int e = cdf_clear(c, c->cdf_report.ptr, c->cdf_sync.ptr, 1)) return e;
    return icp::cdf_finish(r, *policy, report);
}

extern "C" int icp_phase_cdf_build(icp_context* c, const double* d_values, uint32_t kind, uint32_t nt, uint32_t np,
                                   double fwd, double bwd, uint32_t ct, uint32_t cp, const icp_cdf_policy* policy,
                                   double* d_phi, double* d_theta, icp_cdf_report* report)
{
    if (!c || !d_values || !d_phi || !d_theta || !report || !policy)
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_phase_cdf_build: null argument");
    std::memset(report, 0, sizeof *report);
    if (!policy_ok(*policy)) return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid CDF quality policy.");
    if (const int e = icp_phase_cdf_enqueue(c, d_values, kind, nt, np, fwd, bwd, ct, cp, d_phi, d_theta)) return e;
    return icp_phase_cdf_result(c, policy, report);
}

extern "C" int icp_phase_cdf_build_batch(icp_context* c, const double* d_values, uint32_t count, uint32_t nt,
                                         uint32_t np, uint32_t ct, uint32_t cp, const icp_cdf_policy* policy,
                                         double* d_phi, double* d_theta, icp_cdf_report* reports)
{
    if (!c || !d_values || !d_phi || !d_theta || !reports || !policy)
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_phase_cdf_build_batch: null argument");
    if (!count) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_phase_cdf_build_batch: no records");
    const icp_cdf_policy& p = *policy;
    if (!policy_ok(p)) return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid CDF quality policy.");
    if (!nt || !np || (uint64_t)nt * np > 0xffffffffull)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Unsupported phase grid dimensions.");
    if (!ct || !cp || ct > nt || cp > np || nt % ct || np % cp)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Storage dimensions must divide histogram dimensions.");
    ICP_CUDA(cudaSetDevice(c->device));
    std::vector<double> edges;
    if (!H::u_edges(nt, edges)) return fail(ICP_ERR_INVALID_ARGUMENT, "Angular cells cannot be represented in binary64.");
    ICP_CUDA(c->rec_edges.ensure(sizeof(double) * (nt + 1)));
    ICP_CUDA(c->b_reports.ensure(sizeof(CdfDeviceReport) * count));
    ICP_CUDA(c->b_sync.ensure(2 * sizeof(unsigned) * count));
    ICP_CUDA(cudaMemcpyAsync(c->rec_edges.ptr, edges.data(), sizeof(double) * (nt + 1), cudaMemcpyHostToDevice, c->stream));
    std::vector<CdfBatchInput> in(count);
    for (uint32_t r = 0; r < count; ++r) {
        in[r] = CdfBatchInput{};
        in[r].values = d_values + (size_t)nt * np * r;
        in[r].phi = d_phi + (size_t)(cp + 1) * r;
        in[r].theta = d_theta + (size_t)cp * (ct + 1) * r;
    }
    if (const int e = cdf_enqueue_batch(c, in.data(), count, nt, np, ct, cp, (const double*)c->rec_edges.ptr,
                                        (CdfDeviceReport*)c->b_reports.ptr, (unsigned*)c->b_sync.ptr))
        return e;
    std::vector<CdfDeviceReport> dev(count);
    ICP_CUDA(cudaMemcpyAsync(dev.data(), c->b_reports.ptr, sizeof(CdfDeviceReport) * count, cudaMemcpyDeviceToHost,
                             c->stream));
    ICP_CUDA(cudaStreamSynchronize(c->stream));
    int first = ICP_OK;
    for (uint32_t r = 0; r < count; ++r) {
        std::memset(&reports[r], 0, sizeof reports[r]);
        const int e = icp::cdf_finish(dev[r], p, &reports[r]);
        reports[r].status = (uint32_t)e;
        if (e && !first) first = e;
    }
    if (first) return first;
    return ok();
}

int icp::cdf_finish(const CdfDeviceReport& r, const icp_cdf_policy& p, icp_cdf_report* report)
{
    if (r.timeout) return fail(ICP_ERR_TIMEOUT, "CDF grid barrier gave up waiting (co-residency violated?)");
    report->fine_mass = r.fine_mass;
    report->fine_axial = r.fine_axial;
    report->g_source = r.fine_axial / r.fine_mass;
    report->aggregation_relative_error = std::fabs(r.stored_mass / r.fine_mass - 1);
    report->coarsening_tv = r.tv;
    report->l1_error = r.l1;
    report->lost_mass = r.lost;
    report->maximum_cell_error = r.max_err;
    report->cdf_mass = r.recovered;
    report->g_stored = r.axial / r.recovered;
    report->lost_cells = r.lost_cells;
    report->malformed = r.malformed;
    // quality gates of build_host_cdf (hex_phase/src/phase_table.cpp:114-185)
    int status = ICP_OK;
    if (r.invalid) status = fail(ICP_ERR_INVALID_ARGUMENT, "Negative/nonfinite mass.");
    else if (!(r.fine_mass > 0) || !H::finite(r.fine_mass) || !H::finite(r.fine_axial))
        status = fail(ICP_ERR_AUDIT, "Empty/nonfinite histogram.");
    else if (!H::finite(report->coarsening_tv) || report->coarsening_tv > p.max_coarsening_tv ||
             report->aggregation_relative_error > 1e-12)
        status = fail(ICP_ERR_AUDIT, "Conservative coarsening audit failed.");
    else if (r.underflow) status = fail(ICP_ERR_AUDIT, "CDF weight underflow.");
    else if (!(r.total > 0) || !H::finite(r.total)) status = fail(ICP_ERR_AUDIT, "Invalid CDF total.");
    else if (r.malformed) status = fail(ICP_ERR_AUDIT, "Malformed CDF; refusing repair.");
    else if (report->l1_error > p.max_l1_error || report->lost_mass > p.max_lost_mass ||
             std::fabs(report->cdf_mass - 1) > 1e-10 || !H::finite(report->g_stored) ||
             !(report->g_stored > -1 && report->g_stored < 1))
        status = fail(ICP_ERR_AUDIT, "CDF mass / HG audit failed.");
    report->status = (uint32_t)status;
    return status == ICP_OK ? ok() : status;
}

extern "C" int icp_hex_generate(icp_context* c, const icp_hex_record* rec, const icp_orientation* nodes, uint32_t count,
                                double* h_phi, double* h_theta, double* h_u, icp_record_report* report)
{
    if (!c || !rec || !nodes || !count || !h_phi || !h_theta || !h_u || !report)
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_hex_generate: null argument");
    std::memset(report, 0, sizeof *report);
    ICP_CUDA(cudaSetDevice(c->device));
    // grid (make_phase_grid, hex_phase/src/phase_table.cpp:22-29)
    icp_grid g{};
    g.nt = rec->nt;
    g.np = rec->np;
    H::V k;
    H::Frame kf;
    if (!rec->nt || !rec->np || (uint64_t)rec->nt * rec->np > 0xffffffffull || rec->nt > 32u * 65535u || rec->np > 0x7fffffffu)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Unsupported phase grid dimensions.");
    if (!H::normalize({rec->ki[0], rec->ki[1], rec->ki[2]}, k) || !H::make_frame(k, kf))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid incident direction.");
    g.ki[0] = k.x; g.ki[1] = k.y; g.ki[2] = k.z;
    g.e0[0] = kf.e0.x; g.e0[1] = kf.e0.y; g.e0[2] = kf.e0.z;
    g.e1[0] = kf.e1.x; g.e1[1] = kf.e1.y; g.e1[2] = kf.e1.z;
    std::vector<double> edges;
    if (!H::u_edges(rec->nt, edges)) return fail(ICP_ERR_INVALID_ARGUMENT, "Angular cells cannot be represented in binary64.");
    const uint64_t cells = (uint64_t)rec->nt * rec->np;
    ICP_CUDA(c->rec_edges.ensure(sizeof(double) * (rec->nt + 1)));
    ICP_CUDA(c->rec_mass.ensure(sizeof(double) * cells));
    ICP_CUDA(c->rec_phi.ensure(sizeof(double) * (rec->cp + 1)));
    ICP_CUDA(c->rec_theta.ensure(sizeof(double) * (size_t)rec->cp * (rec->ct + 1)));
    ICP_CUDA(cudaMemcpyAsync(c->rec_edges.ptr, edges.data(), sizeof(double) * (rec->nt + 1), cudaMemcpyHostToDevice, c->stream));
    ICP_CUDA(cudaMemsetAsync(c->rec_mass.ptr, 0, sizeof(double) * cells, c->stream));
    // preflight all nodes (generate_hex_phase.cpp:82-88)
    std::vector<icp_hex_node> hn(count);
    H::KahanSum expected;
    uint64_t max_batches = 0;
    for (uint32_t i = 0; i < count; ++i) {
        icp_hex_node& n = hn[i];
        std::memset(&n, 0, sizeof n);
        const icp_orientation& o = nodes[i];
        if (!H::rotation(o.quaternion[0], o.quaternion[1], o.quaternion[2], o.quaternion[3], n.rotation))
            return fail(ICP_ERR_INVALID_ARGUMENT, "Quaternion must be unit length (w,x,y,z).");
        if (!H::finite(o.weight) || !(o.weight > 0) || !o.samples)
            return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid orientation node.");
        n.circumradius_mm = rec->circumradius_mm;
        n.length_mm = rec->length_mm;
        n.exterior_index = rec->exterior_index;
        n.interior_index = rec->interior_index;
        n.tail_tolerance = rec->tail_tolerance;
        n.balance_tolerance = rec->balance_tolerance;
        n.seed = o.seed;
        n.total_samples = o.samples;
        n.first_sample = 0;
        n.sample_count = o.samples;
        n.max_internal_hits = rec->max_internal_hits;
        n.batch_size = rec->batch_size ? rec->batch_size : 4096u;
        n.precision = rec->precision;
        double area = 0;
        if (const int r = icp_hex_node_area(&n, &g, &area)) return r;
        const double weight = o.weight * area;
        if (!(weight > 0) || !H::finite(weight) || !(weight / double(o.samples) > 0))
            return fail(ICP_ERR_INVALID_ARGUMENT, "Orientation area weight over/underflow.");
        expected.add(weight);
        n.area_weight = o.weight * area / double(o.samples);
        max_batches = std::max<uint64_t>(max_batches, (o.samples + n.batch_size - 1) / n.batch_size);
    }
    report->expected_area_mm2 = expected.value;
    uint32_t* d_batch = nullptr;
    unsigned long long* d_max = nullptr;
    if (rec->max_output_records) {
        ICP_CUDA(c->rec_batch.ensure(sizeof(uint32_t) * max_batches + 64));
        d_batch = (uint32_t*)c->rec_batch.ptr;
        d_max = (unsigned long long*)((char*)c->rec_batch.ptr + ((sizeof(uint32_t) * max_batches + 7) / 8) * 8);
    }
    ICP_CUDA(cudaEventRecord(c->ev0, c->stream));
    H::KahanSum escaped, unresolved;
    icp_trace_stats& T = report->trace;
    uint64_t max_batch_out = 0;
    for (uint32_t i = 0; i < count; ++i) {
        icp_trace_stats s{};
        if (d_batch) ICP_CUDA(cudaMemsetAsync(d_batch, 0, sizeof(uint32_t) * max_batches + 8, c->stream));
        if (const int r = icp_hex_trace_bin(c, &hn[i], &g, (const double*)c->rec_edges.ptr, (double*)c->rec_mass.ptr, &s,
                                            d_batch, &rec->tuning))
            return r;
        if (d_batch) {
            const uint64_t nb = (hn[i].total_samples + hn[i].batch_size - 1) / hn[i].batch_size;
            max_u32<<<std::max<uint64_t>(1, std::min<uint64_t>(1024, (nb + 255) / 256)), 256, 0, c->stream>>>(d_batch, nb, d_max);
            ++g_launches;
            unsigned long long m = 0;
            ICP_CUDA(cudaMemcpyAsync(&m, d_max, 8, cudaMemcpyDeviceToHost, c->stream));
            ICP_CUDA(cudaStreamSynchronize(c->stream));
            max_batch_out = std::max<uint64_t>(max_batch_out, m);
        }
        const double w = hn[i].area_weight;
        escaped.add(w * s.escaped);
        unresolved.add(w * s.unresolved);
        report->point_axial_mm2 += w * s.point_axial;
        report->forward_mass_mm2 += w * s.forward_pole;
        report->backward_mass_mm2 += w * s.backward_pole;
        T.escaped += s.escaped;
        T.unresolved += s.unresolved;
        T.point_axial += s.point_axial;
        T.forward_pole += s.forward_pole;
        T.backward_pole += s.backward_pole;
        T.max_ray_balance = std::max(T.max_ray_balance, s.max_ray_balance);
        T.max_interface_balance = std::max(T.max_interface_balance, s.max_interface_balance);
        T.rays += s.rays;
        T.outputs += s.outputs;
        for (int q = 0; q < 8; ++q) T.status_counts[q] += s.status_counts[q];
        T.rejected_rays += s.rejected_rays;
        T.snapped += s.snapped;
        T.near_edge += s.near_edge;
        T.fallback_adds += s.fallback_adds;
        T.invalid += s.invalid;
        T.encounters += s.encounters;
    }
    T.max_batch_outputs = max_batch_out;
    ICP_CUDA(cudaEventRecord(c->ev1, c->stream));
    report->escaped_area_mm2 = escaped.value;
    report->unresolved_area_mm2 = unresolved.value;
    report->point_mass_mm2 = escaped.value;
    ICP_CUDA(cudaEventSynchronize(c->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    report->seconds_trace = ms * 1e-3;
    if (rec->max_output_records && max_batch_out > rec->max_output_records)
        return fail(ICP_ERR_CAPACITY, "Output memory budget exceeded; batch not silently reduced.");
    ICP_CUDA(cudaEventRecord(c->ev0, c->stream));
    const int cr = icp_phase_cdf_build(c, (const double*)c->rec_mass.ptr, ICP_CDF_MASS, rec->nt, rec->np,
                                       report->forward_mass_mm2, report->backward_mass_mm2, rec->ct, rec->cp, &rec->policy,
                                       (double*)c->rec_phi.ptr, (double*)c->rec_theta.ptr, &report->cdf);
    ICP_CUDA(cudaEventRecord(c->ev1, c->stream));
    report->histogram_mass_mm2 = report->cdf.fine_mass;
    report->histogram_axial_mm2 = report->cdf.fine_axial;
    if (cr != ICP_OK) return cr;
    ICP_CUDA(cudaMemcpyAsync(h_phi, c->rec_phi.ptr, sizeof(double) * (rec->cp + 1), cudaMemcpyDeviceToHost, c->stream));
    ICP_CUDA(cudaMemcpyAsync(h_theta, c->rec_theta.ptr, sizeof(double) * (size_t)rec->cp * (rec->ct + 1),
                             cudaMemcpyDeviceToHost, c->stream));
    ICP_CUDA(cudaStreamSynchronize(c->stream));
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    report->seconds_cdf = ms * 1e-3;
    const uint32_t dt = rec->nt / rec->ct;
    for (uint32_t i = 0; i <= rec->ct; ++i) h_u[i] = edges[(size_t)i * dt];
    const double esc = report->escaped_area_mm2;
    report->histogram_relative_error =
        std::max(std::fabs(report->histogram_mass_mm2 / esc - 1), std::fabs(report->point_mass_mm2 / esc - 1));
    return ok();
}
