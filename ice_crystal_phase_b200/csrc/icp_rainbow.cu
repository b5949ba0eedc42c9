// icp_rainbow.cu -- Table-II rainbow diffraction on the query grid (sm_100a) and its C ABI
// (include/icp_b200.h, "Table-II rainbow diffraction").  Built with -fmad=false: every
// binary64 product and sum rounds on its own, and the explicit fma calls stay fused, as in
// the reference's host build of include/rainbow/rainbow_diffraction.hpp.
//
// The model (RainbowDiffraction, rainbow_diffraction.hpp:40-139): an edge between query
// rows r and r + 1 at one phi is a primary transition when the TRT family starts there and
// a secondary one when the TRRT family ends there, provided the total intensity jumps by
// the contrast; every direction within support x sigma of its nearest labelled edge is
// replaced by a solid-angle weighted spherical Gaussian of its neighbourhood (secondary
// sigma = 2 x primary), blended out between inner_blend and support sigmas.
//
// Three kernels, one thread per query direction, grid-stride over the SMs:
//   rainbow_detect_kernel  edge labels; also packs each sample to (s, p) -- NaN when the
//                          sample is unavailable -- and marks the rows that carry a label,
//                          so the filter reads 16 bytes per neighbour instead of the
//                          144-byte focal record and skips unlabelled rows of its search
//                          in one load each.  Label counters by warp-aggregated atomics.
//   rainbow_prepare_kernel the packing and row marks for caller-supplied labels.
//   rainbow_filter_kernel  the nearest-edge search (rows without a label skipped: they
//                          cannot change the result) and the Gaussian over the cap, with
//                          the reference's compensated sums in its row / column order; per
//                          row the distance terms that do not depend on phi are hoisted.
//                          Writes the result, optionally the stage density s + p, and the
//                          result counters.
// Device libm (sin, asin, acos, exp, sqrt) is CUDA's; its last-ulp differences from the
// host's are the only source of difference from the reference's host results.
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "../../include/icp_b200.h"
#include "icp_internal.h"

using namespace icp;

namespace {

thread_local char g_msg[512];

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

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kCapSlack = 0x1p-44; // closed-cap cutoff slack (rainbow_diffraction.hpp:14)
constexpr unsigned kThreads = 256;
constexpr uint32_t kMaxAxis = 32767u;

enum Counter { kPrimary, kSecondary, kUnknown, kFiltered, kUnavailable, kUnderresolved, kCounters };
constexpr uint32_t kUnavailableMask = ICP_DIFFRACTION_INPUT_UNAVAILABLE | ICP_DIFFRACTION_STENCIL_UNAVAILABLE |
                                      ICP_DIFFRACTION_DETECTION_UNAVAILABLE | ICP_DIFFRACTION_INVALID_DATA;

struct Grid {
    double sigma, support, contrast, inner;
    uint32_t nt, np;
};

bool config_ok(uint32_t nt, uint32_t np, const icp_diffraction_config& c)
{
    auto fin = [](double x) { return x >= -DBL_MAX && x <= DBL_MAX; };
    return nt >= 2u && np >= 1u && nt <= kMaxAxis && np <= kMaxAxis && c.primary_sigma_rad > 0 &&
           fin(c.primary_sigma_rad) && c.support_sigma >= 2 && c.support_sigma <= 8 && c.inner_blend_sigma >= 0 &&
           c.inner_blend_sigma < c.support_sigma && 2 * c.primary_sigma_rad * c.support_sigma < kPi &&
           c.transition_contrast >= 0 && c.transition_contrast < 1;
}

__device__ __forceinline__ bool finite64(double x) { return x >= -DBL_MAX && x <= DBL_MAX; }
__device__ __forceinline__ double nan64() { return __longlong_as_double(0x7ff8000000000000ll); }

// (s, p) of a focal record, or NaN when the record is unavailable (flags, sign, finiteness).
__device__ __forceinline__ double2 load_sample(const icp_focal_sample* f, uint64_t i)
{
    const double s = __ldg(&f[i].intensity_s), p = __ldg(&f[i].intensity_p);
    const bool good = __ldg(&f[i].flags) == 0u && s >= 0 && p >= 0 && finite64(s + p);
    return good ? make_double2(s, p) : make_double2(nan64(), nan64());
}
__device__ __forceinline__ bool available(double2 v) { return v.x == v.x; }

__device__ __forceinline__ void warp_count(uint32_t* counters, int which, bool pred)
{
    const unsigned mask = __ballot_sync(0xffffffffu, pred);
    if ((threadIdx.x & 31u) == 0 && mask) atomicAdd(&counters[which], (unsigned)__popc(mask));
}

__global__ void __launch_bounds__(kThreads) rainbow_detect_kernel(const icp_focal_sample* __restrict__ f, Grid g,
                                                                  uint32_t* __restrict__ edges,
                                                                  double2* __restrict__ packed,
                                                                  uint32_t* __restrict__ row_marks,
                                                                  uint32_t* __restrict__ counters)
{
    const uint64_t n = uint64_t(g.nt) * g.np, stride = uint64_t(gridDim.x) * blockDim.x;
    // Whole warps iterate together so that the ballots below see every lane.
    for (uint64_t base = uint64_t(blockIdx.x) * blockDim.x; base < n; base += stride) {
        const uint64_t i = base + threadIdx.x;
        uint32_t e = 0;
        if (i < n) {
            const double2 a = load_sample(f, i);
            packed[i] = a;
            if (i / g.np + 1u != g.nt) {
                const double2 b = load_sample(f, i + g.np);
                if (!available(a) || !available(b))
                    e = ICP_TRANSITION_UNKNOWN;
                else {
                    const double x = a.x + a.y, y = b.x + b.y, peak = fmax(x, y);
                    if (peak > 0 && finite64(peak) && !(fabs(y - x) / peak < g.contrast)) {
                        if (__ldg(&f[i].family_hits[2]) == 0u && __ldg(&f[i + g.np].family_hits[2]) > 0u &&
                            __ldg(&f[i + g.np].family_incoherent[2]) > 0)
                            e |= ICP_TRANSITION_PRIMARY;
                        if (__ldg(&f[i].family_hits[3]) > 0u && __ldg(&f[i + g.np].family_hits[3]) == 0u &&
                            __ldg(&f[i].family_incoherent[3]) > 0)
                            e |= ICP_TRANSITION_SECONDARY;
                    }
                }
            }
            edges[i] = e;
            if (e) atomicOr(&row_marks[i / g.np], 1u);
        }
        warp_count(counters, kPrimary, (e & ICP_TRANSITION_PRIMARY) != 0);
        warp_count(counters, kSecondary, (e & ICP_TRANSITION_SECONDARY) != 0);
        warp_count(counters, kUnknown, (e & ICP_TRANSITION_UNKNOWN) != 0);
    }
}

__global__ void __launch_bounds__(kThreads) rainbow_prepare_kernel(const icp_focal_sample* __restrict__ f,
                                                                   const uint32_t* __restrict__ edges, Grid g,
                                                                   double2* __restrict__ packed,
                                                                   uint32_t* __restrict__ row_marks)
{
    const uint64_t n = uint64_t(g.nt) * g.np, stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        packed[i] = load_sample(f, i);
        if (__ldg(&edges[i])) atomicOr(&row_marks[i / g.np], 1u);
    }
}

__device__ __forceinline__ int wrap_column(int a, int n)
{
    const int r = a % n;
    return r < 0 ? r + n : r;
}

// Per-row terms of the haversine distance between colatitude t and row colatitude tr
// (RainbowDiffraction::angular_distance): only sin(phi / 2) varies along the row.
struct RowTerms {
    double uu, ss; // sin((t - tr) / 2)^2, sin(t) sin(tr)
};
__device__ __forceinline__ RowTerms row_terms(double t, double st, double tr)
{
    const double u = sin(0.5 * (t - tr));
    return {u * u, st * sin(tr)};
}
__device__ __forceinline__ double row_distance(const RowTerms& r, double phi)
{
    const double v = sin(0.5 * phi);
    const double h = fma(r.ss, v * v, r.uu);
    return 2 * asin(sqrt(fmin(1.0, fmax(0.0, h))));
}
// Half-width in columns of the cap's longitude window on row colatitude r, -1 when the row
// misses the cap, nc when the cap wraps it (RainbowDiffraction::phi_radius).
__device__ __forceinline__ int cap_window(double t, double st, double ct, double r, double radius, double cos_radius,
                                          double dp, int nc)
{
    if (fabs(t - r) > radius + kCapSlack) return -1;
    const double a = st * sin(r), b = ct * cos(r);
    if (!(a > 0)) return nc;
    const double x = (cos_radius - b) / a;
    if (x <= -1) return nc;
    if (x >= 1) return 1;
    const int w = int(ceil(acos(x) / dp)) + 1;
    return nc < w ? nc : w;
}

struct Compensated {
    double s = 0, c = 0;
    __device__ __forceinline__ void add(double x)
    {
        const double n = s + x;
        c += fabs(s) >= fabs(x) ? (s - n) + x : (x - n) + s;
        s = n;
    }
    __device__ __forceinline__ double value() const { return s + c; }
};

__device__ icp_diffraction_result filter_direction(const double2* __restrict__ packed,
                                                   const uint32_t* __restrict__ edges,
                                                   const uint32_t* __restrict__ row_marks, const Grid& g,
                                                   uint32_t index)
{
    icp_diffraction_result out{};
    const double2 center = packed[index];
    if (!available(center)) {
        out.flags = ICP_DIFFRACTION_INPUT_UNAVAILABLE;
        out.intensity_s = out.intensity_p = nan64();
        return out;
    }
    out.intensity_s = center.x;
    out.intensity_p = center.y;
    const int nr = int(g.nt), nc = int(g.np), row = int(index / g.np), col = int(index % g.np);
    const double dt = kPi / double(nr), dp = 2 * kPi / double(nc), t = (row + 0.5) * dt;
    const double st = sin(t), ct = cos(t);
    const double support = g.support;

    // Nearest labelled edge within twice the primary support, in units of its own sigma.
    const double search = 2 * g.sigma * support, cos_search = cos(search);
    const int lo = max(0, int(floor((t - search) / dt)) - 1);
    const int hi = min(nr - 2, int(ceil((t + search) / dt)));
    double best = support + 1;
    for (int rr = lo; rr <= hi; ++rr) {
        if (!__ldg(&row_marks[rr])) continue;
        const double tr = (rr + 1.0) * dt;
        const int w = cap_window(t, st, ct, tr, search, cos_search, dp, nc);
        if (w < 0) continue;
        const int count = min(nc, 2 * w + 1), start = count == nc ? 0 : col - w;
        const RowTerms terms = row_terms(t, st, tr);
        const uint32_t* edge_row = edges + uint32_t(rr) * g.np;
        for (int j = 0; j < count; ++j) {
            const int cc = wrap_column(start + j, nc);
            const uint32_t e = __ldg(&edge_row[cc]);
            if (!e) continue;
            const double d = row_distance(terms, (cc - col) * dp);
            if (d > search + kCapSlack) continue;
            if (e & ICP_TRANSITION_UNKNOWN) out.flags |= ICP_DIFFRACTION_DETECTION_UNAVAILABLE;
            for (uint32_t kind = ICP_TRANSITION_PRIMARY; kind <= ICP_TRANSITION_SECONDARY; kind *= 2u) {
                if (!(e & kind)) continue;
                const double sigma = g.sigma * (kind == ICP_TRANSITION_SECONDARY ? 2 : 1);
                const double distance = d / sigma;
                if (distance < support &&
                    (distance < best - 1e-12 || (fabs(distance - best) <= 1e-12 && kind < out.transition_kind))) {
                    best = distance;
                    out.sigma_rad = sigma;
                    out.transition_kind = kind;
                }
            }
        }
    }
    if (out.flags & ICP_DIFFRACTION_DETECTION_UNAVAILABLE) {
        out.intensity_s = out.intensity_p = nan64();
        return out;
    }
    if (out.transition_kind == 0) return out; // unchanged: no global blur

    const double sigma = out.sigma_rad;
    if (dt > 0.5 * sigma || st * dp > 0.5 * sigma) out.flags |= ICP_DIFFRACTION_UNDERRESOLVED;
    out.blend = 1;
    if (best > g.inner) {
        const double x = (best - g.inner) / (support - g.inner);
        out.blend = 1 - x * x * (3 - 2 * x);
    }
    const double radius = support * sigma, cos_radius = cos(radius);
    const int lower = max(0, int(floor((t - radius) / dt)) - 1);
    const int upper = min(nr - 1, int(ceil((t + radius) / dt)));
    const double half_dt = sin(0.5 * dt);
    Compensated sum_s, sum_p, weights;
    bool holes = false;
    for (int rr = lower; rr <= upper; ++rr) {
        const double tr = (rr + 0.5) * dt;
        const int w = cap_window(t, st, ct, tr, radius, cos_radius, dp, nc);
        if (w < 0) continue;
        const int count = min(nc, 2 * w + 1), start = count == nc ? 0 : col - w;
        const double area = 2 * sin(tr) * half_dt * dp;
        const RowTerms terms = row_terms(t, st, tr);
        const double2* sample_row = packed + uint32_t(rr) * g.np;
        for (int j = 0; j < count; ++j) {
            const int cc = wrap_column(start + j, nc);
            const double d = row_distance(terms, (cc - col) * dp);
            if (d > radius + kCapSlack) continue;
            const double2 q = sample_row[cc];
            if (!available(q)) {
                holes = true;
                continue;
            }
            const double weight = exp(-0.5 * (d / sigma) * (d / sigma)) * area;
            weights.add(weight);
            sum_s.add(weight * q.x);
            sum_p.add(weight * q.y);
        }
    }
    if (holes) { // no hole filling: an unavailable neighbour makes the direction unavailable
        out.flags |= ICP_DIFFRACTION_STENCIL_UNAVAILABLE;
        out.intensity_s = out.intensity_p = nan64();
        return out;
    }
    const double total = weights.value();
    if (!(total > 0) || !finite64(total)) {
        out.flags |= ICP_DIFFRACTION_INVALID_DATA;
        out.intensity_s = out.intensity_p = nan64();
        return out;
    }
    // Constant-preserving local normalisation, blended toward the unfiltered value.
    out.intensity_s = fma(out.blend, sum_s.value() / total - center.x, center.x);
    out.intensity_p = fma(out.blend, sum_p.value() / total - center.y, center.y);
    if (!(out.intensity_s >= 0 && out.intensity_p >= 0) || !finite64(out.intensity_s + out.intensity_p)) {
        out.flags |= ICP_DIFFRACTION_INVALID_DATA;
        out.intensity_s = out.intensity_p = nan64();
        return out;
    }
    out.flags |= ICP_DIFFRACTION_FILTERED;
    return out;
}

__global__ void __launch_bounds__(kThreads) rainbow_filter_kernel(const double2* __restrict__ packed,
                                                                  const uint32_t* __restrict__ edges,
                                                                  const uint32_t* __restrict__ row_marks, Grid g,
                                                                  icp_diffraction_result* __restrict__ results,
                                                                  double* __restrict__ density,
                                                                  uint32_t* __restrict__ counters)
{
    const uint64_t n = uint64_t(g.nt) * g.np, stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t base = uint64_t(blockIdx.x) * blockDim.x; base < n; base += stride) {
        const uint64_t i = base + threadIdx.x;
        uint32_t flags = 0;
        bool unavailable = false;
        if (i < n) {
            const icp_diffraction_result r = filter_direction(packed, edges, row_marks, g, uint32_t(i));
            results[i] = r;
            if (density) density[i] = r.intensity_s + r.intensity_p;
            flags = r.flags;
            unavailable = (flags & kUnavailableMask) != 0u;
        }
        warp_count(counters, kFiltered, (flags & ICP_DIFFRACTION_FILTERED) != 0);
        warp_count(counters, kUnavailable, unavailable);
        warp_count(counters, kUnderresolved, (flags & ICP_DIFFRACTION_UNDERRESOLVED) != 0);
    }
}

// Scratch of one call: packed samples (16 B per direction), row marks, counters.
struct Buffers {
    double2* packed;
    uint32_t* rows;
    uint32_t* counters;
};

int prepare(icp_context* ctx, const icp_focal_sample* d_focal, uint32_t nt, uint32_t np,
            const icp_diffraction_config* config, Grid& g, Buffers& b, unsigned& blocks)
{
    if (!ctx || !d_focal || !config) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_rainbow: null argument");
    if (!config_ok(nt, np, *config)) return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid diffraction/grid configuration.");
    g = {config->primary_sigma_rad, config->support_sigma, config->transition_contrast, config->inner_blend_sigma, nt, np};
    const uint64_t n = uint64_t(nt) * np;
    const size_t packed = n * sizeof(double2), rows = (size_t(nt) + 1) & ~size_t(1);
    ICP_CUDA(cudaSetDevice(ctx->device));
    ICP_CUDA(ctx->rainbow.ensure(packed + (rows + kCounters + 2) * sizeof(uint32_t)));
    b.packed = static_cast<double2*>(ctx->rainbow.ptr);
    b.rows = reinterpret_cast<uint32_t*>(static_cast<char*>(ctx->rainbow.ptr) + packed);
    b.counters = b.rows + rows;
    ICP_CUDA(cudaMemsetAsync(b.rows, 0, (rows + kCounters) * sizeof(uint32_t), ctx->stream));
    const uint64_t need = (n + kThreads - 1) / kThreads, cap = uint64_t(ctx->sms > 0 ? ctx->sms : 148) * 8u;
    blocks = unsigned(need < cap ? need : cap);
    return ICP_OK;
}

int finish(icp_context* ctx, const Buffers& b, icp_diffraction_stats* stats)
{
    if (stats) {
        uint32_t c[kCounters];
        ICP_CUDA(cudaMemcpyAsync(c, b.counters, sizeof c, cudaMemcpyDeviceToHost, ctx->stream));
        ICP_CUDA(cudaStreamSynchronize(ctx->stream));
        *stats = {c[kPrimary], c[kSecondary], c[kUnknown], c[kFiltered], c[kUnavailable], c[kUnderresolved]};
    } else
        ICP_CUDA(cudaStreamSynchronize(ctx->stream));
    return ok();
}

} // namespace

extern "C" {

int icp_rainbow_table_sigma(float radius_mm, double* primary_sigma_deg)
{
    // Sadeghi et al. (2012) Table II: primary-bow width (degrees) at radii 0.1 .. 1.0 mm,
    // linear between the tabulated radii, no extrapolation.
    static const float radii[10] = {0.1f, 0.2f, 0.3f, 0.4f, 0.5f, 0.6f, 0.7f, 0.8f, 0.9f, 1.0f};
    static const double widths[10] = {0.70, 0.45, 0.30, 0.25, 0.22, 0.20, 0.18, 0.17, 0.16, 0.15};
    if (!primary_sigma_deg) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_rainbow_table_sigma: null argument");
    if (!(radius_mm >= radii[0] && radius_mm <= radii[9]))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Table II covers radius 0.1..1.0 mm only.");
    for (unsigned j = 0; j < 10; ++j) {
        if (radius_mm == radii[j]) {
            *primary_sigma_deg = widths[j];
            return ok();
        }
        if (j > 0 && radius_mm < radii[j]) {
            const double f = (double(radius_mm) - radii[j - 1]) / (double(radii[j]) - radii[j - 1]);
            *primary_sigma_deg = std::fma(f, widths[j] - widths[j - 1], widths[j - 1]);
            return ok();
        }
    }
    return fail(ICP_ERR_INVALID_ARGUMENT, "Table II covers radius 0.1..1.0 mm only.");
}

int icp_rainbow_detect(icp_context* ctx, const icp_focal_sample* d_focal, uint32_t nt, uint32_t np,
                       const icp_diffraction_config* config, uint32_t* d_transitions)
{
    if (!d_transitions) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_rainbow_detect: null argument");
    Grid g;
    Buffers b;
    unsigned blocks;
    if (const int st = prepare(ctx, d_focal, nt, np, config, g, b, blocks)) return st;
    rainbow_detect_kernel<<<blocks, kThreads, 0, ctx->stream>>>(d_focal, g, d_transitions, b.packed, b.rows, b.counters);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    return finish(ctx, b, nullptr);
}

int icp_rainbow_filter(icp_context* ctx, const icp_focal_sample* d_focal, const uint32_t* d_transitions, uint32_t nt,
                       uint32_t np, const icp_diffraction_config* config, icp_diffraction_result* d_results,
                       double* d_density, icp_diffraction_stats* stats)
{
    if (!d_transitions || !d_results) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_rainbow_filter: null argument");
    Grid g;
    Buffers b;
    unsigned blocks;
    if (const int st = prepare(ctx, d_focal, nt, np, config, g, b, blocks)) return st;
    rainbow_prepare_kernel<<<blocks, kThreads, 0, ctx->stream>>>(d_focal, d_transitions, g, b.packed, b.rows);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    rainbow_filter_kernel<<<blocks, kThreads, 0, ctx->stream>>>(b.packed, d_transitions, b.rows, g, d_results,
                                                                d_density, b.counters);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    return finish(ctx, b, stats);
}

int icp_rainbow_diffraction(icp_context* ctx, const icp_focal_sample* d_focal, uint32_t nt, uint32_t np,
                            const icp_diffraction_config* config, uint32_t* d_transitions,
                            icp_diffraction_result* d_results, double* d_density, icp_diffraction_stats* stats)
{
    if (!d_transitions || !d_results) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_rainbow_diffraction: null argument");
    Grid g;
    Buffers b;
    unsigned blocks;
    if (const int st = prepare(ctx, d_focal, nt, np, config, g, b, blocks)) return st;
    rainbow_detect_kernel<<<blocks, kThreads, 0, ctx->stream>>>(d_focal, g, d_transitions, b.packed, b.rows, b.counters);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    rainbow_filter_kernel<<<blocks, kThreads, 0, ctx->stream>>>(b.packed, d_transitions, b.rows, g, d_results,
                                                                d_density, b.counters);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    return finish(ctx, b, stats);
}

} // extern "C"
