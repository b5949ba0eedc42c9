// icp_atlas.cu -- deterministic single-particle atlas on the device (sm_100a) and its C ABI
// (include/icp_b200.h, "deterministic atlas").  Built with -fmad=false: every binary64
// operation rounds on its own, as the reference's host code does.
//
// Three kernels, none with floating-point atomics:
//   atlas_trace_kernel     one thread per projected-area quadrature ray of one incident node:
//                          the prism's linear R/T chain in FP64 (hex_trace_core.hpp:100-160),
//                          exits binned with the record path's FP64 binning and added as exact
//                          64-bit integers in units of 2^-62 of the node's quadrature weight;
//                          per-ray audits (escaped power as a Kahan sum in emission order,
//                          residual, interface balance, status) for the host's gates.
//   atlas_coupling_kernel  one thread per orientation: fold r^T ki into the D6h fundamental
//                          domain, bilinear incident interpolation, fractional phi shift;
//                          contributions added as exact integers (2^-62 of an upper bound of
//                          the projected area), so the coupling does not depend on the order
//                          in which threads run (atlas_math.py:186-310).
//   atlas_compose_kernel   out[t][p] = sum_(n,q,s) w[n][q][s] * M_n[t][(p - s) mod np]
//                          (phi reflected when q = 1) over the nonzero shifts only, compacted
//                          per (node, parity) in shift order by atlas_weights_compact_kernel
//                          (the couplings are ~4 % nonzero); kTT rows of a node in shared
//                          memory, a thread per cell column; products and sums are rounded
//                          separately in the order node, parity, shift -- the order of
//                          compose_mass's elementwise `out += value * roll(cell)`
//                          (atlas_math.py:431-447), so equal weights give equal bits.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/icp_b200.h"
#include "../host/icp_atlas_host.hpp"
#include "../host/icp_host_math.hpp"
#include "icp_atlas_window.cuh"
#include "icp_hex_kernel.cuh"
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

constexpr double kFix62 = 0x1p62;
constexpr uint64_t kAtlasChunk = 1ull << 20; // quadrature rays per trace launch (72 MiB of scratch)
constexpr double kUnit62 = 0x1p-62;

// ------------------------------------------------------------------ trace
struct AtlasAudit {
    double escaped, residual, max_iface;
    uint32_t status, outputs;
};
static_assert(sizeof(AtlasAudit) == 32, "AtlasAudit layout");

struct AtlasTrace {
    HexGeo<double> geo; // half_len is the only field read (strict_face_point, next_boundary)
    V3<double> k, ke0;
    Media<double> enter, leave;
    double tail;
    uint32_t max_hits;
    BinGridD grid;
    const icp_atlas_ray* rays;
    uint64_t count;
    double scale;              // fixed-point units per mm^2
    unsigned long long* cells; // nt*np
    unsigned long long* acc;   // [0] forward pole, [1] backward pole, [2] exits outside the grid
    AtlasAudit* audits;
};

__global__ void __launch_bounds__(128) atlas_trace_kernel(const AtlasTrace P)
{
    const uint64_t id = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= P.count) return;
    const icp_atlas_ray q = P.rays[id];
    const double wscale = q.weight_mm2 * P.scale;
    double esc = 0, esc_c = 0;
    uint32_t outputs = 0;
    double max_iface = 0, residual = 1;
    int status = ICP_RAY_INVALID;
    // one exit (emit_exit, hex_trace_core.hpp:77-93): 0, or the status that ends the ray
    auto emit = [&](V3<double> d, double pw) -> int {
        if (!(pw >= 0) || !finite_r(pw)) return ICP_RAY_NUMERICAL;
        if (pw == 0) return 0;
        const BinResult b = bin_f64(P.grid, P.grid.edges, d);
        if (!b.valid) {
            // the reference's mass sink refuses the sample: OutputOverflow
            atomicAdd(&P.acc[2], 1ull);
            return ICP_RAY_OVERFLOW;
        }
        const unsigned long long fx = __double2ull_rn(wscale * pw);
        if (fx) {
            if (b.pole > 0) atomicAdd(&P.acc[0], fx);
            else if (b.pole < 0) atomicAdd(&P.acc[1], fx);
            else atomicAdd(&P.cells[b.cell], fx);
        }
        const double y = pw - esc_c, t = esc + y;
        esc_c = (t - esc) - y;
        esc = t;
        ++outputs;
        return 0;
    };
    V3<double> p = v3(q.x, q.y, q.z);
    const unsigned f0 = q.face;
    if (f0 < 8u && !strict_face_point(P.geo, p, f0)) {
        status = ICP_RAY_AMBIGUOUS;
    } else if (f0 < 8u && dot(face_normal<double>(f0), P.k) < 0) {
        Interface<double> sp = split(P.k, P.ke0, Stokes<double>{1.0, 0.0, 0.0, 0.0}, face_normal<double>(f0), P.enter);
        max_iface = fabs(sp.balance);
        int e = emit(sp.dr, sp.r.I);
        if (e) {
            status = e;
        } else if (!sp.has_t) {
            status = ICP_RAY_EXHAUSTED;
            residual = 0;
        } else {
            V3<double> d = sp.dt, ef = sp.s;
            Stokes<double> S = sp.t;
            unsigned face = f0;
            status = -1;
            for (uint32_t enc = 0; enc < P.max_hits; ++enc) {
                const double pw = S.I;
                if (!(pw >= 0) || !finite_r(pw)) { status = ICP_RAY_NUMERICAL; residual = pw; break; }
                if (pw == 0) { status = ICP_RAY_EXHAUSTED; residual = 0; break; }
                if (pw <= P.tail) { status = ICP_RAY_TAIL; residual = pw; break; }
                double t;
                const Boundary hit = next_boundary(P.geo, p, d, face, t);
                if (hit.status) {
                    status = hit.status == 3 ? ICP_RAY_AMBIGUOUS : ICP_RAY_NUMERICAL;
                    residual = pw;
                    break;
                }
                sp = split(d, ef, S, -face_normal<double>(hit.face), P.leave);
                max_iface = fmax(max_iface, fabs(sp.balance));
                if (sp.has_t) {
                    e = emit(sp.dt, sp.t.I);
                    if (e) { status = e; residual = pw; break; }
                }
                d = sp.dr;
                ef = sp.s;
                S = sp.r;
                face = hit.face;
            }
            if (status < 0) {
                residual = S.I;
                status = (!(residual >= 0) || !finite_r(residual)) ? ICP_RAY_NUMERICAL
                         : residual == 0                          ? ICP_RAY_EXHAUSTED
                         : residual <= P.tail                     ? ICP_RAY_TAIL
                                                                  : ICP_RAY_LIMIT;
            }
        }
    }
    P.audits[id] = AtlasAudit{esc, residual, max_iface, (uint32_t)status, outputs};
}

// Cell masses (mm^2) from the fixed-point histogram; pole mass spread evenly over the end
// rows; the exact integer total of the histogram for the audit.
__global__ void __launch_bounds__(256) atlas_mass_kernel(const unsigned long long* cells,
                                                         const unsigned long long* acc, uint32_t nt, uint32_t np,
                                                         double unit, double* mass, unsigned long long* total)
{
    const uint64_t n = (uint64_t)nt * np;
    unsigned long long local = 0;
    const double fwd = (double)acc[0] * unit / np, bwd = (double)acc[1] * unit / np;
    for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long v = cells[c];
        double m = (double)v * unit;
        const uint64_t row = c / np;
        if (row == 0) m += fwd;
        if (row == nt - 1) m += bwd;
        mass[c] = m;
        local += v;
    }
    for (int o = 16; o; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31u) == 0 && local) atomicAdd(total, local);
}

// ------------------------------------------------------------------ coupling
struct AtlasCoupling {
    const double* rot;     // [n][9] row-major
    const double* weight;  // [n]
    uint64_t count;
    double k[3];           // unit incident direction (ensemble frame)
    double o0[3], o1[3];   // output frame e0, e1
    double half_len;       // unused by the math; kept for symmetry checks
    double side_area, cap_area; // R*L, 3 sqrt(3)/2 R^2
    double inv_unit;       // 2^62 / area bound
    uint32_t it, ip, np;
    unsigned long long* acc;      // [(it+1)(ip+1)][2][np]
    unsigned long long* expected; // [1]
    unsigned* error;              // bit 0: fold outside the domain, bit 1: unfolding, bit 2: interpolation, bit 3: non-finite
    unsigned long long* first_bad;
};

__device__ __forceinline__ void unit3(double v[3])
{
    const double s = fmax(fabs(v[0]), fmax(fabs(v[1]), fabs(v[2])));
    v[0] /= s;
    v[1] /= s;
    v[2] /= s;
    const double n = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] /= n;
    v[1] /= n;
    v[2] /= n;
}

__device__ __forceinline__ void coupling_fail(const AtlasCoupling& P, unsigned bit, uint64_t r)
{
    atomicOr(P.error, bit);
    atomicMin(P.first_bad, (unsigned long long)r);
}

__global__ void __launch_bounds__(128) atlas_coupling_kernel(const AtlasCoupling P)
{
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= P.count) return;
    const double* R = P.rot + 9 * r;
    const double nw = P.weight[r];
    // body direction r^T k, made unit (fold_direction, atlas_math.py:186-210)
    double b[3];
    for (int j = 0; j < 3; ++j) b[j] = R[j] * P.k[0] + R[3 + j] * P.k[1] + R[6 + j] * P.k[2];
    unit3(b);
    if (!finite_r(b[0]) || !finite_r(b[1]) || !finite_r(b[2]) || !finite_r(nw)) { coupling_fail(P, 8u, r); return; }
    const double third = kPi / 3, sixth = kPi / 6, two_pi = 2 * kPi;
    const double theta = atan2(hypot(b[0], b[2]), fabs(b[1]));
    double az = fmod(atan2(b[2], b[0]), two_pi);
    if (az < 0) az += two_pi;
    if (az == 0) az = 0.0; // +0 as the remainder of a floor division
    int sector = (int)(az / third);
    if (sector > 5) sector = 5;
    const double local = az - sector * third;
    const bool mirror = local > sixth;
    double phi = mirror ? third - local : local;
    const double slack = 64 * Eps<double>::eps;
    if (phi < -slack || phi > sixth + slack) { coupling_fail(P, 1u, r); return; }
    phi = fmin(sixth, fmax(0.0, phi));
    const double angle = (sector + (mirror ? 1 : 0)) * third;
    const double c = cos(-angle), s = sin(-angle);
    const double sy = b[1] < 0 ? -1.0 : 1.0, sz = mirror ? -1.0 : 1.0;
    // q = Ry(-angle) diag(1, sy, sz); canonical frame k(t,p), e0(t,p)
    const double st = sin(theta), ct = cos(theta), sp = sin(phi), cp = cos(phi);
    const double kc[3] = {st * cp, ct, st * sp};
    const double ec[3] = {ct * cp, -st, ct * sp};
    const double qk[3] = {c * kc[0] + s * sz * kc[2], sy * kc[1], -s * kc[0] + c * sz * kc[2]};
    if (fmax(fabs(qk[0] - b[0]), fmax(fabs(qk[1] - b[1]), fabs(qk[2] - b[2]))) > 2e-12) {
        coupling_fail(P, 2u, r);
        return;
    }
    const double qe[3] = {c * ec[0] + s * sz * ec[2], sy * ec[1], -s * ec[0] + c * sz * ec[2]};
    double ew[3];
    for (int i = 0; i < 3; ++i) ew[i] = R[3 * i] * qe[0] + R[3 * i + 1] * qe[1] + R[3 * i + 2] * qe[2];
    double shift = atan2(ew[0] * P.o1[0] + ew[1] * P.o1[1] + ew[2] * P.o1[2],
                         ew[0] * P.o0[0] + ew[1] * P.o0[1] + ew[2] * P.o0[2]) /
                   two_pi * P.np;
    const double nearest = rint(shift);
    if (fabs(shift - nearest) <= 64 * Eps<double>::eps * P.np) shift = nearest;
    const double lower = floor(shift), frac = shift - lower;
    const int parity = sy * sz < 0 ? 1 : 0;
    // exact projected area at the query (projected_area, atlas_math.py:226-232)
    double u[3] = {b[0], b[1], b[2]};
    unit3(u);
    double area = 0;
    {
        const double h = 0.5, q3 = kSqrt3 / 2;
        const double nx[8] = {1, h, -h, -1, -h, h, 0, 0}, nz[8] = {0, q3, q3, 0, -q3, -q3, 0, 0};
        const double ny[8] = {0, 0, 0, 0, 0, 0, 1, -1};
        for (int f = 0; f < 8; ++f) {
            const double proj = -(nx[f] * u[0] + ny[f] * u[1] + nz[f] * u[2]);
            area += (f < 6 ? P.side_area : P.cap_area) * fmax(0.0, proj);
        }
    }
    // bilinear weights of the incident nodes (interpolation, atlas_math.py:213-223)
    if (!(theta >= -slack && theta <= kPi / 2 + slack && phi >= -slack && phi <= sixth + slack)) {
        coupling_fail(P, 4u, r);
        return;
    }
    double x = theta / (kPi / 2) * P.it, y = phi / sixth * P.ip;
    x = fmin((double)P.it, fmax(0.0, x));
    y = fmin((double)P.ip, fmax(0.0, y));
    const uint32_t i0 = min(P.it - 1, (uint32_t)x), j0 = min(P.ip - 1, (uint32_t)y);
    const double ax = x - i0, by = y - j0;
    const long long np = P.np;
    const long long lo = (long long)lower;
    const uint32_t s0 = (uint32_t)(((lo % np) + np) % np), s1 = (uint32_t)((((lo + 1) % np) + np) % np);
    const double base = nw * area;
    for (int di = 0; di < 2; ++di)
        for (int dj = 0; dj < 2; ++dj) {
            const double mix = (di ? ax : 1 - ax) * (dj ? by : 1 - by);
            if (!(mix > 0)) continue;
            const uint64_t node = (uint64_t)(i0 + di) * (P.ip + 1) + (j0 + dj);
            unsigned long long* row = P.acc + (node * 2 + parity) * P.np;
            const double v = base * mix;
            const unsigned long long a0 = __double2ull_rn(v * (1 - frac) * P.inv_unit);
            const unsigned long long a1 = __double2ull_rn(v * frac * P.inv_unit);
            if (a0) atomicAdd(row + s0, a0);
            if (a1) atomicAdd(row + s1, a1);
        }
    atomicAdd(P.expected, __double2ull_rn(base * P.inv_unit));
}

// One warp per [node][parity] row: fixed point -> weights per node area; optional exact
// orbit average (the row's mean, summed in a fixed order); out += fraction * row.
__global__ void __launch_bounds__(256) atlas_coupling_finish_kernel(const unsigned long long* acc,
                                                                    const double* node_area, uint32_t rows,
                                                                    uint32_t np, double unit, double fraction,
                                                                    int orbit, double* out)
{
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
    if (warp >= rows) return;
    const double scale = unit / node_area[warp >> 1];
    const unsigned long long* a = acc + (uint64_t)warp * np;
    double* o = out + (uint64_t)warp * np;
    if (orbit) {
        double part = 0;
        for (uint32_t s = lane; s < np; s += 32) part += (double)a[s] * scale;
        for (int d = 16; d; d >>= 1) part += __shfl_xor_sync(0xffffffffu, part, d);
        const double mean = part / np;
        for (uint32_t s = lane; s < np; s += 32) o[s] += fraction * mean;
    } else {
        for (uint32_t s = lane; s < np; s += 32) o[s] += fraction * ((double)a[s] * scale);
    }
}

// ------------------------------------------------------------------ compose
constexpr int kTT = 2;                 // rows per block
constexpr int kComposeThreads = 256;   // cells per block row: threads x CPT >= np
constexpr int kCompactThreads = 256;

// The nonzero shifts of one (node, parity) coupling row, ascending, with their weights: one
// block per row, ballot ranks within each warp and the warps' counts in order, so the list's
// order is the shift order (the composition's summation order depends on it).
__global__ void __launch_bounds__(kCompactThreads) atlas_weights_compact_kernel(const double* __restrict__ w, uint32_t np,
                                                                                uint32_t* __restrict__ counts,
                                                                                uint32_t* __restrict__ shifts,
                                                                                double* __restrict__ values)
{
    __shared__ uint32_t warp_count[kCompactThreads / 32];
    __shared__ uint32_t base;
    const uint32_t row = blockIdx.x, lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const double* wr = w + (uint64_t)row * np;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    for (uint32_t s0 = 0; s0 < np; s0 += kCompactThreads) {
        const uint32_t sft = s0 + threadIdx.x;
        const double v = sft < np ? wr[sft] : 0.0;
        const bool nz = v != 0.0;
        const unsigned ballot = __ballot_sync(0xffffffffu, nz);
        if (lane == 0) warp_count[warp] = __popc(ballot);
        __syncthreads();
        uint32_t before = base;
        for (uint32_t k = 0; k < warp; ++k) before += warp_count[k];
        if (nz) {
            const uint32_t slot = before + __popc(ballot & ((1u << lane) - 1u));
            shifts[(uint64_t)row * np + slot] = sft;
            values[(uint64_t)row * np + slot] = v;
        }
        __syncthreads();
        if (threadIdx.x == 0)
            for (uint32_t k = 0; k < kCompactThreads / 32; ++k) base += warp_count[k];
        __syncthreads();
    }
    if (threadIdx.x == 0) counts[row] = base;
}

// out[t][p] = sum over nodes n, parities q and the nonzero shifts s of w[n][q][s] *
// M_n[t][(p - s) mod np] (phi-reflected when q = 1).  A block holds kTT rows of one node in
// shared memory and the (n, q) list of nonzero shifts; thread x owns the cells x + k T of its
// rows (consecutive threads read consecutive cells).  Products and sums rounded separately,
// in the order node, parity, ascending shift -- the order of compose_mass's elementwise
// `out += value * roll(cell)` (atlas_math.py:431-447), so equal weights give equal bits.
template <int CPT>
__global__ void __launch_bounds__(kComposeThreads, 2) atlas_compose_kernel(const double* __restrict__ mass,
                                                                           const uint32_t* __restrict__ counts,
                                                                           const uint32_t* __restrict__ shifts,
                                                                           const double* __restrict__ values,
                                                                           uint32_t nodes, uint32_t nt, uint32_t np,
                                                                           double* __restrict__ out)
{
    extern __shared__ __align__(16) double sm[];
    double* rows = sm;                                             // [kTT][np]
    double* lw = sm + kTT * np;                                    // [np] weights of the list
    uint32_t* ls = reinterpret_cast<uint32_t*>(lw + np);           // [np] shifts of the list
    const uint32_t t0 = blockIdx.x * kTT;
    double acc[kTT][CPT];
#pragma unroll
    for (int t = 0; t < kTT; ++t)
#pragma unroll
        for (int k = 0; k < CPT; ++k) acc[t][k] = 0.0;
    for (uint32_t n = 0; n < nodes; ++n) {
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < kTT * np; e += blockDim.x) {
            const uint32_t t = t0 + e / np;
            rows[e] = t < nt ? mass[((uint64_t)n * nt + t) * np + e % np] : 0.0;
        }
        for (int q = 0; q < 2; ++q) {
            const uint64_t r = (uint64_t)n * 2 + q;
            const uint32_t cnt = counts[r];
            __syncthreads();
            for (uint32_t e = threadIdx.x; e < cnt; e += blockDim.x) {
                lw[e] = values[r * np + e];
                ls[e] = shifts[r * np + e];
            }
            __syncthreads();
            if (threadIdx.x < np)
                for (uint32_t e = 0; e < cnt; ++e) {
                    const double wv = lw[e];
                    // m = (p - s) mod np for p = x + k T, stepped by T per cell (T < np when CPT > 1)
                    uint32_t m = phi_sub(threadIdx.x, ls[e], np);
#pragma unroll
                    for (int k = 0; k < CPT; ++k) {
                        if (k > 0) {
                            if (threadIdx.x + (uint32_t)k * kComposeThreads >= np) break;
                            m += kComposeThreads;
                            if (m >= np) m -= np;
                        }
                        const uint32_t idx = phi_cell(m, np, q);
#pragma unroll
                        for (int t = 0; t < kTT; ++t) acc[t][k] = acc[t][k] + wv * rows[t * np + idx];
                    }
                }
        }
    }
#pragma unroll
    for (int t = 0; t < kTT; ++t) {
        if (t0 + t >= nt) continue;
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const uint32_t p = threadIdx.x + (uint32_t)k * kComposeThreads;
            if (p < np) out[(uint64_t)(t0 + t) * np + p] = acc[t][k];
        }
    }
}

int validate_settings(const icp_atlas_settings* s)
{
    if (!s) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_atlas: null settings");
    const double hl = 0.5 * (s->length_mm / s->circumradius_mm);
    if (!(s->circumradius_mm > 0) || !(s->length_mm > 0) || !H::finite(s->circumradius_mm) ||
        !H::finite(s->length_mm) || !(hl > 0) || !H::finite(hl) || !(s->interior_index > 0) ||
        !(s->exterior_index > 0) || !H::finite(s->interior_index) || !H::finite(s->exterior_index) ||
        s->theta_intervals == 0 || s->phi_intervals == 0 || s->theta_intervals > 4096 || s->phi_intervals > 4096 ||
        s->nt == 0 || s->np == 0 || uint64_t(s->nt) * s->np > 100000000ull || s->subdivisions == 0 ||
        uint64_t(s->subdivisions) * s->subdivisions > 1000000ull || s->max_internal_hits == 0)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid atlas settings.");
    for (double v : {s->tail_tolerance, s->max_unresolved_fraction, s->max_balance_error})
        if (!H::finite(v) || v < 0 || v >= 1) return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid audit tolerance.");
    if (s->tail_tolerance > s->max_unresolved_fraction)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Ray tail exceeds global unresolved budget.");
    return ICP_OK;
}

const char* ray_status_name(uint32_t s)
{
    static const char* names[8] = {"exhausted", "tail_tolerance_reached", "interaction_limit", "ambiguous_boundary",
                                   "invalid_input", "numerical_failure", "output_overflow", "replay_mismatch"};
    return s < 8 ? names[s] : "unknown";
}

} // namespace

extern "C" {

int icp_atlas_area_rule(double circumradius_mm, double length_mm, const double ki[3], uint32_t subdivisions,
                        icp_atlas_ray* rays, uint64_t capacity, uint64_t* count)
{
    if (!ki || !count) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_atlas_area_rule: null argument");
    // a unit direction is used as given (make_area_rule requires one); any other is normalised
    H::V k{ki[0], ki[1], ki[2]};
    if (!H::is_unit(k) && !H::normalize(k, k))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Incident direction must be finite and nonzero.");
    std::vector<H::AtlasRay> r;
    const int st = H::atlas_area_rule(circumradius_mm, length_mm, k, subdivisions, r);
    if (st == H::kRuleInvalid) return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid area quadrature geometry / subdivision count.");
    if (st == H::kRuleBoundary || (st == H::kRuleAudit && !r.empty()))
        return fail(ICP_ERR_AUDIT, "Area quadrature is not representable / lies on ambiguous boundary.");
    if (st == H::kRuleAudit) return fail(ICP_ERR_AUDIT, "Projected-area quadrature failed conservation audit.");
    *count = r.size();
    if (!rays) return ok();
    if (capacity < r.size())
        return fail(ICP_ERR_CAPACITY, "icp_atlas_area_rule: capacity %llu < %zu rays", (unsigned long long)capacity,
                    r.size());
    static_assert(sizeof(icp_atlas_ray) == sizeof(H::AtlasRay), "ray layout");
    std::memcpy(rays, r.data(), r.size() * sizeof(icp_atlas_ray));
    return ok();
}

int icp_atlas_incident_node(uint32_t theta_intervals, uint32_t phi_intervals, uint32_t i, uint32_t j,
                            icp_atlas_incident* out)
{
    if (!out) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_atlas_incident_node: null argument");
    H::AtlasIncident a;
    if (theta_intervals == 0 || phi_intervals == 0 || theta_intervals > 4096 || phi_intervals > 4096)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid atlas settings.");
    if (i > theta_intervals || j > phi_intervals) return fail(ICP_ERR_INVALID_ARGUMENT, "Incident node index.");
    if (!H::atlas_incident(theta_intervals, phi_intervals, i, j, a))
        return fail(ICP_ERR_AUDIT, "Invalid incident spherical frame.");
    *out = icp_atlas_incident{a.theta, a.phi, {a.k.x, a.k.y, a.k.z}, {a.frame.e0.x, a.frame.e0.y, a.frame.e0.z},
                              {a.frame.e1.x, a.frame.e1.y, a.frame.e1.z}, {a.k_rule.x, a.k_rule.y, a.k_rule.z}};
    return ok();
}

int icp_atlas_trace_node(icp_context* ctx, const icp_atlas_settings* s, uint32_t i, uint32_t j, double* d_mass,
                         icp_atlas_node_report* report)
{
    if (!ctx || !d_mass || !report) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_atlas_trace_node: null argument");
    if (int e = validate_settings(s)) return e;
    if (i > s->theta_intervals || j > s->phi_intervals) return fail(ICP_ERR_INVALID_ARGUMENT, "Incident node index.");
    ICP_CUDA(cudaSetDevice(ctx->device));
    std::memset(report, 0, sizeof *report);
    report->first_rejected = -1;
    H::AtlasIncident node;
    if (!H::atlas_incident(s->theta_intervals, s->phi_intervals, i, j, node))
        return fail(ICP_ERR_AUDIT, "Invalid incident spherical frame.");
    std::vector<H::AtlasRay> rays;
    const int st = H::atlas_area_rule(s->circumradius_mm, s->length_mm, node.k_rule, s->subdivisions, rays);
    if (st == H::kRuleInvalid) return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid area quadrature geometry / subdivision count.");
    if (st != H::kRuleOk) return fail(ICP_ERR_AUDIT, "Area quadrature failed at incident node (%u, %u).", i, j);
    const double area = H::prism_faces(s->circumradius_mm, s->length_mm, node.k).area;
    H::KahanSum wsum;
    for (const auto& r : rays) wsum.add(r.weight_mm2);
    // fixed point: 2^62 units = the quadrature's total weight (with a margin for its rounding)
    const double total = wsum.value * (1 + 1e-9);
    const uint64_t nr = rays.size(), cells = uint64_t(s->nt) * s->np;
    std::vector<double> edges;
    if (!H::u_edges(s->nt, edges)) return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid u edges.");
    // scratch: rays | audits (one chunk) | edges | cells | acc[4]
    const uint64_t chunk = std::min<uint64_t>(nr, kAtlasChunk);
    const size_t off_a = (chunk * sizeof(icp_atlas_ray) + 255) & ~size_t(255);
    const size_t off_e = off_a + ((chunk * sizeof(AtlasAudit) + 255) & ~size_t(255));
    const size_t off_c = off_e + (((s->nt + 1) * sizeof(double) + 255) & ~size_t(255));
    const size_t off_x = off_c + cells * sizeof(unsigned long long);
    const size_t bytes = off_x + 4 * sizeof(unsigned long long);
    ICP_CUDA(ctx->atlas_trace.ensure(bytes));
    unsigned char* base = static_cast<unsigned char*>(ctx->atlas_trace.ptr);
    auto* d_rays = reinterpret_cast<icp_atlas_ray*>(base);
    auto* d_audit = reinterpret_cast<AtlasAudit*>(base + off_a);
    auto* d_edges = reinterpret_cast<double*>(base + off_e);
    auto* d_cells = reinterpret_cast<unsigned long long*>(base + off_c);
    auto* d_acc = reinterpret_cast<unsigned long long*>(base + off_x);
    cudaStream_t stream = ctx->stream;
    ICP_CUDA(cudaMemcpyAsync(d_edges, edges.data(), edges.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
    ICP_CUDA(cudaMemsetAsync(d_cells, 0, cells * sizeof(unsigned long long) + 4 * sizeof(unsigned long long), stream));
    AtlasTrace P{};
    P.geo.half_len = 0.5 * (s->length_mm / s->circumradius_mm);
    P.k = v3(node.k.x, node.k.y, node.k.z);
    P.ke0 = v3(node.frame.e0.x, node.frame.e0.y, node.frame.e0.z);
    P.enter = make_media<double>(s->exterior_index, s->interior_index);
    P.leave = make_media<double>(s->interior_index, s->exterior_index);
    P.tail = s->tail_tolerance;
    P.max_hits = s->max_internal_hits;
    const double id9[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    for (int q = 0; q < 9; ++q) P.grid.rot[q] = id9[q];
    const double kk[3] = {node.k.x, node.k.y, node.k.z}, e0[3] = {node.frame.e0.x, node.frame.e0.y, node.frame.e0.z},
                 e1[3] = {node.frame.e1.x, node.frame.e1.y, node.frame.e1.z};
    for (int q = 0; q < 3; ++q) {
        P.grid.ki[q] = kk[q];
        P.grid.e0[q] = e0[q];
        P.grid.e1[q] = e1[q];
    }
    P.grid.edges = d_edges;
    P.grid.nt = s->nt;
    P.grid.np = s->np;
    P.rays = d_rays;
    P.scale = kFix62 / total;
    P.cells = d_cells;
    P.acc = d_acc;
    P.audits = d_audit;
    // host gates (atlas.cpp:98-139): every ray accepted, weighted sums in ray order
    H::KahanSum escaped, unresolved;
    report->projected_area_mm2 = area;
    report->rays = nr;
    std::vector<AtlasAudit> audits(chunk);
    AtlasAudit first_bad{};
    for (uint64_t first = 0; first < nr; first += chunk) {
        const uint64_t n = std::min(chunk, nr - first);
        ICP_CUDA(cudaMemcpyAsync(d_rays, rays.data() + first, n * sizeof(icp_atlas_ray), cudaMemcpyHostToDevice,
                                 stream));
        P.count = n;
        atlas_trace_kernel<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(P);
        ICP_CUDA(cudaGetLastError());
        count_launch();
        ICP_CUDA(cudaMemcpyAsync(audits.data(), d_audit, n * sizeof(AtlasAudit), cudaMemcpyDeviceToHost, stream));
        ICP_CUDA(cudaStreamSynchronize(stream));
        for (uint64_t q = 0; q < n; ++q) {
            const AtlasAudit& a = audits[q];
            const uint64_t r = first + q;
            report->outputs += a.outputs;
            if (a.status < 8) ++report->status[a.status];
            const double bal = std::fabs(a.escaped + a.residual - 1);
            report->max_balance_error = std::max(report->max_balance_error, bal);
            report->max_interface_balance_error = std::max(report->max_interface_balance_error, a.max_iface);
            const bool accepted = (a.status == ICP_RAY_EXHAUSTED || a.status == ICP_RAY_TAIL) &&
                                  H::finite(a.max_iface) && a.max_iface <= s->max_balance_error &&
                                  bal <= s->max_balance_error;
            if (!accepted && report->first_rejected < 0) {
                report->first_rejected = (int64_t)r;
                first_bad = a;
            }
            escaped.add(rays[r].weight_mm2 * a.escaped);
            unresolved.add(rays[r].weight_mm2 * a.residual);
        }
    }
    const unsigned mblocks = (unsigned)std::min<uint64_t>((cells + 255) / 256, uint64_t(ctx->sms) * 8);
    atlas_mass_kernel<<<mblocks, 256, 0, stream>>>(d_cells, d_acc, s->nt, s->np, total * kUnit62, d_mass, d_acc + 3);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    unsigned long long acc[4];
    ICP_CUDA(cudaMemcpyAsync(acc, d_acc, sizeof acc, cudaMemcpyDeviceToHost, stream));
    ICP_CUDA(cudaStreamSynchronize(stream));
    report->invalid_bins = acc[2];
    report->escaped_mm2 = escaped.value;
    report->unresolved_mm2 = unresolved.value;
    report->histogram_mass_mm2 = (double)(acc[3] + acc[0] + acc[1]) * (total * kUnit62);
    report->histogram_relative_error = std::fabs(report->histogram_mass_mm2 / report->escaped_mm2 - 1);
    if (report->first_rejected >= 0) {
        const auto r = (uint64_t)report->first_rejected;
        return fail(ICP_ERR_AUDIT,
                    "Deterministic area ray rejected: local_id=%llu face=%u status=%s residual=%.17g. No jitter, "
                    "dropped ray, or renormalized omission is applied.",
                    (unsigned long long)r, rays[r].face, ray_status_name(first_bad.status), first_bad.residual);
    }
    if (!(report->histogram_mass_mm2 > 0) || !(report->escaped_mm2 > 0))
        return fail(ICP_ERR_AUDIT, "Incomplete atlas node.");
    if (report->histogram_relative_error > s->max_balance_error ||
        std::fabs((report->escaped_mm2 + report->unresolved_mm2) / area - 1) > s->max_balance_error ||
        report->unresolved_mm2 / area > s->max_unresolved_fraction)
        return fail(ICP_ERR_AUDIT, "Atlas area / escaped / residual conservation audit failed.");
    return ok();
}

int icp_atlas_coupling(icp_context* ctx, uint32_t it, uint32_t ip, uint32_t np, double R, double L,
                       const double* h_node_area, const double* d_rotations, const double* d_weights, uint64_t count,
                       const double ki[3], double fraction, int orbit_average, double* d_coupling,
                       double* expected_area)
{
    if (!ctx || !h_node_area || !d_rotations || !d_weights || !ki || !d_coupling || !expected_area)
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_atlas_coupling: null argument");
    if (it == 0 || ip == 0 || it > 4096 || ip > 4096 || np == 0 || count == 0 || !(R > 0) || !(L > 0) ||
        !H::finite(R) || !H::finite(L) || !(fraction > 0) || !(fraction <= 1))
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_atlas_coupling: invalid argument");
    const uint64_t nodes = uint64_t(it + 1) * (ip + 1);
    for (uint64_t n = 0; n < nodes; ++n)
        if (!(h_node_area[n] > 0) || !H::finite(h_node_area[n]))
            return fail(ICP_ERR_INVALID_ARGUMENT, "icp_atlas_coupling: node area %llu not positive",
                        (unsigned long long)n);
    H::V k;
    H::Frame f;
    if (!H::normalize(H::V{ki[0], ki[1], ki[2]}, k) || !H::make_frame(k, f))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Expected finite nonzero three-vector");
    ICP_CUDA(cudaSetDevice(ctx->device));
    // upper bound of the projected area: half the surface area of the convex prism
    const double side = R * L, cap = (3 * H::kSqrt3 / 2) * R * R, bound = 3 * side + cap;
    const uint64_t nacc = nodes * 2 * np;
    const size_t off_area = ((nacc + 4) * sizeof(unsigned long long) + 255) & ~size_t(255);
    const size_t bytes = off_area + nodes * sizeof(double);
    ICP_CUDA(ctx->atlas_coupling.ensure(bytes));
    auto* d_acc = static_cast<unsigned long long*>(ctx->atlas_coupling.ptr);
    auto* d_area = reinterpret_cast<double*>(static_cast<unsigned char*>(ctx->atlas_coupling.ptr) + off_area);
    cudaStream_t stream = ctx->stream;
    ICP_CUDA(cudaMemsetAsync(d_acc, 0, (nacc + 4) * sizeof(unsigned long long), stream));
    const unsigned long long big = ~0ull;
    ICP_CUDA(cudaMemcpyAsync(d_acc + nacc + 3, &big, sizeof big, cudaMemcpyHostToDevice, stream));
    ICP_CUDA(cudaMemcpyAsync(d_area, h_node_area, nodes * sizeof(double), cudaMemcpyHostToDevice, stream));
    AtlasCoupling P{};
    P.rot = d_rotations;
    P.weight = d_weights;
    P.count = count;
    const double kk[3] = {k.x, k.y, k.z}, o0[3] = {f.e0.x, f.e0.y, f.e0.z}, o1[3] = {f.e1.x, f.e1.y, f.e1.z};
    for (int q = 0; q < 3; ++q) {
        P.k[q] = kk[q];
        P.o0[q] = o0[q];
        P.o1[q] = o1[q];
    }
    P.half_len = 0.5 * (L / R);
    P.side_area = side;
    P.cap_area = cap;
    P.inv_unit = kFix62 / bound;
    P.it = it;
    P.ip = ip;
    P.np = np;
    P.acc = d_acc;
    P.expected = d_acc + nacc;
    P.error = reinterpret_cast<unsigned*>(d_acc + nacc + 1);
    P.first_bad = d_acc + nacc + 3;
    atlas_coupling_kernel<<<(unsigned)((count + 127) / 128), 128, 0, stream>>>(P);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    const uint32_t rows = (uint32_t)(nodes * 2);
    atlas_coupling_finish_kernel<<<(rows * 32 + 255) / 256, 256, 0, stream>>>(d_acc, d_area, rows, np,
                                                                             bound * kUnit62, fraction,
                                                                             orbit_average, d_coupling);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    unsigned long long tail[4];
    ICP_CUDA(cudaMemcpyAsync(tail, d_acc + nacc, sizeof tail, cudaMemcpyDeviceToHost, stream));
    ICP_CUDA(cudaStreamSynchronize(stream));
    const unsigned err = (unsigned)tail[1];
    if (err & 8u) return fail(ICP_ERR_INVALID_ARGUMENT, "Nonfinite orientation (rotation %llu).", tail[3]);
    if (err & 1u) return fail(ICP_ERR_AUDIT, "Canonical azimuth outside fundamental region (rotation %llu).", tail[3]);
    if (err & 2u) return fail(ICP_ERR_AUDIT, "Symmetry unfolding is inconsistent (rotation %llu).", tail[3]);
    if (err & 4u) return fail(ICP_ERR_AUDIT, "Incident interpolation outside canonical domain (rotation %llu).", tail[3]);
    *expected_area = (double)tail[0] * (bound * kUnit62);
    return ok();
}

int icp_atlas_compose(icp_context* ctx, uint32_t nodes, uint32_t nt, uint32_t np, const double* d_mass,
                      const double* d_coupling, double* d_out)
{
    if (!ctx || !d_mass || !d_coupling || !d_out) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_atlas_compose: null argument");
    if (nodes == 0 || nt == 0 || np == 0 || uint64_t(nt) * np > 100000000ull)
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_atlas_compose: invalid shape");
    const size_t smem = (size_t(kTT) + 1) * np * sizeof(double) + np * sizeof(uint32_t);
    if (smem > 227u * 1024u || np > 16u * kComposeThreads)
        return fail(ICP_ERR_CAPACITY, "icp_atlas_compose: %u phi cells need %zu bytes of shared memory (limit 227 KiB) "
                    "or more than %u cells per row", np, smem, 16u * kComposeThreads);
    ICP_CUDA(cudaSetDevice(ctx->device));
    // the nonzero coupling shifts of every (node, parity) row, compacted in shift order
    const uint64_t rowsw = uint64_t(nodes) * 2;
    const size_t o_shifts = (rowsw * 4 + 255) / 256 * 256, o_values = o_shifts + (rowsw * np * 4 + 255) / 256 * 256;
    ICP_CUDA(ctx->atlas_list.ensure(o_values + rowsw * np * 8));
    char* base = static_cast<char*>(ctx->atlas_list.ptr);
    auto* counts = reinterpret_cast<uint32_t*>(base);
    auto* shifts = reinterpret_cast<uint32_t*>(base + o_shifts);
    auto* values = reinterpret_cast<double*>(base + o_values);
    atlas_weights_compact_kernel<<<(unsigned)rowsw, kCompactThreads, 0, ctx->stream>>>(d_coupling, np, counts, shifts,
                                                                                      values);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    const uint32_t cpt = (np + kComposeThreads - 1) / kComposeThreads;
    const dim3 grid((nt + kTT - 1) / kTT);
    auto run = [&](auto kernel) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kernel<<<grid, kComposeThreads, smem, ctx->stream>>>(d_mass, counts, shifts, values, nodes, nt, np, d_out);
        return cudaGetLastError();
    };
    cudaError_t e;
    if (cpt <= 1) e = run(atlas_compose_kernel<1>);
    else if (cpt <= 2) e = run(atlas_compose_kernel<2>);
    else if (cpt <= 4) e = run(atlas_compose_kernel<4>);
    else if (cpt <= 8) e = run(atlas_compose_kernel<8>);
    else e = run(atlas_compose_kernel<16>);
    ICP_CUDA(e);
    count_launch();
    ICP_CUDA(cudaStreamSynchronize(ctx->stream));
    return ok();
}

} // extern "C"
