// icp_bin.cuh -- (u,phi) binning and the privatised histogram used by the trace kernels.
//
// Binning follows hex_phase/include/ice_crystal/phase_math.hpp:37-81:
//   x = e0.d, y = e1.d, z = ki.d (d in the ensemble frame), mu = z, s = |(x,y)|;
//   s below the pole tolerance -> forward / backward pole cap (spread over the end row later);
//   u = 0.5 s^2/(1+mu) or 1 - 0.5 s^2/(1-mu); row from the saved u edges; phi = atan2(y,x)
//   with the periodic seam, column = floor(v * np) after a roundoff snap to the nearest edge.
// FP64 path: the reference arithmetic and tolerances.  FP32 path: the same rules with
// tolerances scaled to binary32 rounding (pole cap 2^-15 rad, snap windows of a few ulps),
// the row found analytically from the scattering angle (the edges are uniform in theta) and
// corrected against the stored edges.
#pragma once
#include "icp_device.cuh"

namespace icp {

struct BinResult {
    uint32_t cell;
    int pole;   // +1 forward, -1 backward, 0 cell
    bool valid, snapped;
    double mu;
};

// ------------------------------------------------------------------ FP64 (reference rules)
struct BinGridD {
    double rot[9]; // column-major body -> ensemble
    double ki[3], e0[3], e1[3];
    const double* edges; // nt+1, device (global or shared)
    uint32_t nt, np;
};

__device__ __forceinline__ BinResult bin_f64(const BinGridD& g, const double* edges, V3<double> d)
{
    BinResult b{0u, 0, false, false, 0.0};
    // Rotation::apply (phase_math.hpp:9): x*p.x + y*p.y + z*p.z, column vectors
    const V3<double> cx = v3(g.rot[0], g.rot[1], g.rot[2]);
    const V3<double> cy = v3(g.rot[3], g.rot[4], g.rot[5]);
    const V3<double> cz = v3(g.rot[6], g.rot[7], g.rot[8]);
    const V3<double> w = (cx * d.x + cy * d.y) + cz * d.z;
    const double x = g.e0[0] * w.x + g.e0[1] * w.y + g.e0[2] * w.z;
    const double y = g.e1[0] * w.x + g.e1[1] * w.y + g.e1[2] * w.z;
    const double z = g.ki[0] * w.x + g.ki[1] * w.y + g.ki[2] * w.z;
    const double n = sqrt(x * x + y * y + z * z);
    if (!(n > 0) || !finite_r(n) || fabs(n - 1) > 512 * Eps<double>::eps) return b;
    const double mu = z / n, s = hypot(x, y) / n;
    b.mu = mu;
    if (s <= 256 * Eps<double>::eps) {
        b.pole = mu >= 0 ? 1 : -1;
        b.valid = true;
        return b;
    }
    const double u = mu >= 0 ? (0.5 * s * s) / (1 + mu) : 1 - (0.5 * s * s) / (1 - mu);
    if (!(u >= 0 && u <= 1)) return b;
    uint32_t lo = 0, hi = g.nt;
    while (lo + 1 < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (u >= edges[mid]) lo = mid;
        else hi = mid;
    }
    for (unsigned c = 0; c < 2; ++c) {
        const uint32_t e = lo + c;
        if (e == 0 || e >= g.nt) continue;
        const double width = fmin(edges[e] - edges[e - 1], edges[e + 1] - edges[e]);
        const double tol = fmin(64 * Eps<double>::eps * fmax(fabs(u), fabs(edges[e])), 1e-7 * width);
        if (fabs(u - edges[e]) <= tol) {
            b.snapped = (u != edges[e]);
            lo = e;
            break;
        }
    }
    double phi = atan2(y, x);
    if (phi >= kPi) phi -= 2 * kPi;
    const double v = (phi + kPi) / (2 * kPi);
    double index = v * g.np;
    const double nearest = floor(index + 0.5);
    if (fabs(index - nearest) <= fmin(64 * Eps<double>::eps * g.np, 1e-7)) {
        b.snapped = b.snapped || (index != nearest);
        index = nearest;
    }
    uint32_t j = (uint32_t)index;
    if (j == g.np) j = 0;
    if (j >= g.np) return b;
    b.cell = lo * g.np + j;
    b.valid = true;
    return b;
}

// ------------------------------------------------------------------ FP32 (fast path)
struct BinGridF {
    float m[9];   // rows e0^T R, e1^T R, ki^T R : body direction -> (x, y, z)
    float theta_scale; // nt / pi
    uint32_t nt, np;
    float np_f;
};

constexpr float kPoleTolF = 0x1p-15f;     // rad: far above FP32 direction noise, far below a cell
constexpr float kSnapRelF = 0x1p-21f;     // relative snap window (a few binary32 ulps)

__device__ __forceinline__ BinResult bin_f32(const BinGridF& g, const float* edges, V3<float> d)
{
    BinResult b{0u, 0, false, false, 0.0};
    const float x = fmaf(g.m[0], d.x, fmaf(g.m[1], d.y, g.m[2] * d.z));
    const float y = fmaf(g.m[3], d.x, fmaf(g.m[4], d.y, g.m[5] * d.z));
    const float z = fmaf(g.m[6], d.x, fmaf(g.m[7], d.y, g.m[8] * d.z));
    const float n2 = fmaf(x, x, fmaf(y, y, z * z));
    if (!(n2 > 0.5f && n2 < 2.0f)) return b;
    const float inv = rsqrtf(n2);
    const float s = sqrtf(fmaf(x, x, y * y)) * inv;
    const float mu = z * inv;
    b.mu = mu;
    if (s <= kPoleTolF) {
        b.pole = mu >= 0.f ? 1 : -1;
        b.valid = true;
        return b;
    }
    const float u = mu >= 0.f ? (0.5f * s * s) / (1.f + mu) : 1.f - (0.5f * s * s) / (1.f - mu);
    // rows are uniform in the scattering angle: edges_i = sin^2(pi i / (2 nt)).  The row is
    // guessed from Hastings' acos approximation (Abramowitz & Stegun 4.4.45, |error| <= 6.7e-5
    // rad) and then settled against the stored edges, so the guess only sets where the search
    // starts: one step for rows wider than the error (nt below ~20000), a few more above.
    const float am = fminf(fabsf(mu), 1.f);
    const float acos_am = sqrtf(1.f - am) *
        fmaf(fmaf(fmaf(-0.0187293f, am, 0.0742610f), am, -0.2121144f), am, 1.5707288f);
    const float theta = mu >= 0.f ? acos_am : 3.14159265f - acos_am;
    int i = __float2int_rd(theta * g.theta_scale);
    const int last = (int)g.nt - 1;
    i = i < 0 ? 0 : (i > last ? last : i);
    while (i > 0 && u < edges[i]) --i;
    while (i < last && u >= edges[i + 1]) ++i;
    // canonical half-open assignment within binary32 roundoff of an interior edge
    if (i > 0 && fabsf(u - edges[i]) <= kSnapRelF * fmaxf(u, edges[i])) b.snapped = (u != edges[i]);
    if (i < last && fabsf(u - edges[i + 1]) <= kSnapRelF * fmaxf(u, edges[i + 1])) {
        b.snapped = (u != edges[i + 1]);
        ++i;
    }
    // azimuth: exact edges for directions in the coordinate planes of the frame
    float index;
    if (y == 0.f) index = x > 0.f ? 0.5f * g.np_f : 0.f;
    else if (x == 0.f) index = y > 0.f ? 0.75f * g.np_f : 0.25f * g.np_f;
    else {
        const float phi = atan2f(y, x);
        const float v = fmaf(phi, 0.15915494309189535f, 0.5f); // (phi + pi) / (2 pi)
        index = v * g.np_f;
        const float nearest = rintf(index);
        if (fabsf(index - nearest) <= kSnapRelF * g.np_f) {
            b.snapped = b.snapped || index != nearest;
            index = nearest;
        }
    }
    uint32_t j = (uint32_t)__float2int_rd(index);
    if (j >= g.np) j = (index < 0.f) ? 0u : (j == g.np ? 0u : g.np - 1u);
    b.cell = (uint32_t)i * g.np + j;
    b.valid = true;
    return b;
}

// ------------------------------------------------------------------ privatised histogram
// Shared-memory open-addressing table (key = cell + 1, value = fixed-point power), filled by
// one leader per group of lanes that hit the same cell in a warp step.  Lanes of a group are
// found with match.any; their 44-bit fixed-point values are summed exactly with two 32-bit
// redux.sync operations on 22-bit halves.  Inserts that find no slot within kProbe probes go
// straight to the FP64 global histogram.
constexpr int kProbe = 8;

struct SmemHist {
    uint32_t* keys;
    unsigned long long* vals;
    uint32_t mask; // slots - 1 ; 0 disables the table
};

__device__ __forceinline__ uint32_t hash_cell(uint32_t k) { return (k * 0x9E3779B1u) >> 7; }

__device__ __forceinline__ void hist_add(const SmemHist& h, double* global_mass, double to_mass, bool has,
                                         uint32_t cell, uint64_t v, uint32_t& fallback)
{
    const unsigned act = __ballot_sync(kFull, has);
    if (!act) return;
    if (has) {
        const unsigned peers = __match_any_sync(act, cell);
        const unsigned lo = (unsigned)(v & 0x3FFFFFull), hi = (unsigned)(v >> 22);
        const unsigned slo = __reduce_add_sync(peers, lo);
        const unsigned shi = __reduce_add_sync(peers, hi);
        const unsigned lane = threadIdx.x & 31u;
        if (lane == (unsigned)(__ffs(peers) - 1)) {
            const uint64_t sum = ((uint64_t)shi << 22) + (uint64_t)slo;
            bool done = false;
            if (h.mask) {
                const uint32_t key = cell + 1u;
                uint32_t slot = hash_cell(cell) & h.mask;
#pragma unroll 1
                for (int probe = 0; probe < kProbe; ++probe) {
                    uint32_t k = *((volatile uint32_t*)&h.keys[slot]);
                    if (k == 0u) k = atomicCAS(&h.keys[slot], 0u, key);
                    if (k == 0u || k == key) {
                        atomicAdd(&h.vals[slot], (unsigned long long)sum);
                        done = true;
                        break;
                    }
                    slot = (slot + 1u) & h.mask;
                }
            }
            if (!done) {
                atomicAdd(&global_mass[cell], (double)sum * to_mass);
                ++fallback;
            }
        }
    }
}

// Flush the table (after __syncthreads) into the FP64 histogram and clear it.
__device__ __forceinline__ void hist_flush(const SmemHist& h, double* global_mass, double to_mass)
{
    if (!h.mask) return;
    for (uint32_t s = threadIdx.x; s <= h.mask; s += blockDim.x) {
        const uint32_t k = h.keys[s];
        if (k) {
            atomicAdd(&global_mass[k - 1u], (double)h.vals[s] * to_mass);
            h.keys[s] = 0u;
            h.vals[s] = 0ull;
        }
    }
}

} // namespace icp
