// icp_hex_kernel.cuh -- fused single-particle trace + (u,phi) binning kernel (sm_100a), with
// two geometries: the hexagonal prism (HexGeo) and the axisymmetric drop (DropGeo).
//
// One launch traces one orientation node's ray range [first, first+count) and adds every
// exit into the FP64 cell-mass histogram.  It replaces the reference's count kernel, serial
// prefix, replay kernel, 200-byte CSR round trip and FP64 atomic accumulate
// (hex_trace/device/hex_trace.cu:12-48, hex_phase/device/phase_accumulate.cu:10-28):
//   * persistent warps, each owning a contiguous slice of ray ids; a lane whose ray ends
//     takes the next id of its warp's slice in the next step (no warp idles on long rays);
//   * one event per lane per step: the entry split, or one internal boundary + split; each
//     event emits at most one exit, which the whole warp bins together;
//   * exits go to a shared-memory table through match.any warp aggregation, in 2^-44
//     fixed point; the table is flushed to FP64 once per block.
// Ray algorithm: hex_trace/include/ice_crystal/hex_trace_core.hpp:190-259 (linear R/T chain),
// hex_prism.hpp:64-175 (entry sampling, nearest exit plane), flux_interface.hpp:26-88.
#pragma once
#include <type_traits>
#include "icp_bin.cuh"
#include "icp_device.cuh"
#include "icp_drop.cuh"

namespace icp {

// Accumulators shared by all blocks of one launch (device memory, zeroed by the host).
// Power sums are exact 128-bit fixed-point integers (lo, hi words) in units of 2^-44.
struct DevStats {
    unsigned long long esc[2], unres[2], fwd[2], bwd[2];
    double axial;
    unsigned long long max_bal_bits, max_iface_bits; // bit patterns of non-negative doubles
    unsigned long long rays, outputs, status[8], rejected, snapped, near_edge, fallback, invalid;
    unsigned long long encounters, missed, gauge_evals;
};

__device__ __forceinline__ void add128(unsigned long long* p, unsigned long long t)
{
    if (!t) return;
    const unsigned long long old = atomicAdd(p, t);
    if (old + t < old) atomicAdd(p + 1, 1ull);
}

// Hexagonal prism in units of its circumradius, body frame (long axis +y).
template <class R> struct HexGeo {
    R half_len;
    R cum[8];           // cumulative projected face weights (plain adds in face order)
    uint32_t face_mask; // faces with positive projected weight
    R area;             // total projected weight (Kahan sum, as the reference's projected_area)
};
// Axisymmetric drop in units of its equal-volume radius; rays start on a disk of radius
// `disk` around the axis through the centre, a distance `back` before the centre.
template <class R> struct DropGeo {
    DropShape<R> shape;
    R disk, back;
    V3<R> e1;           // second transverse axis (k x ke0)
};

template <class R, class G> struct TraceParams {
    G geo;
    V3<R> k, ke0;    // incident direction and its frame vector
    R tail, bal_tol;
    unsigned long long tail_fx; // floor(tail * 2^44): the tail test of the fixed-point path
    Media<R> enter, leave; // n_ext -> n_int at entry, n_int -> n_ext inside
    uint64_t seed, total, first, count;
    uint32_t max_hits;
    uint32_t batch_size;
    uint32_t* batch_out;   // per-batch exit counters or nullptr
    // binning
    BinGridF gf;
    BinGridD gd;
    const double* edges_d; // nt+1 (global)
    const float* edges_f;  // nt+1 (global)
    double* mass;          // nt*np FP64 histogram (global)
    double to_mass;        // area weight * 2^-44
    DevStats* stats;
    uint32_t hash_slots;   // power of two, 0 = no shared table
    uint32_t smem_edges;   // 1 = stage edges in shared memory
};

template <class R> __device__ __forceinline__ V3<R> face_normal(unsigned f)
{
    const R h = R(0.5), s = R(kSqrt3 / 2);
    switch (f) {
    case 0: return v3(R(1), R(0), R(0));
    case 1: return v3(h, R(0), s);
    case 2: return v3(-h, R(0), s);
    case 3: return v3(R(-1), R(0), R(0));
    case 4: return v3(-h, R(0), -s);
    case 5: return v3(h, R(0), -s);
    case 6: return v3(R(0), R(1), R(0));
    default: return v3(R(0), R(-1), R(0));
    }
}
template <class R> __device__ __forceinline__ V3<R> hex_vertex(unsigned f)
{
    const R s = R(kSqrt3 / 2);
    switch (f % 6u) {
    case 0: return v3(s, R(0), R(0.5));
    case 1: return v3(R(0), R(0), R(1));
    case 2: return v3(-s, R(0), R(0.5));
    case 3: return v3(-s, R(0), R(-0.5));
    case 4: return v3(R(0), R(0), R(-1));
    default: return v3(s, R(0), R(-0.5));
    }
}
template <class R> __device__ __forceinline__ R face_offset(const HexGeo<R>& P, unsigned f)
{
    return f < 6u ? R(kSqrt3 / 2) : P.half_len;
}

// hex_prism.hpp:54-57 / 108-120 (FP64 path only): every other face strictly outside tolerance.
__device__ __forceinline__ bool strict_face_point(const HexGeo<double>& P, V3<double> p, unsigned face)
{
    const double tol = 128 * Eps<double>::eps * fmax(1.0, fmax(P.half_len, fmax(fabs(p.x), fmax(fabs(p.y), fabs(p.z)))));
    for (unsigned f = 0; f < 8; ++f) {
        const double gap = face_offset(P, f) - dot(face_normal<double>(f), p);
        if (f == face) {
            if (fabs(gap) > tol) return false;
        } else if (!(gap > tol)) return false;
    }
    return true;
}

struct Boundary {
    unsigned face;
    int status; // 0 regular, 3 ambiguous, 5 numerical
    bool near_edge;
};

// Nearest exit plane of the convex prism from a point on `start` (hex_prism.hpp:123-147).
// FP32: exit t = min over forward-facing planes (no positivity filter, so a point rounded
// just outside a neighbouring plane exits there at t = 0); near ties are counted only.
// FP64: the reference rules, ties within geometry tolerance are ambiguous.
template <class R>
__device__ __forceinline__ Boundary next_boundary(const HexGeo<R>& P, V3<R>& p, V3<R> d, unsigned start, R& t_out)
{
    Boundary out{8u, 0, false};
    R best = R(3.0e38), second = R(3.0e38);
    if constexpr (sizeof(R) == 8) {
        best = 1.7976931348623157e308;
        second = best;
        if (!strict_face_point(P, p, start)) { out.status = 3; return out; }
        if (dot(face_normal<R>(start), d) > 128 * Eps<double>::eps) { out.status = 5; return out; }
    }
#pragma unroll
    for (unsigned f = 0; f < 8; ++f) {
        if (f == start) continue;
        const V3<R> n = face_normal<R>(f);
        const R c = dot(n, d);
        if (!(c > R(0))) continue;
        const R t = (face_offset(P, f) - dot(n, p)) / c;
        if constexpr (sizeof(R) == 8) {
            if (!(t > 0) || !finite_r(t)) continue;
        }
        if (t < best) { second = best; best = t; out.face = f; }
        else if (t < second) second = t;
    }
    if (out.face == 8u) { out.status = 5; return out; }
    if constexpr (sizeof(R) == 4) {
        const R t = rmax(best, R(0));
        p = p + d * t;
        out.near_edge = (second - best) <= R(64) * Eps<float>::eps * rmax(R(1), P.half_len);
        t_out = t;
    } else {
        p = p + d * best;
        t_out = best;
        const double tol = 128 * Eps<double>::eps * fmax(1.0, fmax(P.half_len, fmax(fmax(fabs(p.x), fmax(fabs(p.y), fabs(p.z))), fabs(best))));
        if (second - best <= tol || !strict_face_point(P, p, out.face)) out.status = 3;
    }
    return out;
}

// Entry of a fresh ray: point on the particle and the outward normal there.
// Returns 0, ICP_RAY_AMBIGUOUS (3), or -1 when the sampled ray misses the particle.
template <class R>
__device__ __forceinline__ int geo_entry(const HexGeo<R>& G, uint64_t seed, uint64_t id, V3<R>& pos, V3<R>& n,
                                         unsigned& face)
{
    // face in proportion to projected area, point on the face (hex_prism.hpp:64-98)
    const R u0 = uniform<R>(rng_bits(seed, id, 0));
    const R u1 = uniform<R>(rng_bits(seed, id, 1));
    const R u2 = uniform<R>(rng_bits(seed, id, 2));
    const R target = u0 * G.area;
    unsigned f8 = 8u, last = 8u;
#pragma unroll
    for (unsigned f = 0; f < 8; ++f) {
        if ((G.face_mask >> f) & 1u) {
            last = f;
            if (f8 == 8u && target < G.cum[f]) f8 = f;
        }
    }
    if (f8 == 8u) f8 = last;
    face = f8;
    n = face_normal<R>(f8);
    if (f8 < 6u) {
        const V3<R> tangent = v3(-n.z, R(0), n.x);
        pos = (n * R(kSqrt3 / 2) + tangent * (u1 - R(0.5))) + v3(R(0), (R(2) * u2 - R(1)) * G.half_len, R(0));
    } else {
        const R sector = R(6) * u1;
        const unsigned j = (unsigned)sector;
        const R r = sqrt_r(sector - (R)j);
        pos = (hex_vertex<R>(j) * (R(1) - u2) + hex_vertex<R>(j + 1u) * u2) * r;
        pos.y = (f8 == 6u ? R(1) : R(-1)) * G.half_len;
    }
    if constexpr (sizeof(R) == 8) {
        if (!strict_face_point(G, pos, f8)) return 3;
    }
    return 0;
}
// Next exit point of an interior ray: advances p, returns 0 / 3 / 5 and the outward normal.
template <class R>
__device__ __forceinline__ int geo_next(const HexGeo<R>& G, V3<R>& p, V3<R> d, unsigned& face, V3<R>& n, bool& near_edge)
{
    R t;
    const Boundary hit = next_boundary(G, p, d, face, t);
    near_edge = hit.near_edge;
    if (hit.status) return hit.status;
    face = hit.face;
    n = face_normal<R>(hit.face);
    return 0;
}

// Drop: uniform point on the sampling disk (radius^2 uniform, angle uniform) a distance `back`
// before the centre; the reference's drops use a deterministic vertex grid instead
// (raindrop_paths.hpp:52-58), so the counter RNG of the prism path is reused here.
template <class R>
__device__ __forceinline__ V3<R> drop_origin(const DropGeo<R>& G, const V3<R>& k, const V3<R>& e0, uint64_t seed,
                                             uint64_t id)
{
    const R u0 = uniform<R>(rng_bits(seed, id, 0));
    const R u1 = uniform<R>(rng_bits(seed, id, 1));
    const R rad = G.disk * sqrt_r(u0);
    R sn, cs;
    if constexpr (sizeof(R) == 4) sincospif(R(2) * u1, &sn, &cs);
    else sincospi(R(2) * u1, &sn, &cs);
    return (e0 * (rad * cs) + G.e1 * (rad * sn)) - k * G.back;
}

template <class R> struct LaneRay {
    V3<R> p, d, e;
    Stokes<R> S;
    uint64_t id;
    R esc;                       // binary64 path: escaped power of this ray
    unsigned long long pfx, escfx; // binary32 path: power of the continuing branch and escaped
                                   // power, exact integers in units of 2^-44 of one ray
    uint32_t face, hits;
    bool live;
};

// Per-lane accumulators of what changes every step or every ray, summed per warp when a block (or
// a batch chunk) ends.  The power sums are exact 64-bit fixed-point integers; the counts are
// 32-bit: a
// lane traces at most lane_rays_max(max_hits) rays between flushes (the launchers cut launches
// and chunks to that), so that none of them can wrap.
template <class R> struct LaneAcc {
    unsigned long long esc_fx, unres_fx, fwd_fx, bwd_fx;
    uint32_t outputs, fallback, encounters, gauge_evals, snapped, near_edge;
    double axial;
    R max_iface;
    uint64_t cur_batch;
    uint32_t cur_batch_out;
};

// Per-warp tally in shared memory of what changes once per ray or more rarely (the rays per
// status, misses, rejections, invalid exits, the largest energy residual and, for the drop, the
// unresolved and pole powers), added with shared atomics.  Kept out of the lanes' registers, which
// the FP32 kernels need for the ray state at 64 registers; without them the drop kernel's spills
// halve and its DRAM traffic falls from 130 MB to 17 MB per 1e8-ray launch.  The warp's ray count
// is the status counts plus the misses; its power sums stay below 2^60 (lane_rays_max).  The
// prism keeps snapped exits, near-edge hits and the power sums per lane: its symmetric directions
// make them frequent (forward exits through parallel faces), and contended 64-bit shared atomics
// cost it 7 %.
struct Tally {
    unsigned status[8];
    unsigned missed, rejected, invalid, pad;
    unsigned long long unres_fx, fwd_fx, bwd_fx, max_bal_bits;
};
constexpr uint32_t kTallyWarps = 8; // blocks of 64..256 threads
constexpr size_t kTallyBytes = 80;
// whether a trace's power sums go to the tally (the drop) or stay per lane (the prism)
template <class P_> __host__ __device__ constexpr bool power_in_tally()
{
    return !std::is_same_v<std::remove_cv_t<decltype(P_::geo)>, HexGeo<std::remove_cv_t<decltype(P_::tail)>>>;
}
static_assert(sizeof(Tally) == kTallyBytes, "tally layout");
// Byte offset of the tallies in the trace kernel's shared memory (after the histogram table's
// values and keys, 16-byte aligned); the u edges follow the kTallyWarps tallies.
__host__ __device__ constexpr size_t trace_tally_offset(uint32_t hash_slots)
{
    return ((size_t)hash_slots * 12u + 15u) / 16u * 16u;
}

template <class R, class P_>
__device__ __forceinline__ void finish_ray(const P_& P, LaneRay<R>& L, LaneAcc<R>& A, Tally* T, int status,
                                           unsigned long long residual_fx, R residual)
{
    L.live = false;
    double bal;
    if constexpr (sizeof(R) == 4) {
        // escaped + residual is one ray's power exactly unless a branch was lost
        constexpr unsigned long long one = 1ull << kFixBits;
        const unsigned long long total = L.escfx + residual_fx;
        bal = (total >= one ? (double)(total - one) : (double)(one - total)) * kFixUnit;
    } else {
        bal = fabs((double)L.esc + (double)residual - 1.0);
    }
    if constexpr (power_in_tally<P_>()) {
        if (residual_fx) atomicAdd(&T->unres_fx, residual_fx);
    } else {
        A.unres_fx += residual_fx;
    }
    if (bal > 0.0) atomicMax(&T->max_bal_bits, (unsigned long long)__double_as_longlong(bal));
    atomicAdd(&T->status[status], 1u);
    const bool ok = (status == 0 || status == 1) && bal <= P.bal_tol;
    if (!ok) atomicAdd(&T->rejected, 1u);
}

// Ends the ray if the continuing branch is exhausted / below the tail / out of encounters
// (the top-of-loop and after-loop tests of hex_trace_core.hpp:217-251, applied eagerly).
template <class R, class P_>
__device__ __forceinline__ void settle(const P_& P, LaneRay<R>& L, LaneAcc<R>& A, Tally* T)
{
    if constexpr (sizeof(R) == 4) {
        const unsigned long long p = L.pfx;
        if (p == 0ull) finish_ray<R>(P, L, A, T, 0, 0ull, R(0));
        else if (p <= P.tail_fx) finish_ray<R>(P, L, A, T, 1, p, R(0));
        else if (L.hits >= P.max_hits) finish_ray<R>(P, L, A, T, 2, p, R(0));
    } else {
        const R power = L.S.I;
        if (power == R(0)) finish_ray<R>(P, L, A, T, 0, 0ull, R(0));
        else if (power <= P.tail) finish_ray<R>(P, L, A, T, 1, to_fix(power), power);
        else if (L.hits >= P.max_hits) finish_ray<R>(P, L, A, T, 2, to_fix(power), power);
    }
}

// Per-block shared state: the privatised histogram table, this warp's tally and (optionally) the
// u edges.
template <class R> struct BlockShared {
    SmemHist H;
    Tally* T;
    const R* edges;
};

template <class R, class P_>
__device__ __forceinline__ BlockShared<R> block_setup(const P_& P, unsigned char* smem)
{
    BlockShared<R> B;
    unsigned long long* s_vals = reinterpret_cast<unsigned long long*>(smem);
    uint32_t* s_keys = reinterpret_cast<uint32_t*>(s_vals + P.hash_slots);
    Tally* tallies = reinterpret_cast<Tally*>(smem + trace_tally_offset(P.hash_slots));
    B.T = tallies + (threadIdx.x >> 5);
    R* s_edges = reinterpret_cast<R*>(tallies + kTallyWarps);
    const uint32_t nt = P.gf.nt;
    for (uint32_t s = threadIdx.x; s < P.hash_slots; s += blockDim.x) { s_keys[s] = 0u; s_vals[s] = 0ull; }
    for (uint32_t i = threadIdx.x; i < kTallyWarps * kTallyBytes / 4; i += blockDim.x)
        reinterpret_cast<unsigned*>(tallies)[i] = 0u;
    if (P.smem_edges) {
        for (uint32_t i = threadIdx.x; i <= nt; i += blockDim.x) {
            if constexpr (sizeof(R) == 4) s_edges[i] = P.edges_f[i];
            else s_edges[i] = P.edges_d[i];
        }
        B.edges = s_edges;
    } else {
        if constexpr (sizeof(R) == 4) B.edges = P.edges_f;
        else B.edges = P.edges_d;
    }
    B.H = SmemHist{s_keys, s_vals, P.hash_slots ? P.hash_slots - 1u : 0u};
    return B;
}

template <class R> __device__ __forceinline__ void lane_acc_clear(LaneAcc<R>& A)
{
    A.esc_fx = A.unres_fx = A.fwd_fx = A.bwd_fx = 0ull;
    A.outputs = A.fallback = A.encounters = A.gauge_evals = A.snapped = A.near_edge = 0u;
    A.axial = 0.0;
    A.max_iface = R(0);
    A.cur_batch = ~0ull;
    A.cur_batch_out = 0u;
}

// The rays [wnext, wend) of one warp: persistent lanes, one event per lane per step, every
// exit binned by the whole warp (hex_trace_core.hpp:190-259 per ray).
template <class R, class G, class P_>
__device__ __forceinline__ void trace_slice(const P_& P, const BlockShared<R>& B, uint64_t wnext, const uint64_t wend,
                                            LaneAcc<R>& A)
{
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;
    Tally* T = B.T;
    LaneRay<R> L;
    L.live = false;
    while (true) {
        // ---- refill idle lanes from the warp's slice
        const unsigned idle = __ballot_sync(kFull, !L.live);
        bool fresh = false;
        if (idle) {
            if (!L.live) {
                const uint64_t id = wnext + __popc(idle & lt_mask);
                if (id < wend) { L.id = id; fresh = true; }
            }
            wnext += __popc(idle);
        }
        if (!__any_sync(kFull, L.live || fresh)) break;

        bool has = false;
        V3<R> od;
        R opow = R(0);
        unsigned long long efx = 0ull; // fixed-point power of this step's exit
        // ---- gather the inputs of this step's interface: the entry face of a fresh ray,
        // or the next exit plane of a live one (one shared split per lane per step)
        bool do_split = false;
        V3<R> sd, se, sn;
        Stokes<R> sS;
        const Media<R>* media = &P.enter;
        if constexpr (!std::is_same_v<G, HexGeo<R>>) {
            // drop: every active lane runs one intersection -- entering from its sampling-disk
            // origin (fresh) or leaving from its current surface point (live)
            V3<R> q, w, n;
            if (fresh) {
                q = drop_origin(P.geo, P.k, P.ke0, P.seed, L.id);
                w = P.k;
            } else {
                q = L.p;
                w = L.d;
            }
            bool hit = false;
            if (fresh || L.live) {
                R t;
                hit = drop_intersect(P.geo.shape, q, w, fresh, t, A.gauge_evals);
                q = q + w * t;
                if (hit) n = drop_normal(P.geo.shape, q);
            }
            if (fresh) {
                if (!hit) {
                    // a sampled ray that misses the particle carries no incident power
                    atomicAdd(&T->missed, 1u);
                } else {
                    L.live = true;
                    L.esc = R(0);
                    L.pfx = 1ull << kFixBits;
                    L.escfx = 0ull;
                    L.hits = 0u;
                    L.p = q;
                    L.face = 0u;
                    do_split = true;
                    sd = P.k;
                    se = P.ke0;
                    sS = Stokes<R>{R(1), R(0), R(0), R(0)};
                    sn = n;
                    media = &P.enter;
                }
            } else if (L.live) {
                // one internal encounter (hex_trace_core.hpp:217-246)
                L.p = q;
                ++L.hits;
                ++A.encounters;
                do_split = true;
                sd = L.d;
                se = L.e;
                sS = L.S;
                sn = -n;
                media = &P.leave;
            }
        } else if (fresh) {
            V3<R> pos, n;
            unsigned face = 8u;
            const int es = geo_entry(P.geo, P.seed, L.id, pos, n, face);
            if (es < 0) {
                // a sampled ray that misses the particle carries no incident power
                atomicAdd(&T->missed, 1u);
            } else {
                L.live = true;
                L.esc = R(0);
                L.pfx = 1ull << kFixBits;
                L.escfx = 0ull;
                L.hits = 0u;
                L.p = pos;
                L.face = face;
                do_split = true;
                if (es) {
                    finish_ray<R>(P, L, A, T, es, 1ull << kFixBits, R(1));
                    do_split = false;
                }
                sd = P.k;
                se = P.ke0;
                sS = Stokes<R>{R(1), R(0), R(0), R(0)};
                sn = n;
                media = &P.enter;
            }
        } else if (L.live) {
            // one internal encounter (hex_trace_core.hpp:217-246)
            V3<R> n;
            bool near_edge = false;
            const int hs = geo_next(P.geo, L.p, L.d, L.face, n, near_edge);
            if (hs) {
                finish_ray<R>(P, L, A, T, hs, sizeof(R) == 4 ? L.pfx : to_fix(L.S.I), L.S.I);
            } else {
                A.near_edge += near_edge ? 1u : 0u;
                ++L.hits;
                ++A.encounters;
                do_split = true;
                sd = L.d;
                se = L.e;
                sS = L.S;
                sn = -n;
                media = &P.leave;
            }
        }
        if (do_split) {
            const Interface<R> sp = split(sd, se, sS, sn, *media);
            A.max_iface = rmax(A.max_iface, sp.balance);
            // entry: exterior reflection exits, transmission continues;
            // internal: transmission exits, reflection continues
            unsigned long long cont_fx = 0ull;
            if constexpr (sizeof(R) == 4) {
                // the reflected share is rounded once, the transmitted share is the exact rest
                const unsigned long long rq = to_fix(sp.r.I);
                const unsigned long long rfx = (sp.tir || rq > L.pfx) ? L.pfx : rq;
                const unsigned long long tfx = L.pfx - rfx;
                efx = fresh ? rfx : tfx;
                cont_fx = fresh ? tfx : rfx;
                if (efx) {
                    has = true;
                    od = fresh ? sp.dr : sp.dt;
                    opow = (R)efx * R(kFixUnit);
                    L.escfx += efx;
                }
            } else {
                const R epow = fresh ? sp.r.I : (sp.has_t ? sp.t.I : R(0));
                if (epow > R(0)) {
                    has = true;
                    od = fresh ? sp.dr : sp.dt;
                    opow = epow;
                    efx = to_fix(epow);
                    L.esc += opow;
                }
            }
            if (fresh && !sp.has_t) {
                finish_ray<R>(P, L, A, T, 0, 0ull, R(0));
            } else {
                L.d = fresh ? sp.dt : sp.dr;
                L.e = sp.s;
                L.S = fresh ? sp.t : sp.r;
                if constexpr (sizeof(R) == 4) {
                    L.pfx = cont_fx;
                    L.S.I = (R)cont_fx * R(kFixUnit);
                }
                settle<R>(P, L, A, T);
            }
        }

        // ---- bin this step's exits (whole warp)
        uint32_t cell = 0u;
        bool to_table = false;
        uint64_t v = 0ull;
        if (has) {
            BinResult b;
            if constexpr (sizeof(R) == 4) b = bin_f32(P.gf, B.edges, od);
            else b = bin_f64(P.gd, B.edges, od);
            if (!b.valid) {
                atomicAdd(&T->invalid, 1u);
            } else {
                v = efx;
                A.esc_fx += v;
                A.outputs += 1;
                A.snapped += b.snapped ? 1u : 0u;
                A.axial += (double)opow * b.mu;
                if (b.pole > 0) {
                    if constexpr (power_in_tally<P_>()) atomicAdd(&T->fwd_fx, (unsigned long long)v);
                    else A.fwd_fx += v;
                } else if (b.pole < 0) {
                    if constexpr (power_in_tally<P_>()) atomicAdd(&T->bwd_fx, (unsigned long long)v);
                    else A.bwd_fx += v;
                } else {
                    to_table = true;
                    cell = b.cell;
                }
            }
        }
        hist_add(B.H, P.mass, P.to_mass, to_table, cell, v, A.fallback);

        // ---- per-batch exit counts (the prism's capacity audit), flushed when the lane's batch
        // changes
        if constexpr (std::is_same_v<G, HexGeo<R>>) {
            if (P.batch_out && (has || fresh)) {
                const uint64_t bidx = L.id / P.batch_size;
                if (bidx != A.cur_batch) {
                    if (A.cur_batch != ~0ull && A.cur_batch_out) atomicAdd(&P.batch_out[A.cur_batch], A.cur_batch_out);
                    A.cur_batch = bidx;
                    A.cur_batch_out = 0u;
                }
                A.cur_batch_out += has ? 1u : 0u;
            }
        }
    }
    if constexpr (std::is_same_v<G, HexGeo<R>>)
        if (P.batch_out && A.cur_batch != ~0ull && A.cur_batch_out) atomicAdd(&P.batch_out[A.cur_batch], A.cur_batch_out);
}

// The warp's sums into the record's statistics: its lanes' accumulators (shuffled) and its tally
// (lane 0 adds, then clears the tally).  Called by whole warps after the lanes' last update.
template <class R>
__device__ __forceinline__ void warp_stats_flush(DevStats* Gs, const LaneAcc<R>& A, Tally* T)
{
    unsigned long long w[10] = {A.esc_fx, A.outputs, A.fallback, A.encounters, A.gauge_evals, A.snapped, A.near_edge,
                                A.unres_fx, A.fwd_fx, A.bwd_fx};
#pragma unroll
    for (int q = 0; q < 10; ++q)
        for (int o = 16; o; o >>= 1) w[q] += __shfl_xor_sync(kFull, w[q], o);
    double ax = A.axial, mi = (double)A.max_iface;
    for (int o = 16; o; o >>= 1) {
        ax += __shfl_xor_sync(kFull, ax, o);
        mi = fmax(mi, __shfl_xor_sync(kFull, mi, o));
    }
    __syncwarp();
    if ((threadIdx.x & 31u) == 0) {
        add128(Gs->esc, w[0]);
        // one of each pair is zero: the sums sit per lane (the prism) or in the tally (the drop)
        add128(Gs->unres, w[7] + T->unres_fx);
        add128(Gs->fwd, w[8] + T->fwd_fx);
        add128(Gs->bwd, w[9] + T->bwd_fx);
        unsigned long long rays = T->missed;
#pragma unroll
        for (int s = 0; s < 8; ++s) {
            rays += T->status[s];
            if (T->status[s]) atomicAdd(&Gs->status[s], (unsigned long long)T->status[s]);
        }
        const unsigned long long c[10] = {rays, w[1], T->rejected, w[5], w[6], w[2], T->invalid, w[3], T->missed, w[4]};
        unsigned long long* counters[10] = {&Gs->rays, &Gs->outputs, &Gs->rejected, &Gs->snapped, &Gs->near_edge,
                                            &Gs->fallback, &Gs->invalid, &Gs->encounters, &Gs->missed, &Gs->gauge_evals};
#pragma unroll
        for (int q = 0; q < 10; ++q)
            if (c[q]) atomicAdd(counters[q], c[q]);
        if (ax != 0.0) atomicAdd(&Gs->axial, ax);
        atomicMax(&Gs->max_bal_bits, T->max_bal_bits);
        atomicMax(&Gs->max_iface_bits, (unsigned long long)__double_as_longlong(mi));
        *T = Tally{};
    }
    __syncwarp();
}

// Block epilogue (all threads): flush the table into P.mass and every warp's sums into P.stats;
// leaves the table and the tallies cleared.
template <class R, class P_>
__device__ __forceinline__ void block_flush(const P_& P, const BlockShared<R>& B, const LaneAcc<R>& A)
{
    __syncthreads();
    hist_flush(B.H, P.mass, P.to_mass);
    warp_stats_flush<R>(P.stats, A, B.T);
}

// Block shape of the single-record trace: the FP32 drop runs 128-thread blocks, seven per SM at
// 72 registers (fewer spills than four 256-thread blocks at 64 registers: 1 % faster); the FP32
// prism keeps four 256-thread blocks (its 48 KB shared histogram table per block), the FP64
// kernels 256 threads.
template <class R, class G> struct TraceShape {
    static constexpr bool drop32 = sizeof(R) == 4 && !std::is_same_v<G, HexGeo<R>>;
    static constexpr unsigned threads = drop32 ? 128u : 256u;
    static constexpr unsigned min_blocks = sizeof(R) == 4 ? (drop32 ? 7u : 4u) : 1u;
};

// One record: the ray range [first, first+count) split into contiguous per-warp slices.
template <class R, class G>
__global__ void __launch_bounds__(TraceShape<R, G>::threads, TraceShape<R, G>::min_blocks)
    trace_bin_kernel(const TraceParams<R, G> P)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const BlockShared<R> B = block_setup<R>(P, smem);
    __syncthreads();
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const uint64_t warp = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint64_t per = (P.count + warps - 1) / warps;
    const uint64_t wnext = P.first + warp * per;
    const uint64_t wend = min(P.first + P.count, wnext + per);
    LaneAcc<R> A;
    lane_acc_clear(A);
    trace_slice<R, G>(P, B, wnext, wend, A);
    block_flush<R>(P, B, A);
}

} // namespace icp
