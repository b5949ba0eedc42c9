// icp_device.cuh -- device math shared by the trace+bin kernels (sm_100a).
//
// Real = float  : the fast path (FP32 SIMT, FMA contraction allowed, FP32-aware tolerances).
// Real = double : the reference-tolerance path, compiled in its own translation unit with
//                 -fmad=false so that the direction arithmetic follows the reference's
//                 operation order (hex_trace/include/ice_crystal/math.hpp:23-69).
//
// Polarisation is carried as the Stokes vector (I,Q,U,V) of an unpolarised unit input in
// the ray's transverse frame (e, d x e).  This is the first column of the Mueller matrix of
// the reference's two-column Jones response (math.hpp:79-109): the reference's power
// 0.5*sum|J|^2 is exactly I, and the Mueller matrices of the frame rotation and of the
// Fresnel s/p scaling compose like the Jones operations they represent.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace icp {

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kSqrt3 = 1.732050807568877293527446341505872367;
constexpr unsigned kFull = 0xffffffffu;

template <class R> struct V3 { R x, y, z; };

template <class R> __host__ __device__ __forceinline__ V3<R> v3(R x, R y, R z) { return {x, y, z}; }
template <class R> __host__ __device__ __forceinline__ V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> __host__ __device__ __forceinline__ V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> __host__ __device__ __forceinline__ V3<R> operator-(V3<R> a) { return {-a.x, -a.y, -a.z}; }
template <class R> __host__ __device__ __forceinline__ V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> __host__ __device__ __forceinline__ V3<R> operator/(V3<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <class R> __host__ __device__ __forceinline__ R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> __host__ __device__ __forceinline__ V3<R> cross(V3<R> a, V3<R> b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> __host__ __device__ __forceinline__ R rabs(R x) { return x < R(0) ? -x : x; }
template <class R> __host__ __device__ __forceinline__ R rmax(R a, R b) { return a > b ? a : b; }
template <class R> __host__ __device__ __forceinline__ R rmin(R a, R b) { return a < b ? a : b; }
__device__ __forceinline__ float rsqrt_r(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_r(double x) { return 1.0 / sqrt(x); }
__device__ __forceinline__ float sqrt_r(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_r(double x) { return sqrt(x); }

template <class R> struct Eps;
template <> struct Eps<float> {
    static constexpr float eps = 1.1920928955078125e-07f;
};
template <> struct Eps<double> {
    static constexpr double eps = 2.220446049250313080847e-16;
};

template <class R> __device__ __forceinline__ bool finite_r(R x)
{
    return x == x && rabs(x) <= (sizeof(R) == 4 ? R(3.4028234663852886e38) : R(1.7976931348623157e308));
}

// Unit vector.  FP64: the reference's scale-then-normalise (math.hpp:38-47) so that exit
// directions, and hence bins, follow the reference bit pattern where the inputs agree.
// FP32: one reciprocal square root.
__device__ __forceinline__ V3<float> unit(V3<float> a) { return a * rsqrtf(dot(a, a)); }
__device__ __forceinline__ V3<double> unit(V3<double> a)
{
    const double s = fmax(fabs(a.x), fmax(fabs(a.y), fabs(a.z)));
    a = a / s;
    const double n = sqrt(dot(a, a));
    return a / n;
}

// |d x n| as the reference evaluates it (flux_interface.hpp:42-45): scaled by the largest
// component in FP64 so that the refraction cosine, and the exit direction, round identically.
__device__ __forceinline__ float sine_of(V3<float> s) { return sqrtf(dot(s, s)); }
__device__ __forceinline__ double sine_of(V3<double> s)
{
    const double scale = fmax(fabs(s.x), fmax(fabs(s.y), fabs(s.z)));
    if (!(scale > 0)) return 0.0;
    const V3<double> t = s / scale;
    return scale * sqrt(dot(t, t));
}

// ---------------------------------------------------------------- counter RNG
// SplitMix64 finaliser over seed + golden * (3*id + dim + 1) (math.hpp:136-146).
__device__ __forceinline__ uint64_t mix64(uint64_t x)
{
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}
__device__ __forceinline__ uint64_t rng_bits(uint64_t seed, uint64_t id, unsigned dim)
{
    return mix64(seed + 0x9e3779b97f4a7c15ull * (3ull * id + dim + 1ull));
}
// Midpoints of 2^52 cells (the reference's draw, exact in binary64).
__device__ __forceinline__ double uniform_f64(uint64_t bits) { return (double(bits >> 12) + 0.5) * 0x1p-52; }
// FP32 path: the same 64-bit draw rounded to float (round-to-nearest of the 52-bit midpoint,
// kept strictly below 1).
__device__ __forceinline__ float uniform_f32(uint64_t bits)
{
    const float u = __double2float_rn(uniform_f64(bits));
    return u < 1.0f ? u : 0.99999994f;
}
template <class R> __device__ __forceinline__ R uniform(uint64_t bits);
template <> __device__ __forceinline__ float uniform<float>(uint64_t b) { return uniform_f32(b); }
template <> __device__ __forceinline__ double uniform<double>(uint64_t b) { return uniform_f64(b); }

// ---------------------------------------------------------------- Stokes
template <class R> struct Stokes { R I, Q, U, V; };

// Result of one dielectric interface for the branch-independent part.
template <class R> struct Interface {
    V3<R> s;        // s-polarisation unit vector (new frame e0 of both branches)
    V3<R> dr, dt;   // reflected / transmitted directions
    Stokes<R> r, t; // branch Stokes vectors
    R ci;           // cosine of incidence
    bool has_t, tir;
    R balance;      // relative power imbalance of this split
};

// Refraction constants of one oriented interface (incident index ni -> transmitted nt),
// normalised by the larger index as the reference does (flux_interface.hpp:51).
template <class R> struct Media {
    R a, b, eta; // ni/max, nt/max, a/b
    bool matched; // ni == nt: the ray passes unchanged (flux_interface.hpp:34-41)
};
template <class R> __host__ __device__ inline Media<R> make_media(double ni, double nt)
{
    const double ns = ni > nt ? ni : nt, a = ni / ns, b = nt / ns;
    return Media<R>{R(a), R(b), R(a / b), ni == nt};
}

// Fresnel split in flux normalisation (flux_interface.hpp:26-88).  n points into the incident
// medium.  `e` is the ray's current frame vector.  The transmitted flux is 1 - R for each of
// s and p, so power is conserved to one rounding per interface; its Mueller off-diagonal
// term is sqrt(Ts*Tp) = ts*tp.  Partial reflection and total internal reflection are both
// evaluated and selected per lane (no divergent branch between them).
template <class R>
__device__ __forceinline__ Interface<R> split(V3<R> d, V3<R> e, Stokes<R> S, V3<R> n, const Media<R>& M)
{
    Interface<R> out;
    if (M.matched) {
        out.s = e;
        out.dt = d;
        out.t = S;
        out.dr = unit(d - n * (R(2) * dot(d, n)));
        out.r = {R(0), R(0), R(0), R(0)};
        out.ci = -dot(d, n);
        out.has_t = true;
        out.tir = false;
        out.balance = R(0);
        return out;
    }
    R ci = -dot(d, n);
    ci = rmin(R(1), rmax(R(0), ci));
    V3<R> s = cross(d, n);
    const R sine = sine_of(s);
    if (sine > R(0)) s = unit(s);
    else s = e;
    out.s = s;
    // Basis rotation (e, d x e) -> (s, d x s): c = e.s, sg = (d x e).s
    const R c = dot(e, s);
    const R sg = dot(cross(d, e), s);
    const R cos2 = c * c - sg * sg, sin2p = R(2) * c * sg;
    const R Q = cos2 * S.Q + sin2p * S.U;
    const R U = -sin2p * S.Q + cos2 * S.U;
    const R a = M.a, b = M.b;
    const R st = M.eta * sine;
    out.dr = unit(d + n * (R(2) * ci));
    out.ci = ci;
    const bool tir = st > R(1);
    R Rs, Rp, zr, zi, ct;
    if constexpr (sizeof(R) == 8) {
        // reference arithmetic (flux_interface.hpp:59-79)
        if (tir) {
            const R inv = R(1) / st;
            const R beta = st * sqrt_r((R(1) - inv) * (R(1) + inv));
            R x1 = a * ci, y1 = b * beta, x2 = b * ci, y2 = a * beta;
            const R s1 = rmax(rabs(x1), rabs(y1)), s2 = rmax(rabs(x2), rabs(y2));
            x1 /= s1; y1 /= s1; x2 /= s2; y2 /= s2;
            const R d1 = x1 * x1 + y1 * y1, d2 = x2 * x2 + y2 * y2;
            const R rsr = (x1 * x1 - y1 * y1) / d1, rsi = (R(-2) * x1 * y1) / d1;
            const R rpr = (x2 * x2 - y2 * y2) / d2, rpi = (R(-2) * x2 * y2) / d2;
            Rs = R(1);
            Rp = R(1);
            zr = rsr * rpr + rsi * rpi; // rs * conj(rp)
            zi = rsi * rpr - rsr * rpi;
            ct = R(0);
        } else {
            ct = sqrt_r((R(1) - st) * (R(1) + st));
            const R ds = a * ci + b * ct, dp = b * ci + a * ct;
            const R rs = (a * ci - b * ct) / ds, rp = (b * ci - a * ct) / dp;
            Rs = rs * rs;
            Rp = rp * rp;
            zr = rs * rp;
            zi = R(0);
        }
    } else {
        // binary32: both branches, selected per lane
        const R k2 = (R(1) - st) * (R(1) + st);
        ct = sqrt_r(rmax(k2, R(0)));
        const R beta = sqrt_r(rmax(-k2, R(0)));
        // partial reflection
        const R ds = a * ci + b * ct, dp = b * ci + a * ct;
        const R rs = (a * ci - b * ct) / ds, rp = (b * ci - a * ct) / dp;
        // total internal reflection: rs = (x1 - i y1)/(x1 + i y1), rp = (x2 - i y2)/(x2 + i y2)
        const R x1 = a * ci, y1 = b * beta, x2 = b * ci, y2 = a * beta;
        const R i1 = R(1) / (x1 * x1 + y1 * y1), i2 = R(1) / (x2 * x2 + y2 * y2);
        const R rsr = (x1 * x1 - y1 * y1) * i1, rsi = (R(-2) * x1 * y1) * i1;
        const R rpr = (x2 * x2 - y2 * y2) * i2, rpi = (R(-2) * x2 * y2) * i2;
        Rs = tir ? R(1) : rs * rs;
        Rp = tir ? R(1) : rp * rp;
        zr = tir ? rsr * rpr + rsi * rpi : rs * rp;
        zi = tir ? rsi * rpr - rsr * rpi : R(0);
    }
    out.tir = tir;
    out.has_t = !tir;
    const R hs = R(0.5) * (Rs + Rp), hd = R(0.5) * (Rs - Rp);
    out.r.I = hs * S.I + hd * Q;
    out.r.Q = hd * S.I + hs * Q;
    out.r.U = zr * U - zi * S.V;
    out.r.V = zi * U + zr * S.V;
    if (!tir) {
        out.dt = unit((d + n * ci) * M.eta - n * ct);
        const R zt = sqrt_r((R(1) - Rs) * (R(1) - Rp));
        out.t.I = S.I - out.r.I;
        out.t.Q = Q - out.r.Q;
        out.t.U = zt * U;
        out.t.V = zt * S.V;
        out.balance = S.I > R(0) ? rabs(out.r.I + out.t.I - S.I) / S.I : R(0);
    } else {
        out.dt = d;
        out.t = {R(0), R(0), R(0), R(0)};
        out.balance = S.I > R(0) ? rabs(out.r.I - S.I) / S.I : R(0);
    }
    return out;
}

// ------------------------------------------------------- fixed-point power units
// Exit powers are accumulated as unsigned 64-bit integers in units of 2^-44 of the
// incident power of one ray: exact, order-independent sums (no absorbed addends).
constexpr int kFixBits = 44;
__device__ __forceinline__ uint64_t to_fix(float p) { return __float2ull_rn(p * 0x1p44f); }
__device__ __forceinline__ uint64_t to_fix(double p) { return __double2ull_rn(p * 0x1p44); }
constexpr double kFixUnit = 0x1p-44;

} // namespace icp
