// icp_query.cu -- all-hit query of the drop's outgoing patches on the device (sm_100a) and
// its C ABI (include/icp_b200.h, "patch query").  Built with -fmad=false: the ray / patch
// intersection's binary32 and binary64 arithmetic is the reference's operation for operation
// (only its explicit fmaf / fma are fused; sqrt and division are correctly rounded), so hits
// are bit-identical to the reference's host build.
//
// The reference traverses an OptiX BVH over the patches' padded boxes and intersects every
// patch whose box the ray t d (0 <= t <= 4) meets (shaders/entry/patch_query.cu).  Here:
//   query_bin_*_kernel     each patch's box is bounded by a spherical cap (the cone over a
//                          convex box is the spherical hull of its corner directions); the cap
//                          is scattered into the direction bins (256 x 512 in colatitude and
//                          longitude) it overlaps: count, device scan, fill
//   query_count_kernel     one thread per direction: the candidates of its bin, the binary32
//                          slab test against each padded box, the intersection (binary32, and
//                          binary64 when binary32 is not conclusive), roots counted and the
//                          intersector's flags noted
//   query_scan_* kernels   exclusive 64-bit scan of the per-direction counts (block sums, one
//                          block over the sums, add back) -> hit offsets
//   query_fill_kernel      the same per direction, the roots written into its slots, sorted
//                          by (patch_id, compact index, root), duplicates removed and the
//                          summary counted (PatchHitCollector, patch_query_data.hpp:43-128)
// The order in which a bin lists its patches does not matter: the hits are sorted and the
// noted flags / first problem patch are order-independent.
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

constexpr unsigned kThreads = 128;
// The counting and filling passes wait on candidate gathers; six blocks per SM (80 registers, a
// few bytes of spills) keep more of them in flight than the four that 128 registers allowed:
// 3.77 -> 3.47 ms for the 513 x 513 lattice at 360 x 720 directions.
constexpr unsigned kQueryBlocksPerSm = 6;
constexpr unsigned kScanThreads = 1024;
constexpr int kBinRows = 256, kBinCols = 512;
constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kCapMargin = 1e-4; // radians added to every cap (rounding of the box test)

// query flags (PatchQueryFlags) and intersector flags (BilinearHitFlags, BilinearQueryFlags)
enum : uint32_t { qUnresolved = 1, qInvalid = 2, qMismatch = 4, qRefine = 8, qBoundary = 16, qFp64 = 32,
                  qDuplicate = 64, qSingular = 128 };
enum : uint32_t { hBoundary = 1, hSingular = 2, hFp64 = 4 };
enum : uint32_t { bUnresolved = 1, bInvalid = 2, bFp64 = 4 };

// ------------------------------------------------------------------ intersection
struct Hit {
    float u, v, t, residual;
    uint32_t flags;
};
struct Hits {
    Hit hit[2];
    uint32_t count, flags;
};
struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 f3(const icp_vec3f& v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ bool finite32(float x) { return x >= -FLT_MAX && x <= FLT_MAX; }
__device__ __forceinline__ float fdot(F3 a, F3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }

template <class T> struct Num;
template <> struct Num<float> {
    static __device__ __forceinline__ float fma_(float a, float b, float c) { return fmaf(a, b, c); }
    static __device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
    static __device__ __forceinline__ float copysign_(float x, float y) { return copysignf(x, y); }
    static constexpr float eps = 0x1p-23f;
    static constexpr bool is_float = true;
};
template <> struct Num<double> {
    static __device__ __forceinline__ double fma_(double a, double b, double c) { return fma(a, b, c); }
    static __device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
    static __device__ __forceinline__ double copysign_(double x, double y) { return copysign(x, y); }
    static constexpr double eps = 0x1p-52;
    static constexpr bool is_float = false;
};
// |x| and max as x < 0 ? -x : x and a > b ? a : b (zero signs and NaNs as the reference's)
template <class T> __device__ __forceinline__ T absv(T x) { return x < T(0) ? -x : x; }
template <class T> __device__ __forceinline__ T maxv(T a, T b) { return a > b ? a : b; }
template <class T> struct P2 {
    T x, y;
};
template <class T> struct P3 {
    T x, y, z;
};
template <class T> __device__ __forceinline__ T dop(T x, T y, T z, T w)
{
    const T zw = z * w;
    return Num<T>::fma_(x, y, -zw) + Num<T>::fma_(-z, w, zw);
}
template <class T> __device__ __forceinline__ P2<T> add(P2<T> a, P2<T> b) { return {a.x + b.x, a.y + b.y}; }
template <class T> __device__ __forceinline__ P2<T> mul(P2<T> a, T s) { return {a.x * s, a.y * s}; }
template <class T> __device__ __forceinline__ T big(P2<T> a) { return maxv(absv(a.x), absv(a.y)); }
template <class T> __device__ __forceinline__ T crs(P2<T> a, P2<T> b) { return dop(a.x, b.y, a.y, b.x); }
template <class T> __device__ __forceinline__ T comp(P3<T> p, unsigned k) { return k == 0 ? p.x : (k == 1 ? p.y : p.z); }
template <class T> __device__ __forceinline__ P3<T> sub(P3<T> a, P3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> __device__ __forceinline__ P3<T> add(P3<T> a, P3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> __device__ __forceinline__ P3<T> mul(P3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> __device__ __forceinline__ P2<T> project(P3<T> p, P3<T> w, unsigned kz)
{
    const unsigned kx = (kz + 1) % 3, ky = (kz + 2) % 3;
    const T z = comp(w, kz);
    return {dop(z, comp(p, kx), comp(w, kx), comp(p, kz)), dop(z, comp(p, ky), comp(w, ky), comp(p, kz))};
}
__device__ __forceinline__ F3 evaluate(const F3* c, float u, float v)
{
    const F3 lo = {c[0].x * (1.0f - u) + c[1].x * u, c[0].y * (1.0f - u) + c[1].y * u, c[0].z * (1.0f - u) + c[1].z * u};
    const F3 hi = {c[2].x * (1.0f - u) + c[3].x * u, c[2].y * (1.0f - u) + c[3].y * u, c[2].z * (1.0f - u) + c[3].z * u};
    return {lo.x * (1.0f - v) + hi.x * v, lo.y * (1.0f - v) + hi.y * v, lo.z * (1.0f - v) + hi.z * v};
}

// The ray w through the origin against the bilinear patch of the four corner directions,
// in the plane normal to w's dominant axis: a quadratic in u, then three Newton steps.
// Returns true when the result is not conclusive (the caller retries in binary64).
template <class T> __device__ bool solve(const F3* corner, F3 dir, Hits& out)
{
    bool retry = false;
    out = Hits{};
    const P3<T> w = {T(dir.x), T(dir.y), T(dir.z)};
    unsigned kz = 0;
    if (absv(w.y) > absv(w.x)) kz = 1;
    if (absv(w.z) > absv(comp(w, kz))) kz = 2;
    const P3<T> p0 = {T(corner[0].x), T(corner[0].y), T(corner[0].z)}, p1 = {T(corner[1].x), T(corner[1].y), T(corner[1].z)};
    const P3<T> p2 = {T(corner[2].x), T(corner[2].y), T(corner[2].z)}, p3 = {T(corner[3].x), T(corner[3].y), T(corner[3].z)};
    const P3<T> eu = sub(p1, p0), ev = sub(p2, p0), tw = sub(sub(p3, p2), eu);
    P2<T> a = project(p0, w, kz), b = project(eu, w, kz), c = project(ev, w, kz), d = project(tw, w, kz);
    const T scale = maxv(maxv(big(a), big(b)), maxv(big(c), big(d)));
    if (!(scale > T(0))) return true;
    a = mul(a, T(1) / scale);
    b = mul(b, T(1) / scale);
    c = mul(c, T(1) / scale);
    d = mul(d, T(1) / scale);
    const T eps = Num<T>::eps;
    const P2<T> cs[4] = {a, add(a, b), add(a, c), add(add(add(a, b), c), d)};
    T xlo = cs[0].x, xhi = xlo, ylo = cs[0].y, yhi = ylo;
    for (unsigned i = 1; i < 4; ++i) {
        xlo = xlo < cs[i].x ? xlo : cs[i].x;
        xhi = maxv(xhi, cs[i].x);
        ylo = ylo < cs[i].y ? ylo : cs[i].y;
        yhi = maxv(yhi, cs[i].y);
    }
    const T guard = T(64) * eps;
    if (xlo > guard || xhi < -guard || ylo > guard || yhi < -guard) return false;
    const T A = crs(b, d), B = crs(a, d) + crs(b, c), Cc = crs(a, c);
    const T mag = maxv(absv(A), maxv(absv(B), absv(Cc)));
    if (!(mag > T(0))) return true;
    const T qa = A / mag, qb = B / mag, qc = Cc / mag;
    if (Num<T>::is_float && A != T(0) && absv(qa) < T(64) * eps) return true;
    T roots[2] = {T(0), T(0)};
    unsigned nroot = 0;
    bool repeated = false;
    if (A == T(0)) {
        if (B == T(0)) return absv(qc) <= guard;
        roots[nroot++] = -qc / qb;
    } else {
        const T disc = dop(qb, qb, T(4) * qa, qc);
        const T err = T(64) * eps * (qb * qb + absv(T(4) * qa * qc));
        if (disc < T(0)) return disc >= -err;
        if (disc == T(0)) {
            if (Num<T>::is_float) return true;
            roots[nroot++] = -qb / (T(2) * qa);
            repeated = true;
        } else {
            if (disc <= err) return true;
            const T q = -T(0.5) * (qb + Num<T>::copysign_(Num<T>::sqrt_(disc), qb));
            roots[0] = q / qa;
            roots[1] = qc / q;
            if (roots[1] < roots[0]) {
                const T tmp = roots[0];
                roots[0] = roots[1];
                roots[1] = tmp;
            }
            nroot = 2;
        }
    }
    for (unsigned r = 0; r < nroot; ++r) {
        T u = roots[r];
        if (!(u == u)) { retry = true; continue; }
        if (u < -guard || u > T(1) + guard) continue;
        const P2<T> num = add(a, mul(b, u)), den = add(c, mul(d, u));
        if (big(den) <= guard) { retry = true; continue; }
        T v = absv(den.x) >= absv(den.y) ? -num.x / den.x : -num.y / den.y;
        if (!(v == v)) { retry = true; continue; }
        if (v < -guard || v > T(1) + guard) continue;
        T cond = T(1);
        for (unsigned it = 0; it < 3; ++it) {
            const P2<T> fu = add(b, mul(d, v)), fv = add(c, mul(d, u));
            const T det = crs(fu, fv);
            const P2<T> res = add(add(add(a, mul(b, u)), mul(c, v)), mul(d, u * v));
            if (absv(det) <= T(64) * eps * big(fu) * big(fv)) {
                if (!repeated) retry = true;
                break;
            }
            cond = maxv(T(1), maxv(big(fu), big(fv)) / absv(det));
            const T du = crs(res, fv) / det, dv = crs(fu, res) / det;
            u -= du;
            v -= dv;
        }
        const T perr = T(32) * eps * cond;
        if (Num<T>::is_float && (perr > T(2e-5) || u <= perr || u >= T(1) - perr || v <= perr || v >= T(1) - perr)) {
            retry = true;
            continue;
        }
        if (perr > T(1e-5) && !repeated) { retry = true; continue; }
        if (u < -perr || u > T(1) + perr || v < -perr || v > T(1) + perr) continue;
        const bool boundary = u <= perr || u >= T(1) - perr || v <= perr || v >= T(1) - perr;
        if (u < T(0) || u > T(1)) u = u < T(0) ? T(0) : T(1);
        if (v < T(0) || v > T(1)) v = v < T(0) ? T(0) : T(1);
        const P2<T> res = add(add(add(a, mul(b, u)), mul(c, v)), mul(d, u * v));
        if (big(res) > T(256) * eps) { retry = true; continue; }
        const P3<T> lower = add(mul(p0, T(1) - u), mul(p1, u)), upper = add(mul(p2, T(1) - u), mul(p3, u));
        const P3<T> point = add(mul(lower, T(1) - v), mul(upper, v));
        const T t = comp(point, kz) / comp(w, kz);
        if (!(t > T(0))) {
            if (absv(t) <= T(64) * eps) retry = true;
            continue;
        }
        Hit h{float(u), float(v), float(t), 0.0f, 0u};
        if (boundary) h.flags |= hBoundary;
        if (repeated) h.flags |= hSingular;
        if (!Num<T>::is_float) h.flags |= hFp64;
        const F3 e = evaluate(corner, h.u, h.v);
        const F3 e3 = {e.x - dir.x * h.t, e.y - dir.y * h.t, e.z - dir.z * h.t};
        h.residual = maxv(absv(e3.x), maxv(absv(e3.y), absv(e3.z)));
        if (!(h.residual <= 0x1p-21f && h.t < 4.0f)) { retry = true; continue; }
        if (out.count < 2) out.hit[out.count++] = h;
        else retry = true;
    }
    return retry;
}

__device__ Hits intersect(const F3* c, F3 dir)
{
    Hits r{};
    const float n2 = fdot(dir, dir);
    if (!(finite32(dir.x) && finite32(dir.y) && finite32(dir.z)) || !(n2 > 0.99f && n2 < 1.01f)) {
        r.flags = bInvalid;
        return r;
    }
    for (unsigned i = 0; i < 4; ++i)
        if (!(finite32(c[i].x) && finite32(c[i].y) && finite32(c[i].z)) || !(fdot(c[i], c[i]) <= 4.0f)) {
            r.flags = bInvalid;
            return r;
        }
    if (solve<float>(c, dir, r)) {
        const bool unresolved = solve<double>(c, dir, r);
        r.flags |= bFp64;
        if (unresolved) r.flags |= bUnresolved;
    }
    if (r.count == 2 && (r.hit[1].u < r.hit[0].u || (r.hit[1].u == r.hit[0].u && r.hit[1].v < r.hit[0].v))) {
        const Hit t = r.hit[0];
        r.hit[0] = r.hit[1];
        r.hit[1] = t;
    }
    return r;
}

// The ray t dir, 0 <= t <= 4, against a padded box (binary32 slab test).
__device__ __forceinline__ bool ray_box(F3 dir, const icp_patch_aabb& b)
{
    const float lo[3] = {b.min_x, b.min_y, b.min_z}, hi[3] = {b.max_x, b.max_y, b.max_z}, d[3] = {dir.x, dir.y, dir.z};
    float tnear = 0.0f, tfar = 4.0f;
    for (unsigned a = 0; a < 3; ++a) {
        if (d[a] == 0.0f) {
            if (lo[a] > 0.0f || hi[a] < 0.0f) return false;
            continue;
        }
        const float t1 = lo[a] / d[a], t2 = hi[a] / d[a];
        const float tmin = t1 < t2 ? t1 : t2, tmax = t1 < t2 ? t2 : t1;
        if (tmin > tnear) tnear = tmin;
        if (tmax < tfar) tfar = tmax;
    }
    return tnear <= tfar;
}

// ------------------------------------------------------------------ direction bins
__device__ __forceinline__ int bin_row(double z)
{
    const double t = acos(fmin(1.0, fmax(-1.0, z)));
    const int r = int(t / kPi * kBinRows);
    return r < 0 ? 0 : (r >= kBinRows ? kBinRows - 1 : r);
}
__device__ __forceinline__ int bin_col(double x, double y)
{
    const int c = int((atan2(y, x) + kPi) / (2 * kPi) * kBinCols);
    return c < 0 ? 0 : (c >= kBinCols ? kBinCols - 1 : c);
}
__device__ __forceinline__ uint32_t direction_bin(F3 d)
{
    const double n = sqrt(double(d.x) * d.x + double(d.y) * d.y + double(d.z) * d.z);
    if (!(n > 0) || !(n < 1e30)) return 0;
    return uint32_t(bin_row(d.z / n)) * kBinCols + uint32_t(bin_col(d.x / n, d.y / n));
}
// Bins overlapped by the cap that bounds the cone over a patch's box: rows [r0, r1], and per
// row the columns [c0, c0 + nc) modulo kBinCols (nc = kBinCols: the whole row).
struct CapBins {
    int r0, r1, c0, nc;
};
__device__ CapBins cap_bins(const icp_patch_aabb& b)
{
    CapBins all{0, kBinRows - 1, 0, kBinCols};
    const float lo[3] = {b.min_x, b.min_y, b.min_z}, hi[3] = {b.max_x, b.max_y, b.max_z};
    for (unsigned a = 0; a < 3; ++a)
        if (!(finite32(lo[a]) && finite32(hi[a]))) return all;
    if (lo[0] <= 0 && hi[0] >= 0 && lo[1] <= 0 && hi[1] >= 0 && lo[2] <= 0 && hi[2] >= 0) return all;
    double dirs[8][3], c[3] = {0, 0, 0};
    for (unsigned k = 0; k < 8; ++k) {
        const double p[3] = {(k & 1) ? hi[0] : lo[0], (k & 2) ? hi[1] : lo[1], (k & 4) ? hi[2] : lo[2]};
        const double n = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        if (!(n > 0)) return all;
        for (unsigned a = 0; a < 3; ++a) {
            dirs[k][a] = p[a] / n;
            c[a] += dirs[k][a];
        }
    }
    const double cn = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    if (!(cn > 0)) return all;
    for (unsigned a = 0; a < 3; ++a) c[a] /= cn;
    double r = 0;
    for (unsigned k = 0; k < 8; ++k)
        r = fmax(r, acos(fmin(1.0, fmax(-1.0, c[0] * dirs[k][0] + c[1] * dirs[k][1] + c[2] * dirs[k][2]))));
    r += kCapMargin;
    if (!(r < 0.5 * kPi)) return all; // larger than a hemisphere: not convex, take everything
    const double tc = acos(fmin(1.0, fmax(-1.0, c[2])));
    const double dt = kPi / kBinRows, dp = 2 * kPi / kBinCols;
    CapBins out;
    out.r0 = int(floor((tc - r) / dt)) - 1;
    out.r1 = int(floor((tc + r) / dt)) + 1;
    if (tc - r <= 0 || tc + r >= kPi) { // the cap holds a pole
        out.r0 = out.r0 < 0 ? 0 : out.r0;
        out.r1 = out.r1 >= kBinRows ? kBinRows - 1 : out.r1;
        out.c0 = 0;
        out.nc = kBinCols;
        return out;
    }
    out.r0 = out.r0 < 0 ? 0 : out.r0;
    out.r1 = out.r1 >= kBinRows ? kBinRows - 1 : out.r1;
    const double s = sin(r) / sin(tc);
    if (!(s < 1)) {
        out.c0 = 0;
        out.nc = kBinCols;
        return out;
    }
    const double half = asin(s), pc = atan2(c[1], c[0]);
    const int c0 = int(floor((pc - half + kPi) / dp)) - 1, c1 = int(floor((pc + half + kPi) / dp)) + 1;
    out.nc = c1 - c0 + 1;
    if (out.nc >= kBinCols) {
        out.c0 = 0;
        out.nc = kBinCols;
    } else
        out.c0 = ((c0 % kBinCols) + kBinCols) % kBinCols;
    return out;
}

__global__ void __launch_bounds__(kThreads) query_bin_count_kernel(const icp_patch_aabb* __restrict__ boxes,
                                                                   uint32_t patch_count,
                                                                   unsigned long long* __restrict__ counts)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < patch_count; k += gridDim.x * blockDim.x) {
        const CapBins cb = cap_bins(boxes[k]);
        for (int r = cb.r0; r <= cb.r1; ++r)
            for (int j = 0; j < cb.nc; ++j) atomicAdd(&counts[r * kBinCols + (cb.c0 + j) % kBinCols], 1ull);
    }
}
__global__ void __launch_bounds__(kThreads) query_bin_fill_kernel(const icp_patch_aabb* __restrict__ boxes,
                                                                  uint32_t patch_count,
                                                                  const unsigned long long* __restrict__ offsets,
                                                                  uint32_t* __restrict__ fill, uint32_t* __restrict__ list)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < patch_count; k += gridDim.x * blockDim.x) {
        const CapBins cb = cap_bins(boxes[k]);
        for (int r = cb.r0; r <= cb.r1; ++r)
            for (int j = 0; j < cb.nc; ++j) {
                const uint32_t bin = r * kBinCols + (cb.c0 + j) % kBinCols;
                list[offsets[bin] + atomicAdd(&fill[bin], 1u)] = k;
            }
    }
}

// ------------------------------------------------------------------ per direction
struct QueryArgs {
    const icp_outgoing_vertex* vertices;
    const icp_outgoing_patch* patches;
    const icp_patch_aabb* boxes;
    const icp_vec3f* directions;
    const unsigned long long* bin_offsets; // kBinRows * kBinCols + 1
    const uint32_t* bin_list;
    uint32_t vertex_count, patch_count, direction_count;
};

__device__ __forceinline__ bool hit_less(const icp_query_hit& a, const icp_query_hit& b)
{
    if (a.patch_id != b.patch_id) return a.patch_id < b.patch_id;
    if (a.compact_index != b.compact_index) return a.compact_index < b.compact_index;
    return a.root_index < b.root_index;
}

// Intersects the direction with its bin's patches; writes roots into out[capacity] when out
// is given.  Returns the root count; flags / first problem patch as the collector notes them.
__device__ uint32_t collect(const QueryArgs& q, uint32_t i, icp_query_hit* out, uint32_t capacity, uint32_t& flags,
                            uint32_t& first)
{
    const F3 dir = f3(q.directions[i]);
    const float n2 = fdot(dir, dir);
    uint32_t count = 0;
    flags = 0;
    first = 0xffffffffu;
    if (!(finite32(dir.x) && finite32(dir.y) && finite32(dir.z)) || !(n2 > 0.99f && n2 < 1.01f)) {
        flags |= qInvalid;
        return 0;
    }
    const uint32_t bin = direction_bin(dir);
    for (unsigned long long s = q.bin_offsets[bin]; s < q.bin_offsets[bin + 1]; ++s) {
        const uint32_t k = q.bin_list[s];
        if (!ray_box(dir, q.boxes[k])) continue;
        const icp_outgoing_patch& p = q.patches[k];
        F3 c[4];
        bool bad = false;
        for (unsigned j = 0; j < 4; ++j) {
            if (p.vertex_indices[j] >= q.vertex_count) {
                bad = true;
                break;
            }
            c[j] = f3(q.vertices[p.vertex_indices[j]].direction_drop);
        }
        if (bad) {
            flags |= qInvalid;
            continue;
        }
        const Hits h = intersect(c, dir);
        if ((h.flags & (bUnresolved | bInvalid)) && p.patch_id < first) first = p.patch_id;
        if (h.flags & bUnresolved) flags |= qUnresolved;
        if (h.flags & bInvalid) flags |= qInvalid;
        if (h.flags & bFp64) flags |= qFp64;
        for (uint32_t r = 0; r < h.count; ++r) {
            if (out) {
                if (count >= capacity) flags |= qMismatch;
                else out[count] = {k, p.patch_id, r, h.hit[r].flags, h.hit[r].u, h.hit[r].v, h.hit[r].t, h.hit[r].residual};
            }
            ++count;
        }
    }
    return count;
}

// Roots a direction keeps from the counting pass for the fill pass (a direction with more is
// intersected again there).
constexpr uint32_t kCachedRoots = 8;
struct RootCache {
    icp_query_hit* hits; // kCachedRoots per direction, or null (sizing call: nothing kept)
    uint32_t* flags;     // the collector's flags and first problem patch of the direction
    uint32_t* first;
};

__global__ void __launch_bounds__(kThreads, kQueryBlocksPerSm) query_count_kernel(QueryArgs q, unsigned long long* __restrict__ counts,
                                                               RootCache cache)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < q.direction_count; i += gridDim.x * blockDim.x) {
        uint32_t flags, first;
        if (cache.hits) {
            const uint32_t n = collect(q, i, cache.hits + (size_t)i * kCachedRoots, kCachedRoots, flags, first);
            cache.flags[i] = flags;
            cache.first[i] = first;
            counts[i] = n;
        } else
            counts[i] = collect(q, i, nullptr, 0, flags, first);
    }
}

__global__ void __launch_bounds__(kThreads, kQueryBlocksPerSm) query_fill_kernel(QueryArgs q, const unsigned long long* __restrict__ offsets,
                                                              icp_query_summary* __restrict__ summaries,
                                                              icp_query_hit* __restrict__ hits, RootCache cache)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < q.direction_count; i += gridDim.x * blockDim.x) {
        const unsigned long long begin = offsets[i], end = offsets[i + 1];
        const uint32_t capacity = uint32_t(end - begin);
        icp_query_hit* out = hits + begin;
        uint32_t flags, first, count;
        if (cache.hits && capacity <= kCachedRoots) {
            // the counting pass kept every root of this direction, in the order it found them
            const icp_query_hit* kept = cache.hits + (size_t)i * kCachedRoots;
            for (uint32_t a = 0; a < capacity; ++a) out[a] = kept[a];
            count = capacity;
            flags = cache.flags[i];
            first = cache.first[i];
        } else
            count = collect(q, i, out, capacity, flags, first);
        icp_query_summary sm{};
        sm.candidate_count = capacity;
        if (count != capacity) flags |= qMismatch;
        sm.first_problem_patch_id = first;
        if (count <= capacity) {
            for (uint32_t a = 1; a < count; ++a) { // insertion sort (stable)
                const icp_query_hit x = out[a];
                uint32_t b = a;
                while (b != 0 && hit_less(x, out[b - 1])) {
                    out[b] = out[b - 1];
                    --b;
                }
                out[b] = x;
            }
            uint32_t kept = 0;
            for (uint32_t a = 0; a < count; ++a) {
                const icp_query_hit h = out[a];
                if (kept != 0 && h.compact_index == out[kept - 1].compact_index && h.root_index == out[kept - 1].root_index) {
                    flags |= qDuplicate;
                    continue;
                }
                if (h.compact_index >= q.patch_count) {
                    flags |= qInvalid;
                    continue;
                }
                out[kept++] = h;
                const uint32_t st = q.patches[h.compact_index].status;
                if (st == 3u) {
                    ++sm.refinement_hits;
                    flags |= qRefine;
                } else if (st == 1u || st == 2u)
                    ++sm.regular_hits;
                else
                    flags |= qInvalid;
                if (h.flags & hBoundary) {
                    ++sm.boundary_hits;
                    flags |= qBoundary;
                }
                if (h.flags & hSingular) flags |= qSingular;
            }
            sm.hit_count = kept;
        }
        sm.flags = flags;
        summaries[i] = sm;
    }
}

// ------------------------------------------------------------------ 64-bit exclusive scan
// Exclusive scan of one chunk of up to kScanThreads values starting at `carry`; every thread
// returns the chunk's total.  A thread reads only its own element before writing it, so in and
// out may be the same array.
__device__ unsigned long long chunk_scan(const unsigned long long* in, unsigned long long* out, uint64_t base,
                                         uint64_t n, unsigned long long carry)
{
    __shared__ unsigned long long warp_sums[kScanThreads / 32];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint64_t i = base + threadIdx.x;
    const unsigned long long x = i < n ? in[i] : 0ull;
    unsigned long long incl = x;
    for (unsigned d = 1; d < 32; d *= 2) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += y;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        unsigned long long w = warp_sums[lane];
        for (unsigned d = 1; d < 32; d *= 2) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= d) w += y;
        }
        warp_sums[lane] = w;
    }
    __syncthreads();
    const unsigned long long total = warp_sums[kScanThreads / 32 - 1];
    const unsigned long long before = (warp ? warp_sums[warp - 1] : 0ull) + incl - x;
    __syncthreads(); // warp_sums is reused by the next chunk
    if (i < n) out[i] = carry + before;
    return total;
}
// Per-block totals of in[n] (kScanThreads values per block).
__global__ void __launch_bounds__(kScanThreads) scan_block_sums(const unsigned long long* __restrict__ in, uint64_t n,
                                                                unsigned long long* __restrict__ sums)
{
    __shared__ unsigned long long part[kScanThreads / 32];
    const uint64_t i = uint64_t(blockIdx.x) * kScanThreads + threadIdx.x;
    unsigned long long x = i < n ? in[i] : 0ull;
    for (unsigned d = 16; d; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
    if ((threadIdx.x & 31u) == 0) part[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned long long y = part[threadIdx.x];
        for (unsigned d = 16; d; d >>= 1) y += __shfl_down_sync(0xffffffffu, y, d);
        if (threadIdx.x == 0) sums[blockIdx.x] = y;
    }
}
// One block: exclusive scan of the block totals in place; the grand total into sums[nblocks].
__global__ void __launch_bounds__(kScanThreads) scan_sums(unsigned long long* sums, uint64_t nblocks)
{
    unsigned long long carry = 0;
    for (uint64_t base = 0; base < nblocks; base += kScanThreads) carry += chunk_scan(sums, sums, base, nblocks, carry);
    if (threadIdx.x == 0) sums[nblocks] = carry;
}
// out[i] = exclusive prefix of in[i]; out[n] = total.
__global__ void __launch_bounds__(kScanThreads) scan_add(const unsigned long long* __restrict__ in, uint64_t n,
                                                         const unsigned long long* __restrict__ sums,
                                                         unsigned long long* __restrict__ out)
{
    chunk_scan(in, out, uint64_t(blockIdx.x) * kScanThreads, n, sums[blockIdx.x]);
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = sums[gridDim.x];
}
// Exclusive scan of in[n] into out[n + 1] with sums[ceil(n / kScanThreads) + 1] of scratch.
int exclusive_scan(const unsigned long long* in, uint64_t n, unsigned long long* sums, unsigned long long* out,
                   cudaStream_t stream)
{
    const uint64_t blocks = n ? (n + kScanThreads - 1) / kScanThreads : 1;
    scan_block_sums<<<unsigned(blocks), kScanThreads, 0, stream>>>(in, n, sums);
    scan_sums<<<1, kScanThreads, 0, stream>>>(sums, blocks);
    scan_add<<<unsigned(blocks), kScanThreads, 0, stream>>>(in, n, sums, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ICP_ERR_DEVICE, "patch query scan: %s", cudaGetErrorString(e));
    count_launch();
    count_launch();
    count_launch();
    return ICP_OK;
}

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

} // namespace

extern "C" int icp_query_directions(uint32_t theta_count, uint32_t phi_count, const float axis[3], const float e0[3],
                                    float* directions)
{
    // QueryDirectionGrid::make / directions (include/rainbow/query_direction_grid.hpp:14-58)
    if (!axis || !e0 || !directions) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_query_directions: null argument");
    if (theta_count == 0 || phi_count == 0 || uint64_t(theta_count) * phi_count > 0xffffffffull)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid query grid dimensions.");
    auto dotf = [](const float* a, const float* b) { return std::fma(a[0], b[0], std::fma(a[1], b[1], a[2] * b[2])); };
    auto fin = [](const float* a) {
        for (int k = 0; k < 3; ++k)
            if (!(a[k] >= -FLT_MAX && a[k] <= FLT_MAX)) return false;
        return true;
    };
    if (!fin(axis) || !fin(e0) || std::fabs(dotf(axis, axis) - 1.0f) > 1e-5f || std::fabs(dotf(e0, e0) - 1.0f) > 1e-5f ||
        std::fabs(dotf(axis, e0)) > 1e-5f)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Query grid requires an orthonormal incident frame.");
    float e1[3] = {axis[1] * e0[2] - axis[2] * e0[1], axis[2] * e0[0] - axis[0] * e0[2], axis[0] * e0[1] - axis[1] * e0[0]};
    const float n1 = std::sqrt(dotf(e1, e1));
    for (float& x : e1) x = x / n1;
    for (uint32_t row = 0; row < theta_count; ++row) {
        const double t = kPi * (double(row) + 0.5) / double(theta_count), st = std::sin(t), ct = std::cos(t);
        for (uint32_t col = 0; col < phi_count; ++col) {
            const double p = -kPi + 2.0 * kPi * (double(col) + 0.5) / double(phi_count);
            const double x = st * std::cos(p), y = st * std::sin(p);
            float w[3];
            for (int k = 0; k < 3; ++k) w[k] = float(double(axis[k]) * ct + double(e0[k]) * x + double(e1[k]) * y);
            const float n = std::sqrt(dotf(w, w));
            float* o = directions + 3 * (size_t(row) * phi_count + col);
            for (int k = 0; k < 3; ++k) o[k] = w[k] / n;
        }
    }
    return ok();
}

extern "C" int icp_patch_query(icp_context* ctx, const icp_outgoing_vertex* d_vertices, uint32_t vertex_count,
                               const icp_outgoing_patch* d_patches, const icp_patch_aabb* d_aabbs, uint32_t patch_count,
                               const icp_vec3f* d_directions, uint32_t direction_count, uint64_t* d_offsets,
                               icp_query_summary* d_summaries, icp_query_hit* d_hits, uint64_t hit_capacity,
                               uint64_t* hit_count)
{
    if (!ctx || !d_vertices || (patch_count && (!d_patches || !d_aabbs)) || (direction_count && !d_directions) ||
        !d_offsets || !hit_count)
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_patch_query: null argument");
    if (direction_count > 0x7fffffffu || patch_count > 0x7fffffffu)
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_patch_query: too many patches or directions");
    const uint64_t bins = uint64_t(kBinRows) * kBinCols;
    const uint64_t nscan = (bins > direction_count ? bins : direction_count);
    const uint64_t sum_blocks = (nscan + kScanThreads - 1) / kScanThreads + 1;
    // scratch: bin counts (u64), bin offsets (u64, +1), bin fill (u32), scan block sums (u64),
    // per-direction counts (u64), then the bin list (u32, sized after the bin scan)
    const size_t o_counts = 0, o_offsets = align_up(o_counts + bins * 8), o_fill = align_up(o_offsets + (bins + 1) * 8);
    const size_t o_sums = align_up(o_fill + bins * 4), o_dir = align_up(o_sums + sum_blocks * 8);
    const size_t o_list = align_up(o_dir + (size_t(direction_count) + 1) * 8);
    // a call that fills keeps up to kCachedRoots roots per direction from the counting pass
    const bool keep = d_hits && d_summaries;
    const size_t o_chits = o_list, o_cflags = align_up(o_chits + (keep ? sizeof(icp_query_hit) * kCachedRoots * direction_count : 0));
    const size_t o_cfirst = align_up(o_cflags + (keep ? 4 * size_t(direction_count) : 0));
    const size_t o_end = align_up(o_cfirst + (keep ? 4 * size_t(direction_count) : 0));
    ICP_CUDA(cudaSetDevice(ctx->device));
    ICP_CUDA(ctx->query.ensure(o_end));
    char* base = static_cast<char*>(ctx->query.ptr);
    auto* bin_counts = reinterpret_cast<unsigned long long*>(base + o_counts);
    auto* bin_offsets = reinterpret_cast<unsigned long long*>(base + o_offsets);
    auto* bin_fill = reinterpret_cast<uint32_t*>(base + o_fill);
    auto* sums = reinterpret_cast<unsigned long long*>(base + o_sums);
    auto* dir_counts = reinterpret_cast<unsigned long long*>(base + o_dir);
    RootCache cache{nullptr, nullptr, nullptr};
    if (keep)
        cache = {reinterpret_cast<icp_query_hit*>(base + o_chits), reinterpret_cast<uint32_t*>(base + o_cflags),
                 reinterpret_cast<uint32_t*>(base + o_cfirst)};
    const unsigned pblocks = unsigned(patch_count ? (patch_count + kThreads - 1) / kThreads : 1);
    ICP_CUDA(cudaMemsetAsync(base, 0, o_sums, ctx->stream)); // counts, offsets, fill
    if (patch_count) {
        query_bin_count_kernel<<<pblocks, kThreads, 0, ctx->stream>>>(d_aabbs, patch_count, bin_counts);
        ICP_CUDA(cudaGetLastError());
        count_launch();
    }
    if (const int st = exclusive_scan(bin_counts, bins, sums, bin_offsets, ctx->stream)) return st;
    unsigned long long list_len = 0;
    ICP_CUDA(cudaMemcpyAsync(&list_len, bin_offsets + bins, 8, cudaMemcpyDeviceToHost, ctx->stream));
    ICP_CUDA(cudaStreamSynchronize(ctx->stream));
    ICP_CUDA(ctx->query_list.ensure(size_t(list_len ? list_len : 1) * 4));
    auto* bin_list = static_cast<uint32_t*>(ctx->query_list.ptr);
    if (patch_count) {
        query_bin_fill_kernel<<<pblocks, kThreads, 0, ctx->stream>>>(d_aabbs, patch_count, bin_offsets, bin_fill, bin_list);
        ICP_CUDA(cudaGetLastError());
        count_launch();
    }
    const QueryArgs q{d_vertices, d_patches, d_aabbs, d_directions, bin_offsets, bin_list, vertex_count, patch_count,
                      direction_count};
    const uint64_t need = (uint64_t(direction_count) + kThreads - 1) / kThreads;
    const uint64_t cap = uint64_t(ctx->sms > 0 ? ctx->sms : 148) * 16u;
    const unsigned dblocks = unsigned(need ? (need < cap ? need : cap) : 1);
    if (direction_count) {
        query_count_kernel<<<dblocks, kThreads, 0, ctx->stream>>>(q, dir_counts, cache);
        ICP_CUDA(cudaGetLastError());
        count_launch();
    }
    auto* offsets = reinterpret_cast<unsigned long long*>(d_offsets);
    if (const int st = exclusive_scan(dir_counts, direction_count, sums, offsets, ctx->stream)) return st;
    unsigned long long total = 0;
    ICP_CUDA(cudaMemcpyAsync(&total, offsets + direction_count, 8, cudaMemcpyDeviceToHost, ctx->stream));
    ICP_CUDA(cudaStreamSynchronize(ctx->stream));
    *hit_count = total;
    if (!d_hits || !d_summaries) return ok(); // sizing call
    if (total > hit_capacity)
        return fail(ICP_ERR_CAPACITY, "icp_patch_query: %llu hits, capacity %llu", total,
                    (unsigned long long)hit_capacity);
    if (direction_count) {
        query_fill_kernel<<<dblocks, kThreads, 0, ctx->stream>>>(q, offsets, d_summaries, d_hits, cache);
        ICP_CUDA(cudaGetLastError());
        count_launch();
    }
    ICP_CUDA(cudaStreamSynchronize(ctx->stream));
    return ok();
}
