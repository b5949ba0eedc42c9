// icp_lattice.cu -- the drop's outgoing-ray lattice traced on the device (sm_100a) and its C ABI
// (include/icp_b200.h, "lattice trace").
//
// The wave stages of a drop record start from one incident ray per vertex of a W x H lattice
// spanning the drop's silhouette, each followed through the four path families R, TT, TRT and
// TRRT (RaindropPathTracer::trace_vertex_unpolarized, include/rainbow/raindrop_paths.hpp:
// 27-107).  The reference runs that chain in an OptiX raygen program
// (shaders/entry/raindrop_trace.cu:49-83) and answers each boundary query with a custom-
// primitive intersection program that calls RaindropIntersector for the drop's one bounding box
// (src/raindrop_tracer.cpp:116-177).  A single convex body needs no acceleration structure:
// here one thread per vertex calls the intersector itself.  The box cannot change an answer --
// it only culls rays that miss a box enclosing the drop by 2^-15, for which the intersector
// finds no root either, and a reported distance minus the start offset always lies within the
// box program's [0, 8 r_out + 4] because the intersector searches exactly that range.
//
// Every record equals the reference's bit for bit.  The unit is built with -fmad=false and IEEE
// division and square root, as the reference builds its device modules
// (cmake/rainbow_modules.cmake:23-28), and every expression keeps the reference's association
// and its explicit fma calls:
//   * the surface root (raindrop_intersection.hpp:203-382): outward-rounded interval bounds of
//     the implicit function and its derivative on [start, 8 r_out + 4], depth-first bisection
//     on a 64-entry stack (16384 visits at most), a safeguarded Newton iteration (96 steps) on
//     a bracket whose monotonicity the bounds certify; binary32 first, binary64 again when the
//     binary32 solve is inconclusive or grazes (|n . d| < 0.05);
//   * the interface (dielectric_interface.hpp:37-135): the Fresnel split of the two-column
//     Jones response in the fixed s / p convention, binary64 re-evaluation near the critical
//     angle, the total-internal-reflection phase;
//   * the optical path (optical_path.hpp, phase_cycles.hpp): float-pair distances in cycles,
//     whole turns and a fraction.
// Outward rounding steps to the neighbouring representable number (the IEEE 754 nextUp /
// nextDown operations, here on the bit patterns), as the reference's nextafter calls do.
//
// The reference validates a finished trace with a separate reduction (PhaseCdf::validate_trace,
// src/phase_cdf.cpp:238-253; phase_validate_trace, device/phase_cdf.cu:67-83); here the same
// test runs on each record as it is written, with the per-family status histogram, in the trace
// kernel itself.
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

// vertex status (rainbow::VertexStatus) and diagnostics (rainbow::TraceDiagnostic)
enum : uint32_t { kUnwritten = 0, kValid = 1, kMiss = 2, kTir = 3, kUnresolved = 4, kInvalid = 5, kOverflow = 6 };
enum : uint32_t { kIsectFallback = 1, kSnellFallback = 2 };
enum Code : uint32_t { kCodeMiss = 0, kCodeHit = 1, kCodeUnresolved = 2 };

// ------------------------------------------------------------------ scalar steps
template <class T> __host__ __device__ __forceinline__ T fused(T a, T b, T c)
{
    if constexpr (std::is_same_v<T, float>) return fmaf(a, b, c);
    else return fma(a, b, c);
}
template <class T> __host__ __device__ __forceinline__ T root(T x)
{
    if constexpr (std::is_same_v<T, float>) return sqrtf(x);
    else return sqrt(x);
}
// nextUp: the least representable number above x (+inf and NaN unchanged, either zero to the
// least positive subnormal); nextDown(x) = -nextUp(-x).
__device__ __forceinline__ float next_up(float x)
{
    if (!(x < INFINITY)) return x;
    if (x == 0.0f) return __int_as_float(1);
    const int b = __float_as_int(x);
    return __int_as_float(b >= 0 ? b + 1 : b - 1);
}
__device__ __forceinline__ double next_up(double x)
{
    if (!(x < (double)INFINITY)) return x;
    if (x == 0.0) return __longlong_as_double(1ll);
    const long long b = __double_as_longlong(x);
    return __longlong_as_double(b >= 0 ? b + 1 : b - 1);
}
template <class T> __device__ __forceinline__ T next_down(T x) { return -next_up(-x); }
template <class T> __device__ __forceinline__ T lesser(T a, T b) { return a < b ? a : b; }
template <class T> __device__ __forceinline__ T greater(T a, T b) { return a > b ? a : b; }
template <class T> __device__ __forceinline__ T magnitude(T x) { return x < T(0) ? -x : x; }
template <class T> __device__ __forceinline__ T infinity_of() { return T(INFINITY); }

// ------------------------------------------------------------------ vectors
template <class T> struct V {
    T x, y, z;
};
template <class T> __device__ __forceinline__ V<T> operator+(V<T> a, V<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> __device__ __forceinline__ V<T> operator-(V<T> a, V<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> __device__ __forceinline__ V<T> operator-(V<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> __device__ __forceinline__ V<T> operator*(V<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> __device__ __forceinline__ V<T> operator/(V<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> __device__ __forceinline__ T dot(V<T> a, V<T> b) { return fused(a.x, b.x, fused(a.y, b.y, a.z * b.z)); }
// the symmetric difference, so that cross(v, v) is exactly zero
template <class T> __device__ __forceinline__ V<T> cross(V<T> a, V<T> b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> __device__ __forceinline__ T length(V<T> a) { return root(dot(a, a)); }
template <class T> __device__ __forceinline__ V<T> unit(V<T> a) { return a / length(a); }
template <class T> __device__ __forceinline__ V<T> along(V<T> o, V<T> d, T t)
{
    return {fused(t, d.x, o.x), fused(t, d.y, o.y), fused(t, d.z, o.z)};
}
template <class U, class T> __device__ __forceinline__ V<U> to(V<T> a) { return {U(a.x), U(a.y), U(a.z)}; }
template <class T> __device__ __forceinline__ bool finite(V<T> a)
{
    const T m = std::is_same_v<T, float> ? T(FLT_MAX) : T(DBL_MAX);
    return a.x >= -m && a.x <= m && a.y >= -m && a.y <= m && a.z >= -m && a.z <= m;
}
using F3 = V<float>;
using D3 = V<double>;
__device__ __forceinline__ F3 f3(const icp_vec3f& v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ icp_vec3f store3(F3 v) { return {v.x, v.y, v.z}; }

// ------------------------------------------------------------------ outward-rounded intervals
template <class T> struct Iv {
    T lo, hi;
};
template <class T> __device__ __forceinline__ Iv<T> at_point(T x) { return {x, x}; }
template <class T> __device__ __forceinline__ Iv<T> operator+(Iv<T> a, Iv<T> b)
{
    return {next_down(a.lo + b.lo), next_up(a.hi + b.hi)};
}
template <class T> __device__ __forceinline__ Iv<T> operator-(Iv<T> a) { return {-a.hi, -a.lo}; }
template <class T> __device__ __forceinline__ Iv<T> operator-(Iv<T> a, Iv<T> b) { return a + (-b); }
template <class T> __device__ __forceinline__ Iv<T> operator*(Iv<T> a, Iv<T> b)
{
    const T p = a.lo * b.lo, q = a.lo * b.hi, r = a.hi * b.lo, s = a.hi * b.hi;
    return {next_down(lesser(lesser(p, q), lesser(r, s))), next_up(greater(greater(p, q), greater(r, s)))};
}
template <class T> __device__ __forceinline__ Iv<T> operator/(Iv<T> a, Iv<T> b)
{
    if (b.lo <= T(0) && b.hi >= T(0)) return {-infinity_of<T>(), infinity_of<T>()};
    return a * Iv<T>{next_down(T(1) / b.hi), next_up(T(1) / b.lo)};
}
template <class T> __device__ __forceinline__ Iv<T> squared(Iv<T> a)
{
    const T p = a.lo * a.lo, q = a.hi * a.hi;
    return {a.lo <= T(0) && a.hi >= T(0) ? T(0) : greater(T(0), next_down(lesser(p, q))), next_up(greater(p, q))};
}
template <class T> __device__ __forceinline__ Iv<T> square_root(Iv<T> a)
{
    return {greater(T(0), next_down(root(greater(T(0), a.lo)))), next_up(root(greater(T(0), a.hi)))};
}
template <class T> __device__ __forceinline__ bool excludes_zero(Iv<T> a) { return a.lo > T(0) || a.hi < T(0); }

// ------------------------------------------------------------------ the drop's surface
// r/a = 1 + sum_n c_n T_n(mu), mu = cos(chi) from the -y axis (raindrop_shape.hpp:69-100);
// `last` is the highest n with c_n != 0 (the interval series skips zero terms, so the
// recurrence beyond it feeds nothing).
struct Shape {
    float c[8];
    float inner, outer;
    unsigned last;
};

template <class T> __device__ __forceinline__ T series(const Shape& S, T mu, T& derivative)
{
    T previous = T(1), current = mu, d_previous = T(0), d_current = T(1);
    T radius = T(1) + T(S.c[0]) + T(S.c[1]) * mu;
    derivative = T(S.c[1]);
#pragma unroll
    for (unsigned n = 2; n < 8; ++n) {
        const T next = T(2) * mu * current - previous;
        const T d_next = T(2) * current + T(2) * mu * d_current - d_previous;
        radius += T(S.c[n]) * next;
        derivative += T(S.c[n]) * d_next;
        previous = current;
        current = next;
        d_previous = d_current;
        d_current = d_next;
    }
    return radius;
}
template <class T> __device__ __forceinline__ T implicit(const Shape& S, V<T> p)
{
    const T r = length(p);
    if (r < T(S.inner) * T(0.25)) return r - T(S.inner); // deep inside: the sign is all that matters
    T derivative;
    return r - series(S, -p.y / r, derivative);
}
template <class T> __device__ __forceinline__ V<T> gradient(const Shape& S, V<T> p)
{
    const T r = length(p);
    const V<T> u = p / r;
    T derivative;
    const T mu = -u.y;
    (void)series(S, mu, derivative);
    return u - (V<T>{T(0), T(-1), T(0)} - u * mu) * (derivative / r);
}

template <class T> struct Bounds {
    Iv<T> value, derivative;
};
// Interval enclosure of f(o + t w) = |p| - R(mu) and of its t-derivative for t in [lower, upper].
template <class T> __device__ Bounds<T> bound_surface(const Shape& S, V<T> o, V<T> w, T lower, T upper)
{
    using I = Iv<T>;
    const T inf = infinity_of<T>();
    const I t{lower, upper};
    const I px = at_point(o.x) + t * at_point(w.x);
    const I py = at_point(o.y) + t * at_point(w.y);
    const I pz = at_point(o.z) + t * at_point(w.z);
    const I r = square_root(squared(px) + squared(py) + squared(pz));
    if (r.hi < T(S.inner)) return {{-T(1), -T(1)}, {-inf, inf}};
    if (r.lo > T(S.outer)) return {{T(1), T(1)}, {-inf, inf}};
    if (r.lo <= T(0)) return {{-inf, inf}, {-inf, inf}};
    I mu = (-py) / r;
    mu.lo = greater(mu.lo, -T(1));
    mu.hi = lesser(mu.hi, T(1));
    I previous = at_point(T(1)), current = mu, dp = at_point(T(0)), dc = at_point(T(1));
    I radius = at_point(T(1)) + at_point(T(S.c[0])) + at_point(T(S.c[1])) * mu;
    I slope = at_point(T(S.c[1]));
    const I two = at_point(T(2));
    for (unsigned n = 2; n <= S.last; ++n) {
        const I next = two * mu * current - previous;
        const I dn = two * current + two * mu * dc - dp;
        if (S.c[n] != 0.0f) {
            radius = radius + at_point(T(S.c[n])) * next;
            slope = slope + at_point(T(S.c[n])) * dn;
        }
        previous = current;
        current = next;
        dp = dc;
        dc = dn;
    }
    const I dr = (px * at_point(w.x) + py * at_point(w.y) + pz * at_point(w.z)) / r;
    const I dm = (at_point(-w.y) - mu * dr) / r;
    return {r - radius, dr - slope * dm};
}

struct Query {
    F3 origin, direction;
    float start; // self-hit exclusion along the ray, not part of the returned distance
    bool inside;
};
template <class T> struct Root {
    Code code;
    T distance;
};
template <class T> struct Segment {
    T lo, hi;
};

template <class T> __device__ Root<T> solve_surface(const Shape& S, const Query& q)
{
    const V<T> o = to<T>(q.origin), w = to<T>(q.direction);
    const T start = T(q.start);
    const T limit = T(8) * T(S.outer) + T(4);
    const T tolerance = std::is_same_v<T, float> ? T(0x1p-22) : T(0x1p-44);
    if (q.inside) {
        const T f = implicit(S, along(o, w, start));
        if (!(f < T(0))) return {kCodeUnresolved, T(0)}; // a grazing chord is not skipped silently
    }
    Segment<T> stack[64];
    unsigned size = 0, visits = 0;
    stack[size++] = {start, limit};
    while (size != 0) {
        if (++visits > 16384u) return {kCodeUnresolved, T(0)};
        const Segment<T> s = stack[--size];
        const Bounds<T> b = bound_surface(S, o, w, s.lo, s.hi);
        if (excludes_zero(b.value)) continue;
        const T mid = s.lo + (s.hi - s.lo) * T(0.5);
        const T width_tolerance = tolerance * greater(T(1), magnitude(mid));
        if (excludes_zero(b.derivative)) {
            T lo = s.lo, hi = s.hi;
            T f_lo = implicit(S, along(o, w, lo));
            T f_hi = implicit(S, along(o, w, hi));
            if ((f_lo < T(0)) == (f_hi < T(0))) {
                // monotone with equal end signs: excluded once the end values' signs are certain
                const Iv<T> left = bound_surface(S, o, w, lo, lo).value;
                const Iv<T> right = bound_surface(S, o, w, hi, hi).value;
                if ((left.lo > T(0) && right.lo > T(0)) || (left.hi < T(0) && right.hi < T(0))) continue;
            }
            if (f_lo == T(0) && lo > start) return {kCodeHit, lo};
            if (f_hi == T(0) && hi > start) return {kCodeHit, hi};
            if ((f_lo < T(0)) != (f_hi < T(0))) {
                T x = mid;
                for (unsigned it = 0; it < 96u; ++it) {
                    const V<T> p = along(o, w, x);
                    const T f = implicit(S, p);
                    if (f == T(0) || hi - lo <= width_tolerance) return {kCodeHit, x};
                    if ((f < T(0)) == (f_lo < T(0))) {
                        lo = x;
                        f_lo = f;
                    } else {
                        hi = x;
                        f_hi = f;
                    }
                    const T slope = dot(gradient(S, p), w);
                    const T candidate = x - f / slope;
                    const T guard = (hi - lo) * T(0.1);
                    x = candidate > lo + guard && candidate < hi - guard ? candidate : lo + (hi - lo) * T(0.5);
                }
                return {kCodeUnresolved, T(0)};
            }
        }
        if (s.hi - s.lo <= width_tolerance || mid == s.lo || mid == s.hi || size + 2 > 64u)
            return {kCodeUnresolved, T(0)};
        stack[size++] = {mid, s.hi};
        stack[size++] = {s.lo, mid};
    }
    return {kCodeMiss, T(0)};
}

struct Hit {
    Code code;
    F3 position, normal;
    uint32_t diagnostics;
};
// RaindropIntersector::intersect (raindrop_intersection.hpp:337-382)
__device__ Hit intersect(const Shape& S, const Query& q)
{
    Hit h{kCodeMiss, {0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}, 0u};
    const Root<float> r = solve_surface<float>(S, q);
    bool fallback = r.code == kCodeUnresolved;
    if (r.code == kCodeHit) {
        const F3 p = along(q.origin, q.direction, r.distance);
        const float incidence = fabsf(dot(unit(gradient(S, p)), q.direction));
        fallback = incidence < 0.05f; // grazing: binary32 is ill-conditioned there
    }
    h.code = r.code;
    if (fallback) {
        const Root<double> d = solve_surface<double>(S, q);
        h.code = d.code;
        h.diagnostics |= kIsectFallback;
        if (d.code == kCodeHit) {
            const D3 p = along(to<double>(q.origin), to<double>(q.direction), d.distance);
            h.position = to<float>(p);
            h.normal = unit(to<float>(unit(gradient(S, p))));
        }
    } else if (r.code == kCodeHit) {
        h.position = along(q.origin, q.direction, r.distance);
        h.normal = unit(gradient(S, h.position));
    }
    return h;
}

// ------------------------------------------------------------------ Jones responses
struct C32 {
    float re, im;
};
__device__ __forceinline__ C32 operator+(C32 a, C32 b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ C32 operator*(C32 a, float s) { return {a.re * s, a.im * s}; }
__device__ __forceinline__ C32 operator*(C32 a, C32 b)
{
    return {fmaf(a.re, b.re, -(a.im * b.im)), fmaf(a.re, b.im, a.im * b.re)};
}
struct Field {
    C32 x, y;
};
// columns: the output fields for unit input states 0 and 1; `columns` = 1 for a single input
struct Response {
    Field col[2];
};
__device__ __forceinline__ bool finite(float v) { return v >= -FLT_MAX && v <= FLT_MAX; }
__device__ __forceinline__ bool finite(const Field& f)
{
    return finite(f.x.re) && finite(f.x.im) && finite(f.y.re) && finite(f.y.im);
}

struct Ray {
    F3 direction, e0, e1; // e0, e1, direction right-handed
    Response field;
};
struct Branches {
    Ray reflected, transmitted;
    bool has_transmission, valid;
    uint32_t diagnostics;
};

__device__ __forceinline__ C32 tir_coefficient(float a, float b)
{
    // (a - i b) / (a + i b): the total-reflection phase for the exp(i k z - i w t) convention
    const float scale = fmaxf(fabsf(a), fabsf(b));
    const float x = a / scale, y = b / scale, den = fmaf(x, x, y * y);
    return {fmaf(x, x, -y * y) / den, (-2.0f * x * y) / den};
}

// DielectricInterface::split (dielectric_interface.hpp:37-135): amplitude coefficients,
// s = normalize(w_i x n), p = w x s for each ray, n pointing into the incident medium.
__device__ Branches split(const Ray& in, F3 n, float n_i, float n_t, unsigned columns)
{
    Branches out{};
    out.has_transmission = false;
    out.valid = false;
    out.diagnostics = 0u;
    const F3 wi = in.direction;
    float cosine = -dot(wi, n);
    if (!(cosine >= -0x1p-19f && cosine <= 1.0f + 0x1p-19f && n_i > 0 && n_t > 0)) return out;
    cosine = fminf(1.0f, fmaxf(0.0f, cosine));
    F3 s = cross(wi, n);
    const float sin2 = dot(s, s);
    if (sin2 > 0x1p-40f) s = s / sqrtf(sin2);
    else s = unit(in.e0 - wi * dot(wi, in.e0));
    const F3 pi = unit(cross(wi, s));
    const float a = dot(in.e0, s), b = dot(in.e1, s), c = dot(in.e0, pi), d = dot(in.e1, pi);
    Response local{};
    for (unsigned j = 0; j < columns; ++j)
        local.col[j] = {in.field.col[j].x * a + in.field.col[j].y * b, in.field.col[j].x * c + in.field.col[j].y * d};

    const float eta = n_i / n_t;
    float discriminant = fmaf(-(eta * eta), sin2, 1.0f);
    if (fabsf(discriminant) < 0x1p-15f) {
        // near the critical angle the branch can change: binary64 decides
        const D3 wd = unit(to<double>(wi)), nd = unit(to<double>(n));
        const double ratio = double(n_i) / double(n_t);
        const D3 sd = cross(wd, nd);
        discriminant = static_cast<float>(fma(-ratio * ratio, dot(sd, sd), 1.0));
        cosine = static_cast<float>(-dot(wd, nd));
        out.diagnostics |= kSnellFallback;
    }
    const F3 wr = unit(along(wi, n, 2.0f * cosine));
    out.reflected.direction = wr;
    out.reflected.e0 = s;
    out.reflected.e1 = unit(cross(wr, s));
    C32 rs{0.0f, 0.0f}, rp{0.0f, 0.0f};
    if (discriminant < 0.0f) {
        const float beta = sqrtf(-discriminant);
        rs = tir_coefficient(n_i * cosine, n_t * beta);
        rp = tir_coefficient(n_t * cosine, n_i * beta);
    } else {
        const float ct = sqrtf(discriminant);
        const float ds = n_i * cosine + n_t * ct;
        const float dp = n_t * cosine + n_i * ct;
        if (!(ds > 0.0f && dp > 0.0f)) return out;
        rs = {(n_i * cosine - n_t * ct) / ds, 0.0f};
        rp = {(n_t * cosine - n_i * ct) / dp, 0.0f};
        const float ts = 2.0f * n_i * cosine / ds;
        const float tp = 2.0f * n_i * cosine / dp;
        const F3 wt = unit(wi * eta + n * (eta * cosine - ct));
        out.transmitted.direction = wt;
        out.transmitted.e0 = s;
        out.transmitted.e1 = unit(cross(wt, s));
        for (unsigned j = 0; j < columns; ++j) out.transmitted.field.col[j] = {local.col[j].x * ts, local.col[j].y * tp};
        out.has_transmission = true;
    }
    for (unsigned j = 0; j < columns; ++j) out.reflected.field.col[j] = {local.col[j].x * rs, local.col[j].y * rp};
    out.valid = finite(wr) && (!out.has_transmission || finite(out.transmitted.direction));
    return out;
}

// ------------------------------------------------------------------ optical path
// A binary32 value and its rounding error (optical_path.hpp:10-60).
struct Pair {
    float hi, lo;
};
__device__ __forceinline__ Pair two_sum(float a, float b)
{
    const float s = a + b, v = s - a;
    return {s, (a - (s - v)) + (b - v)};
}
__device__ __forceinline__ Pair two_product(float a, float b)
{
    const float p = a * b;
    return {p, fmaf(a, b, -p)};
}
__device__ __forceinline__ Pair operator+(Pair a, Pair b)
{
    const Pair s = two_sum(a.hi, b.hi), t = two_sum(a.lo, b.lo);
    const Pair v = two_sum(s.lo, t.hi), w = two_sum(s.hi, v.hi);
    return two_sum(w.hi, (w.lo + v.lo) + t.lo);
}
__device__ __forceinline__ Pair operator-(Pair a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ Pair operator-(Pair a, Pair b) { return a + (-b); }
__device__ __forceinline__ Pair operator*(Pair a, Pair b)
{
    const Pair p = two_product(a.hi, b.hi);
    return two_sum(p.hi, fmaf(a.hi, b.lo, fmaf(a.lo, b.hi, p.lo)) + a.lo * b.lo);
}
__device__ __forceinline__ Pair divided(Pair a, float d)
{
    const float q = a.hi / d;
    const float residual = fmaf(-q, d, a.hi) + a.lo;
    return two_sum(q, residual / d);
}
__device__ __forceinline__ Pair pair_sqrt(Pair a)
{
    const float r = sqrtf(a.hi);
    if (r == 0.0f) return {0.0f, 0.0f};
    return two_sum(r, (fmaf(-r, r, a.hi) + a.lo) / (2.0f * r));
}
__device__ __forceinline__ Pair pair_dot(F3 a, F3 b) { return two_product(a.x, b.x) + two_product(a.y, b.y) + two_product(a.z, b.z); }
__device__ __forceinline__ Pair pair_distance(F3 a, F3 b)
{
    const Pair x = two_sum(a.x, -b.x), y = two_sum(a.y, -b.y), z = two_sum(a.z, -b.z);
    return pair_sqrt(x * x + y * y + z * z);
}

// Whole turns and a fraction in [0, 1) (phase_cycles.hpp:15-150).
struct Cycles {
    int32_t turns;
    float fraction;
};
__device__ __forceinline__ bool cycles_valid(Cycles c) { return c.fraction >= 0.0f && c.fraction < 1.0f; }
__device__ __forceinline__ bool normalize(Cycles& c, long long whole, float hi, float lo)
{
    const float integral = floorf(hi);
    whole += static_cast<long long>(integral);
    float fraction = (hi - integral) + lo;
    if (fraction < 0.0f) {
        --whole;
        fraction += 1.0f;
    }
    if (fraction >= 1.0f) { // a tiny negative plus one can round to one
        ++whole;
        fraction -= 1.0f;
    }
    if (whole < -2147483648ll || whole > 2147483647ll) return false;
    c.turns = static_cast<int32_t>(whole);
    c.fraction = fraction == 0.0f ? 0.0f : fraction;
    return true;
}
__device__ __forceinline__ bool set_parts(Cycles& c, int32_t whole, float residual)
{
    if (!(residual > -0x1p32f && residual < 0x1p32f)) return false;
    return normalize(c, static_cast<long long>(whole), residual, 0.0f);
}
__device__ __forceinline__ bool add_cycles(Cycles& c, Cycles r)
{
    if (!cycles_valid(c) || !cycles_valid(r)) return false;
    const float sum = c.fraction + r.fraction;
    const float r_virtual = sum - c.fraction;
    const float c_virtual = sum - r_virtual;
    const float error = (c.fraction - c_virtual) + (r.fraction - r_virtual);
    return normalize(c, static_cast<long long>(c.turns) + static_cast<long long>(r.turns), sum, error);
}
// q = (radius_mm 10^6 / wavelength_nm) n distance, in cycles
struct Path {
    Cycles phase;
    Pair per_unit;
};
__device__ __forceinline__ bool add_distance(Path& p, Pair distance, float n)
{
    const Pair q = (p.per_unit * Pair{n, 0.0f}) * distance;
    if (!(q.hi >= 0.0f && q.hi < 0x1p31f && fabsf(q.lo) < 0x1p31f)) return false;
    const float integral = floorf(q.hi);
    Cycles increment{0, 0.0f}, correction{0, 0.0f}, candidate = p.phase;
    if (!set_parts(increment, static_cast<int32_t>(integral), q.hi - integral) || !set_parts(correction, 0, q.lo) ||
        !add_cycles(increment, correction) || !add_cycles(candidate, increment))
        return false;
    p.phase = candidate;
    return true;
}

// ------------------------------------------------------------------ the lattice kernel
struct TraceArgs {
    Shape shape;
    F3 incident, basis_x;
    Field input; // the single-input field (columns == 1)
    float radius_mm, wavelength_nm, n_out, n_in;
    float half_extent, reference_distance, outgoing_distance;
    uint32_t width, height, columns;
};

// Per-block tallies: status per family, the two fallbacks, the trace-validation failures.
struct BlockTally {
    unsigned status[4][8];
    unsigned isect_fallback, snell_fallback, incomplete;
    unsigned long long first_problem;
};

__global__ void __launch_bounds__(kThreads) lattice_trace_kernel(const __grid_constant__ TraceArgs A,
                                                                 icp_outgoing_vertex* __restrict__ vertices,
                                                                 icp_field32* __restrict__ second,
                                                                 unsigned long long* __restrict__ tally)
{
    __shared__ BlockTally T;
    for (unsigned i = threadIdx.x; i < 32u; i += blockDim.x) (&T.status[0][0])[i] = 0u;
    if (threadIdx.x == 0) {
        T.isect_fallback = T.snell_fallback = T.incomplete = 0u;
        T.first_problem = ~0ull;
    }
    __syncthreads();

    const uint32_t count = A.width * A.height;
    const uint32_t index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index < count) {
        const bool two = A.columns == 2u;
        // One record: written whole (the reference clears every record first, then fills it),
        // validated as phase_validate_trace would, and tallied.
        auto put = [&](unsigned family, uint32_t status, uint32_t diagnostics, const Ray* ray, F3 point, Cycles cyc) {
            icp_outgoing_vertex v{};
            icp_field32 s2 = {{0.0f, 0.0f}, {0.0f, 0.0f}};
            v.status = status;
            v.diagnostics = diagnostics;
            bool bad = !(status == kValid || status == kMiss || status == kTir);
            if (status == kValid) {
                v.position_drop = store3(point);
                v.direction_drop = store3(ray->direction);
                v.basis_x = store3(ray->e0);
                const Field& f0 = ray->field.col[0];
                v.field = {{f0.x.re, f0.x.im}, {f0.y.re, f0.y.im}};
                v.optical_cycles = {cyc.turns, cyc.fraction};
                if (two) {
                    const Field& f1 = ray->field.col[1];
                    s2 = {{f1.x.re, f1.x.im}, {f1.y.re, f1.y.im}};
                }
                bad = !finite(point) || !finite(ray->direction) || !finite(ray->e0) || !cycles_valid(cyc) ||
                      !finite(ray->field.col[0]) || (two && !finite(ray->field.col[1]));
            }
            const size_t slot = size_t(family) * count + index;
            vertices[slot] = v;
            if (two) second[slot] = s2;
            atomicAdd(&T.status[family][status & 7u], 1u);
            if (diagnostics & kIsectFallback) atomicAdd(&T.isect_fallback, 1u);
            if (diagnostics & kSnellFallback) atomicAdd(&T.snell_fallback, 1u);
            if (bad) {
                atomicAdd(&T.incomplete, 1u);
                atomicMin(&T.first_problem, (unsigned long long)slot);
            }
        };
        const F3 zero{0.0f, 0.0f, 0.0f};
        const Cycles none{0, 0.0f};
        auto mark_remaining = [&](unsigned first, uint32_t status, uint32_t diagnostics) {
            for (unsigned f = first; f < 4u; ++f) put(f, status, diagnostics, nullptr, zero, none);
        };
        // emit (raindrop_paths.hpp:126-143): a leaving ray with its path to the outgoing
        // reference plane; `path` is a copy
        auto emit = [&](unsigned family, const Ray& out, F3 point, Path path, uint32_t diagnostics) {
            const Pair after = Pair{A.outgoing_distance, 0.0f} - pair_dot(point, out.direction);
            const bool fin = finite(out.field.col[0]) && (!two || finite(out.field.col[1]));
            if (!fin) return put(family, kInvalid, diagnostics, nullptr, zero, none);
            if (!add_distance(path, after, A.n_out)) return put(family, kOverflow, diagnostics, nullptr, zero, none);
            put(family, kValid, diagnostics, &out, point, path.phase);
        };

        const uint32_t ix = index % A.width, iy = index / A.width;
        const float u = (2.0f * static_cast<float>(ix) / static_cast<float>(A.width - 1) - 1.0f) * A.half_extent;
        const float v = (2.0f * static_cast<float>(iy) / static_cast<float>(A.height - 1) - 1.0f) * A.half_extent;
        const F3 w = A.incident;
        Ray active;
        active.direction = w;
        active.e0 = A.basis_x;
        active.e1 = unit(cross(w, A.basis_x));
        if (two) {
            active.field.col[0] = {{1.0f, 0.0f}, {0.0f, 0.0f}};
            active.field.col[1] = {{0.0f, 0.0f}, {1.0f, 0.0f}};
        } else {
            active.field.col[0] = A.input;
            active.field.col[1] = {{0.0f, 0.0f}, {0.0f, 0.0f}};
        }
        const F3 grid_point = (active.e0 * u + active.e1 * v) - w * A.reference_distance;
        const Hit entry = intersect(A.shape, Query{grid_point, w, 0.0f, false});
        uint32_t diagnostics = entry.diagnostics;
        if (entry.code != kCodeHit) {
            mark_remaining(0, entry.code == kCodeMiss ? kMiss : kUnresolved, diagnostics);
        } else {
            Path path;
            path.phase = {0, 0.0f};
            path.per_unit = divided(two_product(A.radius_mm, 1000000.0f), A.wavelength_nm);
            const Pair before = Pair{A.reference_distance, 0.0f} + pair_dot(entry.position, w);
            if (!add_distance(path, before, A.n_out)) {
                mark_remaining(0, kOverflow, diagnostics);
            } else {
                const Branches first = split(active, entry.normal, A.n_out, A.n_in, A.columns);
                diagnostics |= first.diagnostics;
                if (!first.valid) {
                    mark_remaining(0, kInvalid, diagnostics);
                } else {
                    emit(0, first.reflected, entry.position, path, diagnostics);
                    if (!first.has_transmission) {
                        mark_remaining(1, kTir, diagnostics);
                    } else {
                        active = first.transmitted;
                        F3 previous = entry.position;
                        for (unsigned family = 1; family < 4u; ++family) {
                            // along-ray self-hit exclusion only; the path uses the physical points
                            const Hit hit = intersect(A.shape, Query{previous, active.direction, 0x1p-17f, true});
                            diagnostics |= hit.diagnostics;
                            if (hit.code != kCodeHit) {
                                mark_remaining(family, kUnresolved, diagnostics);
                                break;
                            }
                            if (!add_distance(path, pair_distance(previous, hit.position), A.n_in)) {
                                mark_remaining(family, kOverflow, diagnostics);
                                break;
                            }
                            const Branches b = split(active, -hit.normal, A.n_in, A.n_out, A.columns);
                            diagnostics |= b.diagnostics;
                            if (!b.valid) {
                                mark_remaining(family, kInvalid, diagnostics);
                                break;
                            }
                            if (b.has_transmission) emit(family, b.transmitted, hit.position, path, diagnostics);
                            else put(family, kTir, diagnostics, nullptr, zero, none);
                            // no pruning: internal reflection continues after TIR, Brewster or a zero field
                            active = b.reflected;
                            previous = hit.position;
                        }
                    }
                }
            }
        }
    }
    __syncthreads();
    // one global add per nonzero tally: [0, 32) status, 32 / 33 fallbacks, 34 incomplete,
    // 35 smallest failing record
    for (unsigned i = threadIdx.x; i < 35u; i += blockDim.x) {
        const unsigned x = i < 32u ? (&T.status[0][0])[i] : i == 32u ? T.isect_fallback : i == 33u ? T.snell_fallback : T.incomplete;
        if (x) atomicAdd(&tally[i], (unsigned long long)x);
    }
    if (threadIdx.x == 0 && T.first_problem != ~0ull) atomicMin(&tally[35], T.first_problem);
}

// ------------------------------------------------------------------ host side
bool finite_host(float x) { return std::isfinite(x); }
float fdot(const float a[3], const float b[3]) { return std::fmaf(a[0], b[0], std::fmaf(a[1], b[1], a[2] * b[2])); }

} // namespace

// RaindropSettings::make_config (include/rainbow/raindrop_settings.hpp:19-43) for an
// unpolarised trace, with the shape either from Table I (RaindropShape::try_make) or explicit.
extern "C" int icp_raindrop_config_make(float radius_mm, int sphere, const float* coefficients, float wavelength_nm,
                                        float interior_index, const float incident_direction[3], uint32_t grid_width,
                                        uint32_t grid_height, icp_raindrop_config* out)
{
    if (!incident_direction || !out) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_raindrop_config_make: null argument");
    icp_raindrop_config c;
    std::memset(&c, 0, sizeof c);
    if (!(radius_mm > 0.0f && radius_mm <= 3.0f))
        return fail(ICP_ERR_INVALID_ARGUMENT, "radius_mm must be in (0,3]; no coefficient extrapolation is implemented.");
    if (coefficients) {
        for (int k = 0; k < 8; ++k) {
            if (!finite_host(coefficients[k])) return fail(ICP_ERR_INVALID_ARGUMENT, "Shape coefficients must be finite.");
            c.coefficients[k] = coefficients[k];
        }
    } else {
        static const float radii[6] = {0.4f, 1.0f, 1.5f, 2.0f, 2.5f, 3.0f};
        static const float table[6][8] = {
            {0, 0, 0, 0, 0, 0, 0, 0},
            {-0.0131f, -0.0120f, -0.0376f, -0.0096f, -0.0004f, 0.0015f, 0.0005f, 0},
            {-0.0282f, -0.0230f, -0.0779f, -0.0175f, 0.0021f, 0.0046f, 0.0011f, -0.0006f},
            {-0.0458f, -0.0335f, -0.1211f, -0.0227f, 0.0083f, 0.0089f, 0.0012f, -0.0021f},
            {-0.0644f, -0.0416f, -0.1629f, -0.0246f, 0.0176f, 0.0131f, 0.0002f, -0.0044f},
            {-0.0840f, -0.0480f, -0.2034f, -0.0237f, 0.0297f, 0.0166f, -0.0021f, -0.0072f}};
        if (!sphere && radius_mm > radii[0]) {
            unsigned hi = 1;
            while (hi < 5 && radius_mm > radii[hi]) ++hi;
            const float t = (radius_mm - radii[hi - 1]) / (radii[hi] - radii[hi - 1]);
            for (unsigned k = 0; k < 8; ++k)
                c.coefficients[k] = std::fmaf(t, table[hi][k] - table[hi - 1][k], table[hi - 1][k]);
        }
    }
    // conservative bounding radii from |T_n| <= 1, rounded outwards
    const float inf = INFINITY;
    float abs_sum = 0.0f;
    for (unsigned k = 1; k < 8; ++k) abs_sum = std::nextafterf(abs_sum + std::fabs(c.coefficients[k]), inf);
    const float center = 1.0f + c.coefficients[0];
    c.inner_radius = std::nextafterf(center - abs_sum - 0x1p-20f, -inf);
    c.outer_radius = std::nextafterf(center + abs_sum + 0x1p-20f, inf);
    if (!(c.inner_radius > 0.0f))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Shape coefficients leave no positive inner radius.");
    if (!(wavelength_nm >= 380.0f && wavelength_nm <= 830.0f))
        return fail(ICP_ERR_INVALID_ARGUMENT, "wavelength_nm must be in [380,830] for this implementation.");
    if (!(interior_index >= 1.0f && interior_index <= 2.0f))
        return fail(ICP_ERR_INVALID_ARGUMENT, "interior_index must be in [1,2]; exterior_index is 1.");
    if (grid_width < 2 || grid_height < 2 || uint64_t(grid_width) * grid_height > uint64_t(0xffffffffu) / 4)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid grid dimensions or 32-bit path-major index overflow.");
    const float* d = incident_direction;
    const float len = std::sqrt(fdot(d, d));
    if (!(finite_host(d[0]) && finite_host(d[1]) && finite_host(d[2])) || !std::isfinite(len) || !(len > 0.0f))
        return fail(ICP_ERR_INVALID_ARGUMENT, "incident_direction must be a finite nonzero vector.");
    const float w[3] = {d[0] / len, d[1] / len, d[2] / len};
    // TransverseFrame::from_direction (include/rainbow/vec3.hpp): e0 from the z axis, or the x
    // axis when the direction is within |w_z| >= 0.9 of it
    const float axis[3] = {std::fabs(w[2]) < 0.9f ? 0.0f : 1.0f, 0.0f, std::fabs(w[2]) < 0.9f ? 1.0f : 0.0f};
    const float wa = fdot(w, axis);
    const float e[3] = {axis[0] - w[0] * wa, axis[1] - w[1] * wa, axis[2] - w[2] * wa};
    const float el = std::sqrt(fdot(e, e));
    c.incident_direction = {w[0], w[1], w[2]};
    c.incident_basis_x = {e[0] / el, e[1] / el, e[2] / el};
    c.incident_field = {{1.0f, 0.0f}, {0.0f, 0.0f}};
    c.radius_mm = radius_mm;
    c.wavelength_nm = wavelength_nm;
    c.exterior_index = 1.0f;
    c.interior_index = interior_index;
    c.grid_half_extent = c.outer_radius * 1.01f;
    c.reference_distance = c.outgoing_reference_distance = 2.0f * c.outer_radius;
    c.grid_width = grid_width;
    c.grid_height = grid_height;
    *out = c;
    return ok();
}

extern "C" int icp_lattice_trace(icp_context* ctx, const icp_raindrop_config* config, icp_outgoing_vertex* d_vertices,
                                 icp_field32* d_second_fields, icp_lattice_stats* stats)
{
    if (!ctx || !config || !d_vertices) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_lattice_trace: null argument");
    const icp_raindrop_config& c = *config;
    if (c.grid_width < 2 || c.grid_height < 2 || uint64_t(c.grid_width) * c.grid_height > uint64_t(0xffffffffu) / 4)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid grid dimensions or 32-bit path-major index overflow.");
    bool fin = true;
    for (int k = 0; k < 8; ++k) fin = fin && std::isfinite(c.coefficients[k]);
    const float scalars[] = {c.inner_radius, c.outer_radius, c.incident_direction.x, c.incident_direction.y,
                             c.incident_direction.z, c.incident_basis_x.x, c.incident_basis_x.y, c.incident_basis_x.z,
                             c.radius_mm, c.wavelength_nm, c.exterior_index, c.interior_index, c.grid_half_extent,
                             c.reference_distance, c.outgoing_reference_distance, c.incident_field.x.real,
                             c.incident_field.x.imag, c.incident_field.y.real, c.incident_field.y.imag};
    for (float x : scalars) fin = fin && std::isfinite(x);
    if (!fin) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_lattice_trace: the configuration holds a non-finite value");
    if (!(c.inner_radius > 0.0f && c.outer_radius >= c.inner_radius && c.radius_mm > 0.0f && c.wavelength_nm > 0.0f))
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_lattice_trace: invalid shape radii, radius or wavelength");

    TraceArgs A;
    std::memset(&A, 0, sizeof A);
    for (int k = 0; k < 8; ++k) A.shape.c[k] = c.coefficients[k];
    A.shape.inner = c.inner_radius;
    A.shape.outer = c.outer_radius;
    A.shape.last = 1;
    for (unsigned k = 2; k < 8; ++k)
        if (c.coefficients[k] != 0.0f) A.shape.last = k;
    A.incident = {c.incident_direction.x, c.incident_direction.y, c.incident_direction.z};
    A.basis_x = {c.incident_basis_x.x, c.incident_basis_x.y, c.incident_basis_x.z};
    A.input = {{c.incident_field.x.real, c.incident_field.x.imag}, {c.incident_field.y.real, c.incident_field.y.imag}};
    A.radius_mm = c.radius_mm;
    A.wavelength_nm = c.wavelength_nm;
    A.n_out = c.exterior_index;
    A.n_in = c.interior_index;
    A.half_extent = c.grid_half_extent;
    A.reference_distance = c.reference_distance;
    A.outgoing_distance = c.outgoing_reference_distance;
    A.width = c.grid_width;
    A.height = c.grid_height;
    A.columns = d_second_fields ? 2u : 1u;

    const uint32_t count = c.grid_width * c.grid_height;
    ICP_CUDA(cudaSetDevice(ctx->device));
    ICP_CUDA(ctx->lattice.ensure(36 * sizeof(unsigned long long)));
    auto* tally = static_cast<unsigned long long*>(ctx->lattice.ptr);
    ICP_CUDA(cudaMemsetAsync(tally, 0, 35 * sizeof(unsigned long long), ctx->stream));
    ICP_CUDA(cudaMemsetAsync(tally + 35, 0xff, sizeof(unsigned long long), ctx->stream));
    const unsigned blocks = (count + kThreads - 1) / kThreads;
    lattice_trace_kernel<<<blocks, kThreads, 0, ctx->stream>>>(A, d_vertices, d_second_fields, tally);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    unsigned long long h[36];
    ICP_CUDA(cudaMemcpyAsync(h, tally, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    ICP_CUDA(cudaStreamSynchronize(ctx->stream));
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        for (int f = 0; f < 4; ++f)
            for (int s = 0; s < 8; ++s) stats->status_counts[f][s] = h[f * 8 + s];
        stats->intersection_fallbacks = h[32];
        stats->snell_fallbacks = h[33];
        stats->incomplete = h[34];
        stats->first_problem = h[35];
    }
    return ok();
}
