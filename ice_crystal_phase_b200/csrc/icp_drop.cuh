// icp_drop.cuh -- axisymmetric water-drop geometry for the drop trace kernel (sm_100a).
//
// Shape (include/rainbow/raindrop_shape.hpp:11-100): r/a = 1 + sum_{n=0}^{7} c_n T_n(mu), with
// mu = cos(chi) and chi measured from the particle's -y axis (gravity), coordinates in units
// of the equal-volume radius a.  R(mu) and dR/dmu use the Chebyshev recurrence, so no acos and
// no division by sin(chi) is needed at the poles.
//
// Intersection: the reference brackets f = |p| - R(mu) with outward-rounded intervals and
// polishes with safeguarded Newton (raindrop_intersection.hpp:203-382).  Here the drop is a
// convex body, so its gauge rho(p) = |p| / R(mu(p)) is a convex function along any line.  On a
// convex function Newton's method started where rho >= 1 moves monotonically towards the
// nearest root without overshoot: started on an enclosing spheroid it converges to
// the entry point (from before the body) or to the exit point (from beyond it), and a line
// that misses the body shows up as rho' >= 0 while rho > 1.  A point that rounding left
// slightly off the surface does not change which root is reached.  Spheres (c_1..c_7 = 0) use
// the closed-form quadratic.
#pragma once
#include "icp_device.cuh"

namespace icp {

template <class R> struct DropShape {
    R c[8];
    R m[8];      // binary32 path: R(mu) = sum_k m_k mu^k (the series in monomial form)
    R md[7];     //                dR/dmu = sum_k md_k mu^k
    R r_out;     // conservative bounding radius (outer sphere)
    R r_center;  // 1 + c_0 (the sphere radius when c_1..c_7 vanish)
    R ea_inv, eb_inv, ey0; // enclosing spheroid (x^2 + z^2) / A^2 + (y - y0)^2 / B^2 <= 1: 1/A, 1/B, y0
    bool sphere;
};

// R(mu) and dR/dmu.  binary64: the Chebyshev recurrence of the reference (raindrop_shape.hpp:
// 70-84); binary32: Horner on the monomial form (13 FMAs; the coefficients are converted in
// binary64 on the host, and |mu| <= 1 keeps the cancellation below the binary32 rounding).
template <class R> __device__ __forceinline__ R drop_radius(const DropShape<R>& S, R mu, R& dr)
{
    if constexpr (sizeof(R) == 4) {
        R r = S.m[7], d = S.md[6];
#pragma unroll
        for (int k = 6; k >= 0; --k) r = fmaf(r, mu, S.m[k]);
#pragma unroll
        for (int k = 5; k >= 0; --k) d = fmaf(d, mu, S.md[k]);
        dr = d;
        return r;
    }
    R prev = R(1), cur = mu, dprev = R(0), dcur = R(1);
    R radius = R(1) + S.c[0] + S.c[1] * mu;
    R deriv = S.c[1];
#pragma unroll
    for (int n = 2; n < 8; ++n) {
        const R next = R(2) * mu * cur - prev;
        const R dnext = R(2) * cur + R(2) * mu * dcur - dprev;
        radius += S.c[n] * next;
        deriv += S.c[n] * dnext;
        prev = cur;
        cur = next;
        dprev = dcur;
        dcur = dnext;
    }
    dr = deriv;
    return radius;
}

// Outward surface normal at p (gradient of |p| - R(mu), raindrop_shape.hpp:92-100), unit.
template <class R> __device__ __forceinline__ V3<R> drop_normal(const DropShape<R>& S, V3<R> p)
{
    if (S.sphere) return unit(p);
    const R r = sqrt_r(dot(p, p));
    const V3<R> u = p * (R(1) / r);
    const R mu = -u.y;
    R dr;
    (void)drop_radius(S, mu, dr);
    const V3<R> g = u - (v3(R(0), R(-1), R(0)) - u * mu) * (dr / r);
    return unit(g);
}

// Gauge rho(p + t d) - 1 and its t-derivative.
template <class R> __device__ __forceinline__ R gauge(const DropShape<R>& S, V3<R> p, V3<R> d, R& dh)
{
    const R r = sqrt_r(dot(p, p));
    const R inv_r = R(1) / r;
    const R rd = dot(p, d) * inv_r;             // d|p|/dt
    const R mu = -p.y * inv_r;
    const R dmu = (-d.y - mu * rd) * inv_r;     // dmu/dt
    R dR;
    const R Rm = drop_radius(S, mu, dR);
    const R invR = R(1) / Rm;
    dh = (rd - r * invR * dR * dmu) * invR;
    return r * invR - R(1);
}

// Roots of |p + t d| = rad (d unit): false when the line misses the sphere.
template <class R> __device__ __forceinline__ bool sphere_roots(V3<R> p, V3<R> d, R rad, R& t0, R& t1)
{
    const R b = dot(p, d);
    const R c = dot(p, p) - rad * rad;
    const R disc = b * b - c;
    if (!(disc >= R(0))) return false;
    const R q = sqrt_r(disc);
    t0 = -b - q;
    t1 = -b + q;
    return true;
}

// Roots of the line p + t d with the drop's enclosing spheroid (the Newton start: much closer
// to an oblate drop's surface than the outer sphere, so fewer gauge evaluations per root).
template <class R> __device__ __forceinline__ bool spheroid_roots(const DropShape<R>& S, V3<R> p, V3<R> d, R& t0, R& t1)
{
    const V3<R> P = v3(p.x * S.ea_inv, (p.y - S.ey0) * S.eb_inv, p.z * S.ea_inv);
    const V3<R> D = v3(d.x * S.ea_inv, d.y * S.eb_inv, d.z * S.ea_inv);
    const R a = dot(D, D), b = dot(P, D), c = dot(P, P) - R(1);
    const R disc = b * b - a * c;
    if (!(disc >= R(0))) return false;
    const R q = sqrt_r(disc), ia = R(1) / a;
    t0 = (-b - q) * ia;
    t1 = (-b + q) * ia;
    return true;
}

constexpr int kNewtonMax = 40;

// Newton on the smooth gauge converges quadratically: successive steps s_{k-1}, s_k estimate
// the constant C = s_k / s_{k-1}^2 of e_{k+1} = C e_k^2, so the error left after applying s_k is
// about s_k^3 / s_{k-1}^2.  When that is below a sixteenth of the rounding tolerance of t the
// root is reached without one more gauge evaluation (which would only confirm a step below tol).
template <class R> __device__ __forceinline__ bool newton_done(R step, R prev_step, R tol)
{
    const R a = rabs(step);
    return prev_step != R(0) && a * a * a <= R(0.0625) * tol * prev_step * prev_step;
}

// Intersection of the line q + t w (w unit) with the drop: entering from outside, the first
// root; leaving from a surface point, the far root.  Both run one Newton loop on the gauge from
// the bounding sphere (the near root entering, the far root leaving), so lanes entering and
// leaving the drop execute the same instructions.  False only for an entering line that misses.
template <class R>
__device__ __forceinline__ bool drop_intersect(const DropShape<R>& S, V3<R> q, V3<R> w, bool entering, R& t,
                                               unsigned& iters)
{
    R t0, t1;
    if (!(S.sphere ? sphere_roots(q, w, S.r_center, t0, t1) : spheroid_roots(S, q, w, t0, t1))) {
        t = R(0);
        return !entering;
    }
    if (S.sphere) {
        t = entering ? t0 : rmax(t1, R(0));
        return !entering || t0 >= R(0);
    }
    t = rmax(entering ? t0 : t1, R(0));
    const R sgn = entering ? R(-1) : R(1);
    R prev_h = R(1e30), prev_step = R(0);
    for (int it = 0; it < kNewtonMax; ++it) {
        R dh;
        const R h = gauge(S, q + w * t, w, dh);
        ++iters;
        if (h <= R(0)) return true;           // converged onto the root from outside the drop
        if (!(sgn * dh > R(0))) return !entering; // entering: non-decreasing while outside -> miss;
                                                  // leaving: degenerate tangent chord, stay at t
        const R step = h / dh;
        t -= step;
        if (entering ? (t > t1) : (t <= R(0))) {
            if (!entering) t = R(0);
            return !entering;
        }
        const R tol = R(4) * Eps<R>::eps * rmax(R(1), rabs(t));
        if (!(h < prev_h) || rabs(step) <= tol) return true;
        if (newton_done(step, prev_step, tol)) return true;
        prev_h = h;
        prev_step = step;
    }
    return true;
}

// First surface point along the line from an exterior point: t of the entry, false on a miss.
// `iters` counts the gauge evaluations (the dominant arithmetic of a non-spherical drop).
template <class R> __device__ __forceinline__ bool drop_entry(const DropShape<R>& S, V3<R> o, V3<R> d, R& t,
                                                              unsigned& iters)
{
    R t0, t1;
    if (S.sphere) {
        if (!sphere_roots(o, d, S.r_center, t0, t1)) return false;
        t = t0;
        return t0 >= R(0);
    }
    if (!spheroid_roots(S, o, d, t0, t1)) return false;
    t = rmax(t0, R(0));
    R prev_h = R(1e30), prev_step = R(0);
    for (int it = 0; it < kNewtonMax; ++it) {
        R dh;
        const R h = gauge(S, o + d * t, d, dh);
        ++iters;
        if (h <= R(0)) return true;          // converged from outside to the entry root
        if (!(dh < R(0))) return false;       // convex and non-decreasing while outside: miss
        const R step = h / dh;                // negative
        t -= step;
        if (t > t1) return false;
        const R tol = R(4) * Eps<R>::eps * rmax(R(1), rabs(t));
        if (!(h < prev_h) || rabs(step) <= tol) return true;
        if (newton_done(step, prev_step, tol)) return true;
        prev_step = step;
        prev_h = h;
    }
    return true;
}

// Exit point along an interior chord that starts on (or rounding-close to) the surface.
template <class R> __device__ __forceinline__ R drop_exit(const DropShape<R>& S, V3<R> p, V3<R> d, unsigned& iters)
{
    R t0, t1;
    if (S.sphere) {
        // larger root of |p + t d| = R; p may be off the sphere by rounding
        if (!sphere_roots(p, d, S.r_center, t0, t1)) return R(0);
        return rmax(t1, R(0));
    }
    if (!sphere_roots(p, d, S.r_out, t0, t1)) return R(0);
    R t = rmax(t1, R(0));
    R prev_h = R(1e30);
    for (int it = 0; it < kNewtonMax; ++it) {
        R dh;
        const R h = gauge(S, p + d * t, d, dh);
        ++iters;
        if (h <= R(0)) break;                 // reached the exit root from beyond it
        if (!(dh > R(0))) break;              // degenerate tangent chord: stay at t
        const R step = h / dh;                // positive
        t -= step;
        if (t <= R(0)) return R(0);
        if (!(h < prev_h) || step <= R(4) * Eps<R>::eps * rmax(R(1), t)) break;
        prev_h = h;
    }
    return t;
}

} // namespace icp
