// icp_drop_host.hpp -- host-side binary64 inputs of a drop record: shape coefficients, the
// projected area, the water index and the incident frame.  All run once per record on the
// CPU; the projected-area integral stays in binary64 on the CPU by design.
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <vector>

#include "icp_host_math.hpp"

namespace icp::host {

// ---------------------------------------------------------------- drop shape
// Radial cosine series r/a = 1 + sum_n c_n cos(n chi), chi from the particle's -y axis, with
// coefficients interpolated in radius from Sadeghi et al. (2012) Table I, as the reference's
// drop model does (include/rainbow/raindrop_shape.hpp:22-67): binary32 coefficients, linear
// interpolation between tabulated radii, no extrapolation beyond 3 mm, spheres at <= 0.4 mm.
struct DropShapeHost {
    float c[8] = {};
    float inner = 1.0f, outer = 1.0f; // conservative bounding radii (|T_n| <= 1)
};

// Conservative inner / outer radii from |T_n(mu)| <= 1, rounded outwards.
inline void bounding_radii(DropShapeHost& s)
{
    const float inf = std::numeric_limits<float>::infinity();
    float abs_sum = 0.0f;
    for (unsigned k = 1; k < 8; ++k) abs_sum = std::nextafterf(abs_sum + std::fabs(s.c[k]), inf);
    const float center = 1.0f + s.c[0];
    s.inner = std::nextafterf(center - abs_sum - 0x1p-20f, -inf);
    s.outer = std::nextafterf(center + abs_sum + 0x1p-20f, inf);
}

inline bool drop_shape_from_radius(float radius_mm, bool sphere, DropShapeHost& out)
{
    if (!(radius_mm > 0.0f && radius_mm <= 3.0f)) return false;
    static const float radii[6] = {0.4f, 1.0f, 1.5f, 2.0f, 2.5f, 3.0f};
    static const float table[6][8] = {
        {0, 0, 0, 0, 0, 0, 0, 0},
        {-0.0131f, -0.0120f, -0.0376f, -0.0096f, -0.0004f, 0.0015f, 0.0005f, 0},
        {-0.0282f, -0.0230f, -0.0779f, -0.0175f, 0.0021f, 0.0046f, 0.0011f, -0.0006f},
        {-0.0458f, -0.0335f, -0.1211f, -0.0227f, 0.0083f, 0.0089f, 0.0012f, -0.0021f},
        {-0.0644f, -0.0416f, -0.1629f, -0.0246f, 0.0176f, 0.0131f, 0.0002f, -0.0044f},
        {-0.0840f, -0.0480f, -0.2034f, -0.0237f, 0.0297f, 0.0166f, -0.0021f, -0.0072f}};
    DropShapeHost s;
    if (!sphere && radius_mm > radii[0]) {
        unsigned hi = 1;
        while (hi < 5 && radius_mm > radii[hi]) ++hi;
        const float t = (radius_mm - radii[hi - 1]) / (radii[hi] - radii[hi - 1]);
        for (unsigned k = 0; k < 8; ++k) s.c[k] = std::fmaf(t, table[hi][k] - table[hi - 1][k], table[hi - 1][k]);
    }
    bounding_radii(s);
    out = s;
    return true;
}

// R(mu), dR/dmu, d2R/dmu2 by Chebyshev recurrences.
inline double drop_radius(const double c[8], double mu, double* d1 = nullptr, double* d2 = nullptr)
{
    double t0 = 1, t1 = mu, p0 = 0, p1 = 1, q0 = 0, q1 = 0;
    double r = 1 + c[0] + c[1] * mu, rp = c[1], rpp = 0;
    for (unsigned n = 2; n < 8; ++n) {
        const double t = 2 * mu * t1 - t0, p = 2 * t1 + 2 * mu * p1 - p0, q = 4 * p1 + 2 * mu * q1 - q0;
        r += c[n] * t;
        rp += c[n] * p;
        rpp += c[n] * q;
        t0 = t1; t1 = t; p0 = p1; p1 = p; q0 = q1; q1 = q;
    }
    if (d1) *d1 = rp;
    if (d2) *d2 = rpp;
    return r;
}

// Strict convexity of the surface of revolution, sampled densely in mu: r > 0,
// G = r + mu r' > 0 and Q = r^2 + 2(1-mu^2) r'^2 - r[(1-mu^2) r'' - mu r'] > 0 (curvatures of
// the meridian and of the parallel).  The reference proves the same conditions with
// outward-rounded interval arithmetic (src/projected_area.cpp:45-87); here a 20001-point
// sampling plus a relative margin is used.
inline bool drop_convex(const double c[8])
{
    for (int k = 0; k <= 20000; ++k) {
        const double mu = -1.0 + 2.0 * k / 20000.0;
        double rp, rpp;
        const double r = drop_radius(c, mu, &rp, &rpp);
        const double s2 = 1 - mu * mu;
        const double g = r + mu * rp;
        const double q = r * r + 2 * s2 * rp * rp - r * (s2 * rpp - mu * rp);
        if (!(r > 1e-6) || !(g > 1e-6) || !(q > 1e-6)) return false;
    }
    return true;
}

// Gauss-Legendre nodes / weights on [-1,1] from Newton's method on P_n (no tables).
struct GaussLegendre {
    std::vector<double> x, w;
    explicit GaussLegendre(int n)
    {
        x.resize(n);
        w.resize(n);
        for (int i = 0; i < n; ++i) {
            double z = std::cos(kPi * (i + 0.75) / (n + 0.5)), pp = 0;
            for (int it = 0; it < 100; ++it) {
                double p1 = 1, p2 = 0;
                for (int j = 1; j <= n; ++j) {
                    const double p3 = p2;
                    p2 = p1;
                    p1 = ((2.0 * j - 1) * z * p2 - (j - 1.0) * p3) / j;
                }
                pp = n * (z * p1 - p2) / (z * z - 1);
                const double dz = p1 / pp;
                z -= dz;
                if (std::fabs(dz) < 1e-16) break;
            }
            x[i] = z;
            w[i] = 2 / ((1 - z * z) * pp * pp);
        }
    }
};

// Projected area of the convex drop along unit k (mm^2).  Half the integral of |k . n| dA
// over the surface; the azimuthal integral is done in closed form,
//   int_0^2pi |a cos(psi) + b| dpsi = 2 pi |b|  (|a| <= |b|),  4 (sqrt(a^2-b^2) + |b| asin(|b|/|a|))  otherwise,
// and the polar integral by adaptive 16/32-point Gauss-Legendre bisection (the integrand has
// square-root kinks at the terminator).  Spheres: pi (1+c0)^2 a^2.
struct ProjectedArea {
    double area_mm2 = 0, error_estimate_mm2 = 0;
    uint32_t panels = 0;
    bool sphere = false;
};
inline ProjectedArea drop_projected_area(const double c[8], double radius_mm, const double k_in[3])
{
    ProjectedArea out;
    const double norm = std::hypot(k_in[0], k_in[1], k_in[2]);
    if (!(norm > 0) || !finite(norm) || !(radius_mm > 0)) throw std::invalid_argument("Invalid projected-area input.");
    bool sphere = true;
    for (int n = 1; n < 8; ++n) sphere = sphere && c[n] == 0;
    if (sphere) {
        const double r = 1 + c[0];
        out.area_mm2 = kPi * r * r * radius_mm * radius_mm;
        out.sphere = true;
        return out;
    }
    if (!drop_convex(c)) throw std::invalid_argument("Projected area: nonconvex or invalid radial shape.");
    const double kt = std::hypot(k_in[0], k_in[2]) / norm, ky = std::fabs(k_in[1]) / norm;
    auto f = [&](double chi) {
        const double mu = std::cos(chi), sn = std::sin(chi);
        double rp;
        const double r = drop_radius(c, mu, &rp);
        const double a = std::fabs(kt * r * sn * sn * (r + mu * rp));
        const double b = std::fabs(ky * r * sn * (mu * r - sn * sn * rp));
        const double j = a <= b ? 2 * kPi * b : 4 * (std::sqrt((a - b) * (a + b)) + b * std::asin(b / a));
        return 0.5 * j;
    };
    static const GaussLegendre g16(16), g32(32);
    auto panel = [&](double lo, double hi, const GaussLegendre& g) {
        const double m = 0.5 * (lo + hi), h = 0.5 * (hi - lo);
        double s = 0;
        for (size_t i = 0; i < g.x.size(); ++i) s += g.w[i] * f(m + h * g.x[i]);
        return s * h;
    };
    struct P { double lo, hi; };
    std::vector<P> todo;
    for (int i = 0; i < 64; ++i) todo.push_back({kPi * i / 64, kPi * (i + 1) / 64});
    double total = 0, err = 0;
    KahanSum sum;
    while (!todo.empty()) {
        const P p = todo.back();
        todo.pop_back();
        const double a = panel(p.lo, p.hi, g16), b = panel(p.lo, p.hi, g32);
        if (std::fabs(a - b) <= 1e-15 * std::max(1.0, std::fabs(b)) || p.hi - p.lo < 1e-9) {
            sum.add(b);
            err += std::fabs(a - b);
            ++out.panels;
            if (out.panels > 1000000) throw std::runtime_error("Projected-area quadrature did not converge.");
        } else {
            const double mid = 0.5 * (p.lo + p.hi);
            todo.push_back({mid, p.hi});
            todo.push_back({p.lo, mid});
        }
    }
    total = sum.value;
    out.area_mm2 = total * radius_mm * radius_mm;
    out.error_estimate_mm2 = err * radius_mm * radius_mm;
    return out;
}

// ---------------------------------------------------------------- water index
// IAPWS R9-97 (1997) refractive index of water (absolute, real), from the published
// formulation: (n^2-1)/(n^2+2)/rho* = a0 + a1 rho* + a2 T* + a3 lambda*^2 T* + a4/lambda*^2
//   + a5/(lambda*^2 - l_uv^2) + a6/(lambda*^2 - l_ir^2) + a7 rho*^2,
// rho* = rho/1000 kg m^-3, T* = T/273.15 K, lambda* = lambda/0.589 um.
inline double water_index_r9_97(double wavelength_nm, double temperature_k, double density)
{
    static const double a[8] = {0.244257733, 9.74634476e-3, -3.73234996e-3, 2.68678472e-4,
                                1.58920570e-3, 2.45934259e-3, 0.900704920, -1.66626219e-2};
    const double luv = 0.2292020, lir = 5.432937;
    const double r = density / 1000.0, t = temperature_k / 273.15, l = wavelength_nm / 589.0, l2 = l * l;
    const double rhs = a[0] + a[1] * r + a[2] * t + a[3] * l2 * t + a[4] / l2 + a[5] / (l2 - luv * luv) +
                       a[6] / (l2 - lir * lir) + a[7] * r * r;
    const double x = r * rhs;
    return std::sqrt((1 + 2 * x) / (1 - x));
}
// ---------------------------------------------------------------- IAPWS-95 liquid density
// Density of liquid water from the IAPWS-95 equation of state (IAPWS R6-95(2018); Wagner & Pruss,
// J. Phys. Chem. Ref. Data 31, 387 (2002)): p = rho R T (1 + delta dphi_r/ddelta), delta =
// rho / 322 kg m^-3, tau = 647.096 K / T, R = 461.51805 J kg^-1 K^-1, with all 56 terms of the
// residual Helmholtz energy (Table 2 of the release: 7 polynomial, 44 exponential, 3 Gaussian,
// 2 non-analytic), inverted for rho on the liquid branch by bisection.  The reference solves
// the same equation (src/water_refractive_index.cpp:84-187); the density it reports is a
// function of its operation order, so this evaluation keeps that order: terms in table order,
// each as ((n delta^d) tau^t) e^(-delta^c) times its delta-derivative factor, added with the
// compensated (Neumaier) sum; bisection on [970, 1060] kg m^-3 until the bracket is at most
// 2e-10 wide, then the end with the smaller pressure residual.
namespace iapws95 {

struct Term {
    double n, t;
    int d, c; // c = 0: polynomial term (no exponential)
};
// n_i, t_i, d_i, c_i of the polynomial and exponential terms (IAPWS R6-95 Table 2, i = 1..51)
inline const Term* terms()
{
    static const Term k[51] = {
        {0.12533547935523e-1, -0.5, 1, 0},    {0.78957634722828e1, 0.875, 1, 0},   {-0.87803203303561e1, 1.0, 1, 0},
        {0.31802509345418, 0.5, 2, 0},        {-0.26145533859358, 0.75, 2, 0},     {-0.78199751687981e-2, 0.375, 3, 0},
        {0.88089493102134e-2, 1.0, 4, 0},     {-0.66856572307965, 4.0, 1, 1},      {0.20433810950965, 6.0, 1, 1},
        {-0.66212605039687e-4, 12.0, 1, 1},   {-0.19232721156002, 1.0, 2, 1},      {-0.25709043003438, 5.0, 2, 1},
        {0.16074868486251, 4.0, 3, 1},        {-0.40092828925807e-1, 2.0, 4, 1},   {0.39343422603254e-6, 13.0, 4, 1},
        {-0.75941377088144e-5, 9.0, 5, 1},    {0.56250979351888e-3, 3.0, 7, 1},    {-0.15608652257135e-4, 4.0, 9, 1},
        {0.11537996422951e-8, 11.0, 10, 1},   {0.36582165144204e-6, 4.0, 11, 1},   {-0.13251180074668e-11, 13.0, 13, 1},
        {-0.62639586912454e-9, 1.0, 15, 1},   {-0.10793600908932, 7.0, 1, 2},      {0.17611491008752e-1, 1.0, 2, 2},
        {0.22132295167546, 9.0, 2, 2},        {-0.40247669763528, 10.0, 2, 2},     {0.58083399985759, 10.0, 3, 2},
        {0.49969146990806e-2, 3.0, 4, 2},     {-0.31358700712549e-1, 7.0, 4, 2},   {-0.74315929710341, 10.0, 4, 2},
        {0.47807329915480, 10.0, 5, 2},       {0.20527940895948e-1, 6.0, 6, 2},    {-0.13636435110343, 10.0, 6, 2},
        {0.14180634400617e-1, 10.0, 7, 2},    {0.83326504880713e-2, 1.0, 9, 2},    {-0.29052336009585e-1, 2.0, 9, 2},
        {0.38615085574206e-1, 3.0, 9, 2},     {-0.20393486513704e-1, 4.0, 9, 2},   {-0.16554050063734e-2, 8.0, 9, 2},
        {0.19955571979541e-2, 6.0, 10, 2},    {0.15870308324157e-3, 9.0, 10, 2},   {-0.16388568342530e-4, 8.0, 12, 2},
        {0.43613615723811e-1, 16.0, 3, 3},    {0.34994005463765e-1, 22.0, 4, 3},   {-0.76788197844621e-1, 23.0, 4, 3},
        {0.22446277332006e-1, 23.0, 5, 3},    {-0.62689710414685e-4, 10.0, 14, 4}, {-0.55711118565645e-9, 50.0, 3, 6},
        {-0.19905718354408, 44.0, 6, 6},      {0.31777497330738, 46.0, 6, 6},      {-0.11841182425981, 50.0, 6, 6}};
    return k;
}

// Compensated sum (Neumaier 1974): the rounding error of each addition is carried separately.
struct NSum {
    double s = 0.0, e = 0.0;
    void add(double x)
    {
        const double t = s + x;
        e += std::fabs(s) >= std::fabs(x) ? (s - t) + x : (x - t) + s;
        s = t;
    }
    double value() const { return s + e; }
};

// delta * d(phi_r)/d(delta)
inline double delta_phir_delta(double delta, double tau)
{
    NSum sum;
    const Term* k = terms();
    for (int i = 0; i < 51; ++i) {
        const Term& a = k[i];
        const double dc = a.c ? std::pow(delta, double(a.c)) : 0.0;
        const double term = a.n * std::pow(delta, double(a.d)) * std::pow(tau, a.t) * (a.c ? std::exp(-dc) : 1.0);
        sum.add(term * (double(a.d) - double(a.c) * dc));
    }
    // Gaussian bell terms i = 52..54: d = 3, epsilon = 1 (n, t, alpha, beta, gamma)
    static const double gauss[3][5] = {{-0.31306260323435e2, 0.0, 20.0, 150.0, 1.21},
                                       {0.31546140237781e2, 1.0, 20.0, 150.0, 1.21},
                                       {-0.25213154341695e4, 4.0, 20.0, 250.0, 1.25}};
    for (const auto& g : gauss) {
        const double x = delta - 1.0, y = tau - g[4];
        const double term = g[0] * delta * delta * delta * std::pow(tau, g[1]) * std::exp(-g[2] * x * x - g[3] * y * y);
        sum.add(term * (3.0 - 2.0 * g[2] * delta * x));
    }
    // non-analytic terms i = 55, 56 (n, b, C, D) with a = 3.5, beta = 0.3, A = 0.32, B = 0.2; the
    // liquid bracket stays far from delta = 1, where their derivatives need no special case
    static const double crit[2][4] = {{-0.14874640856724, 0.85, 28.0, 700.0}, {0.31806110878444, 0.95, 32.0, 800.0}};
    const double x = delta - 1.0, x2 = x * x;
    const double A = 0.32, B = 0.2, ea = 3.5, eb = 0.3;
    const double theta = 1.0 - tau + A * std::pow(x2, 1.0 / (2.0 * eb));
    const double theta_d = A / eb * x * std::pow(x2, 1.0 / (2.0 * eb) - 1.0);
    const double dist = theta * theta + B * std::pow(x2, ea);
    const double dist_d = 2.0 * theta * theta_d + 2.0 * B * ea * x * std::pow(x2, ea - 1.0);
    for (const auto& v : crit) {
        const double psi = std::exp(-v[2] * x2 - v[3] * (tau - 1.0) * (tau - 1.0));
        const double term = v[0] * delta * std::pow(dist, v[1]) * psi;
        sum.add(term * (1.0 + delta * (v[1] * dist_d / dist - 2.0 * v[2] * x)));
    }
    return sum.value();
}

inline double pressure(double temperature_k, double density)
{
    const double R = 461.51805, Tc = 647.096, rhoc = 322.0; // the release's constants
    return density * R * temperature_k * (1.0 + delta_phir_delta(density / rhoc, Tc / temperature_k));
}

} // namespace iapws95

// Liquid density (kg m^-3) at T (K) and p (Pa); throws std::runtime_error where the reference's
// solve fails (no bracket, nonfinite pressure, residual above 0.02 Pa, no convergence).  The
// pressure residual of the returned density and the final bracket width go to *residual_pa and
// *bracket_width when given.
inline double water_density(double temperature_k, double pressure_pa, double* residual_pa = nullptr,
                            double* bracket_width = nullptr)
{
    double lo = 970.0, hi = 1060.0;
    double flo = iapws95::pressure(temperature_k, lo) - pressure_pa;
    double fhi = iapws95::pressure(temperature_k, hi) - pressure_pa;
    if (!(std::isfinite(flo) && std::isfinite(fhi) && flo < 0.0 && fhi > 0.0))
        throw std::runtime_error("IAPWS-95: liquid density bracket unavailable.");
    for (int it = 0; it < 100; ++it) {
        const double mid = (lo + hi) / 2; // std::midpoint of two finite doubles of this range
        const double fm = iapws95::pressure(temperature_k, mid) - pressure_pa;
        if (!std::isfinite(fm)) throw std::runtime_error("IAPWS-95: nonfinite pressure.");
        if (fm < 0.0) {
            lo = mid;
            flo = fm;
        } else {
            hi = mid;
            fhi = fm;
        }
        if (hi - lo <= 2e-10) {
            const bool take_lo = std::fabs(flo) < std::fabs(fhi);
            if (std::fabs(take_lo ? flo : fhi) > 0.02)
                throw std::runtime_error("IAPWS-95: density pressure residual is too large.");
            if (residual_pa) *residual_pa = take_lo ? flo : fhi;
            if (bracket_width) *bracket_width = hi - lo;
            return take_lo ? lo : hi;
        }
    }
    throw std::runtime_error("IAPWS-95: liquid density solve did not converge.");
}
struct WaterState {
    double index = 0, density = 0, temperature_k = 0, pressure_pa = 0, residual_pa = 0, bracket_width = 0;
};
inline WaterState water_optics(double wavelength_nm, double temperature_c = 20.0, double pressure_pa = 101325.0)
{
    // domain and messages of evaluate_water_optics (src/water_refractive_index.cpp:139-162)
    if (!(temperature_c >= 0 && temperature_c <= 60 && pressure_pa >= 5e4 && pressure_pa <= 1e8))
        throw std::invalid_argument("Water material supports liquid branch at 0..60 C and 50 kPa..100 MPa.");
    if (!(wavelength_nm >= 200 && wavelength_nm <= 1100))
        throw std::invalid_argument("IAPWS R9-97: wavelength/state outside supported range.");
    WaterState s;
    s.temperature_k = temperature_c + 273.15;
    s.pressure_pa = pressure_pa;
    s.density = water_density(s.temperature_k, pressure_pa, &s.residual_pa, &s.bracket_width);
    s.index = water_index_r9_97(wavelength_nm, s.temperature_k, s.density);
    return s;
}

// ---------------------------------------------------------------- drop frame
// Incident direction for an inclination alpha (degrees): ki = (cos a, -sin a, 0) in binary32
// and normalised in binary32, and its transverse frame e0 from the helper axis z (x when
// |k_z| >= 0.9), then promoted to binary64 and re-orthonormalised -- the drop path's coordinate
// convention (include/rainbow/vec3.hpp:324-333, apps/generate_phase.cpp:239-244).
struct DropFrame {
    double k[3], e0[3], e1[3];
    float kf[3], e0f[3];
};
inline DropFrame drop_frame(double inclination_deg)
{
    const double a = inclination_deg * kPi / 180.0;
    float kx = (float)std::cos(a), ky = (float)-std::sin(a), kz = 0.0f;
    const float kn = std::sqrt(std::fmaf(kx, kx, std::fmaf(ky, ky, kz * kz)));
    kx /= kn; ky /= kn; kz /= kn;
    const float ax = std::fabs(kz) < 0.9f ? 0.0f : 1.0f, az = std::fabs(kz) < 0.9f ? 1.0f : 0.0f;
    const float kd = std::fmaf(kx, ax, std::fmaf(ky, 0.0f, kz * az));
    float ex = ax - kx * kd, ey = 0.0f - ky * kd, ez = az - kz * kd;
    const float en = std::sqrt(std::fmaf(ex, ex, std::fmaf(ey, ey, ez * ez)));
    ex /= en; ey /= en; ez /= en;
    DropFrame F;
    F.kf[0] = kx; F.kf[1] = ky; F.kf[2] = kz;
    F.e0f[0] = ex; F.e0f[1] = ey; F.e0f[2] = ez;
    double k[3] = {kx, ky, kz};
    const double n = std::sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]);
    for (double& v : k) v /= n;
    double e[3] = {ex, ey, ez};
    const double d = e[0] * k[0] + e[1] * k[1] + e[2] * k[2];
    for (int i = 0; i < 3; ++i) e[i] -= d * k[i];
    const double m = std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
    for (double& v : e) v /= m;
    for (int i = 0; i < 3; ++i) {
        F.k[i] = k[i];
        F.e0[i] = e[i];
    }
    F.e1[0] = k[1] * e[2] - k[2] * e[1];
    F.e1[1] = k[2] * e[0] - k[0] * e[2];
    F.e1[2] = k[0] * e[1] - k[1] * e[0];
    return F;
}

// ---------------------------------------------------------------- analytic diffraction
// Fraunhofer diffraction of the circle-equivalent aperture (radius sqrt(A/pi)) as a separate
// stage: the power within scattering angle theta is Rayleigh's encircled energy
// L(theta) = 1 - J0(x sin theta)^2 - J1(x sin theta)^2, x = 2 pi a_eq / lambda, taken over
// the forward hemisphere and normalised there.  Returns per-row masses (mm^2) that sum to A,
// spread uniformly in azimuth by the caller.
inline std::vector<double> diffraction_rows(const std::vector<double>& u_edges, double area_mm2, double wavelength_nm)
{
    const size_t nt = u_edges.size() - 1;
    const double a_eq = std::sqrt(area_mm2 / kPi); // mm
    const double x = 2 * kPi * a_eq / (wavelength_nm * 1e-6);
    auto L = [&](double u) {
        if (u >= 0.5) u = 0.5;
        const double st = 2 * std::sqrt(u * (1 - u)); // sin(theta) from u = (1 - cos theta)/2
        const double z = x * st;
        const double j0 = ::j0(z), j1 = ::j1(z);
        return 1 - j0 * j0 - j1 * j1;
    };
    const double total = L(0.5);
    std::vector<double> rows(nt, 0.0);
    double prev = 0.0;
    for (size_t i = 0; i < nt; ++i) {
        const double cur = L(u_edges[i + 1]);
        rows[i] = area_mm2 * (cur - prev) / total;
        prev = cur;
    }
    return rows;
}

} // namespace icp::host
