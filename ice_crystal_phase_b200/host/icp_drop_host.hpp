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
// Liquid density (kg m^-3) of air-free water.  At 1 atm: Tanaka et al. (2001, Metrologia 38,
// 301) below 35 C, Kell (1975, J. Chem. Eng. Data 20, 97) above 45 C, blended linearly in
// between; pressure through the secant bulk modulus of pure water of the UNESCO 1981
// equation of state, rho(p) = rho(1 atm) / (1 - p/K(t, p)), p gauge in bar.  The reference
// inverts the IAPWS-95 pressure equation of state instead; against it this stays within
// 0.036 kg m^-3 over 0..60 C and 50 kPa..100 MPa, i.e. n within 2.5e-6 up to 10 MPa and
// 1.2e-5 up to 100 MPa.
inline double water_density(double temperature_c, double pressure_pa)
{
    const double t = temperature_c;
    const double tanaka = 999.974950 * (1 - (t - 3.983035) * (t - 3.983035) * (t + 301.797) / (522528.9 * (t + 69.34881)));
    const double kell = (999.83952 + 16.945176 * t - 7.9870401e-3 * t * t - 46.170461e-6 * t * t * t +
                         105.56302e-9 * t * t * t * t - 280.54253e-12 * t * t * t * t * t) /
                        (1 + 16.879850e-3 * t);
    const double w = std::min(1.0, std::max(0.0, (t - 35.0) / 10.0));
    const double rho0 = (1 - w) * tanaka + w * kell;
    const double pb = (pressure_pa - 101325.0) * 1e-5;
    const double k0 = 19652.21 + 148.4206 * t - 2.327105 * t * t + 1.360477e-2 * t * t * t - 5.155288e-5 * t * t * t * t;
    const double ka = 3.239908 + 1.43713e-3 * t + 1.16092e-4 * t * t - 5.77905e-7 * t * t * t;
    const double kb = 8.50935e-5 - 6.12293e-6 * t + 5.2787e-8 * t * t;
    return rho0 / (1 - pb / (k0 + ka * pb + kb * pb * pb));
}
struct WaterState {
    double index = 0, density = 0, temperature_k = 0, pressure_pa = 0;
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
    s.density = water_density(temperature_c, pressure_pa);
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
