// icp_atlas_host.hpp -- host-side setup of the deterministic single-particle atlas: the
// projected-area quadrature of a hexagonal prism and the incident nodes of the symmetry
// domain.  Binary64, no random numbers; the values handed to the device are the reference's
// bit patterns (operation order follows hex_atlas/src/atlas.cpp:11-51 and :76-97).
// Build with -ffp-contract=off.
//
// Quadrature: every lit face is cut into S x S cells of equal area in a 2-D parameter square
// (side faces: the rectangle itself; end caps: six triangles, each mapped area-preservingly by
// r = sqrt(x) along the sector), and each cell carries a 2 x 3 tensor Gauss-Legendre rule.  A
// point's weight is (face area x |n.k|) / sectors / S^2 x (1/2 for the 2-point rule) x the
// 3-point weight, so the weights of a face add up to its projected area exactly in real
// arithmetic; the sum over faces is checked against the analytic projected area (1e-12).
//
// Incident nodes: the domain t in [0, pi/2] (polar angle from the body +y axis), p in
// [0, pi/6] (azimuth in the x-z plane) with end points included; k(t,p) =
// (sin t cos p, cos t, sin t sin p), e0 = (cos t cos p, -sin t, cos t sin p), e1 = k x e0.
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>

#include "icp_host_math.hpp"

namespace icp::host {

struct AtlasRay {
    uint32_t face;
    uint32_t pad;
    double x, y, z;   // entry point in units of the circumradius (body frame)
    double weight_mm2;
};
static_assert(sizeof(AtlasRay) == 40, "AtlasRay layout");

inline V prism_vertex(unsigned f)
{
    switch (f % 6) {
    case 0: return {kSqrt3 / 2, 0, 0.5};
    case 1: return {0, 0, 1};
    case 2: return {-kSqrt3 / 2, 0, 0.5};
    case 3: return {-kSqrt3 / 2, 0, -0.5};
    case 4: return {0, 0, -1};
    default: return {kSqrt3 / 2, 0, -0.5};
    }
}

// A point strictly inside face `face` and strictly inside every other face plane, within the
// geometry tolerance 128 eps max(1, half length, |p|_max) (hex_prism.hpp:54-57, 108-120).
inline bool strict_face_point(double half_len, V p, unsigned face)
{
    if (face >= 8 || !vfinite(p)) return false;
    const double tol = 128 * kEps * maxd(1, maxd(half_len, maxd(maxabs(p), 0.0)));
    for (unsigned f = 0; f < 8; ++f) {
        const double offset = f < 6 ? kSqrt3 / 2 : half_len;
        const double gap = offset - dot(prism_normal(f), p);
        if (f == face) {
            if (std::fabs(gap) > tol) return false;
        } else if (!(gap > tol)) {
            return false;
        }
    }
    return true;
}

enum AtlasRuleStatus { kRuleOk = 0, kRuleInvalid = 1, kRuleBoundary = 2, kRuleAudit = 3 };

// Quadrature points of the prism (circumradius R, full length L) lit from unit direction k.
inline int atlas_area_rule(double R, double L, V k, uint32_t S, std::vector<AtlasRay>& rays)
{
    rays.clear();
    const double half_len = 0.5 * (L / R);
    if (!(R > 0) || !(L > 0) || !finite(R) || !finite(L) || !(half_len > 0) || !finite(half_len) || !is_unit(k) ||
        S == 0 || uint64_t(S) * S > 1000000)
        return kRuleInvalid;
    // 2-point rule along the first parameter, 3-point rule along the second, on [0, 1]
    const double g2 = 1 / std::sqrt(3.0), g3 = std::sqrt(3.0 / 5.0);
    const double x2[2] = {(1 - g2) / 2, (1 + g2) / 2};
    const double y3[3] = {(1 - g3) / 2, 0.5, (1 + g3) / 2};
    const double w3[3] = {5.0 / 18, 4.0 / 9, 5.0 / 18};
    KahanSum total;
    for (unsigned f = 0; f < 8; ++f) {
        const V n = prism_normal(f);
        const double lit = prism_face_area(R, L, f) * maxd(0, -dot(n, k));
        if (lit == 0) continue;
        const unsigned sectors = f < 6 ? 1 : 6;
        for (unsigned sector = 0; sector < sectors; ++sector)
            for (uint32_t a = 0; a < S; ++a)
                for (uint32_t b = 0; b < S; ++b)
                    for (unsigned i = 0; i < 2; ++i)
                        for (unsigned j = 0; j < 3; ++j) {
                            const double x = (a + x2[i]) / S, y = (b + y3[j]) / S;
                            V p;
                            if (f < 6) {
                                const V t{-n.z, 0, n.x};
                                p = add(add(mul(n, kSqrt3 / 2), mul(t, x - 0.5)), V{0, (2 * y - 1) * half_len, 0});
                            } else {
                                p = mul(add(mul(prism_vertex(sector), 1 - y), mul(prism_vertex(sector + 1), y)),
                                        std::sqrt(x));
                                p.y = (f == 6 ? 1 : -1) * half_len;
                            }
                            AtlasRay r{f, 0u, p.x, p.y, p.z, (lit / sectors / double(S) / S) * 0.5 * w3[j]};
                            if (!(r.weight_mm2 > 0) || !finite(r.weight_mm2)) return kRuleAudit;
                            if (!strict_face_point(half_len, p, f)) return kRuleBoundary;
                            rays.push_back(r);
                            total.add(r.weight_mm2);
                        }
    }
    if (rays.empty() || std::fabs(total.value / prism_faces(R, L, k).area - 1) > 1e-12) return kRuleAudit;
    return kRuleOk;
}

struct AtlasIncident {
    double theta, phi;
    V k_rule;  // direction the quadrature is built for (normalised once)
    V k;       // direction of the trace (normalised again, as the trace settings do)
    Frame frame;
};

// Incident node (i, j) of T x P intervals; the end points use exact sines and cosines.
inline bool atlas_incident(uint32_t T, uint32_t P, uint32_t i, uint32_t j, AtlasIncident& out)
{
    if (T == 0 || P == 0 || T > 4096 || P > 4096 || i > T || j > P) return false;
    out.theta = (kPi / 2) * i / T;
    out.phi = (kPi / 6) * j / P;
    const double st = i == 0 ? 0 : (i == T ? 1 : std::sin(out.theta));
    const double ct = i == 0 ? 1 : (i == T ? 0 : std::cos(out.theta));
    const double sp = j == 0 ? 0 : (j == P ? 0.5 : std::sin(out.phi));
    const double cp = j == 0 ? 1 : (j == P ? kSqrt3 / 2 : std::cos(out.phi));
    if (!normalize(V{st * cp, ct, st * sp}, out.k_rule)) return false;
    if (!normalize(out.k_rule, out.k)) return false;
    V e;
    if (!normalize(V{ct * cp, -st, ct * sp}, e)) return false;
    out.frame.e0 = e;
    out.frame.e1 = cross(out.k, e);
    return frame_valid(out.frame, out.k);
}

} // namespace icp::host
