// icp_host_math.hpp -- host-side binary64 geometry shared by the C ABI and the CLIs.
//
// These are the record-setup computations that stay on the CPU in FP64: unit vectors and
// transverse frames (hex_trace/include/ice_crystal/math.hpp:38-69), the saved u edges
// (include/rainbow/phase_cdf_math.hpp:16-32), quaternion rotations
// (hex_phase/src/phase_table.cpp:11-21) and prism face projections
// (hex_trace/include/ice_crystal/hex_prism.hpp:37-43, 64-80).  Operation order follows the
// reference so that the values handed to the device are the reference's bit patterns.
// Build with -ffp-contract=off.
#pragma once
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <vector>

namespace icp::host {

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kSqrt3 = 1.732050807568877293527446341505872367;
constexpr double kEps = DBL_EPSILON;

inline bool finite(double x) { return x >= -DBL_MAX && x <= DBL_MAX; }
inline double maxd(double a, double b) { return a > b ? a : b; }

struct V {
    double x = 0, y = 0, z = 0;
};
inline V add(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V sub(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V mul(V a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V divv(V a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V cross(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline bool vfinite(V a) { return finite(a.x) && finite(a.y) && finite(a.z); }
inline double maxabs(V a) { return maxd(std::fabs(a.x), maxd(std::fabs(a.y), std::fabs(a.z))); }

inline bool normalize(V a, V& out)
{
    const double s = maxabs(a);
    if (!(s > 0) || !finite(s)) return false;
    a = divv(a, s);
    const double n = std::sqrt(dot(a, a));
    if (!(n > 0) || !finite(n)) return false;
    out = divv(a, n);
    return vfinite(out);
}
inline bool is_unit(V a) { return vfinite(a) && std::fabs(dot(a, a) - 1.0) <= 128 * kEps; }

struct Frame {
    V e0, e1;
};
inline bool frame_valid(const Frame& f, V k)
{
    return is_unit(k) && is_unit(f.e0) && is_unit(f.e1) && std::fabs(dot(k, f.e0)) <= 128 * kEps &&
           std::fabs(dot(k, f.e1)) <= 128 * kEps && maxabs(sub(cross(k, f.e0), f.e1)) <= 256 * kEps;
}
// Transverse frame: helper axis = coordinate axis least aligned with k.
inline bool make_frame(V k, Frame& f)
{
    if (!is_unit(k)) return false;
    const double ax = std::fabs(k.x), ay = std::fabs(k.y), az = std::fabs(k.z);
    const V a = (ax <= ay && ax <= az) ? V{1, 0, 0} : (ay <= az ? V{0, 1, 0} : V{0, 0, 1});
    if (!normalize(sub(a, mul(k, dot(k, a))), f.e0)) return false;
    if (!normalize(cross(k, f.e0), f.e1)) return false;
    return frame_valid(f, k);
}

// Saved u edges: symmetric sin^2 construction with exact endpoints.
inline bool u_edges(uint32_t n, std::vector<double>& e)
{
    if (n == 0) return false;
    e.assign(std::size_t(n) + 1, 0.0);
    e.front() = 0;
    e.back() = 1;
    for (uint32_t i = 1; i < n; ++i) {
        const uint32_t k = i < n - i ? i : n - i;
        const double s = std::sin((0.5 * kPi) * double(k) / double(n));
        e[i] = i <= n / 2u ? s * s : 1.0 - s * s;
    }
    for (uint32_t i = 0; i < n; ++i)
        if (!(e[i + 1] > e[i])) return false;
    return true;
}

// Column-major body -> ensemble rotation from an active Hamilton quaternion (w,x,y,z).
inline bool rotation(double w, double x, double y, double z, double r[9])
{
    const double n = w * w + x * x + y * y + z * z;
    if (!finite(n) || std::fabs(n - 1) > 2e-12) return false;
    const double k = 1 / std::sqrt(n);
    w *= k;
    x *= k;
    y *= k;
    z *= k;
    const V cx{1 - 2 * (y * y + z * z), 2 * (x * y + w * z), 2 * (x * z - w * y)};
    const V cy{2 * (x * y - w * z), 1 - 2 * (x * x + z * z), 2 * (y * z + w * x)};
    const V cz{2 * (x * z + w * y), 2 * (y * z - w * x), 1 - 2 * (x * x + y * y)};
    if (!(is_unit(cx) && is_unit(cy) && is_unit(cz) && std::fabs(dot(cx, cy)) <= 128 * kEps &&
          maxabs(sub(cross(cx, cy), cz)) <= 256 * kEps))
        return false;
    r[0] = cx.x; r[1] = cx.y; r[2] = cx.z;
    r[3] = cy.x; r[4] = cy.y; r[5] = cy.z;
    r[6] = cz.x; r[7] = cz.y; r[8] = cz.z;
    return true;
}
inline bool rotation_valid(const double r[9])
{
    const V cx{r[0], r[1], r[2]}, cy{r[3], r[4], r[5]}, cz{r[6], r[7], r[8]};
    return is_unit(cx) && is_unit(cy) && is_unit(cz) && std::fabs(dot(cx, cy)) <= 128 * kEps &&
           maxabs(sub(cross(cx, cy), cz)) <= 256 * kEps;
}
// Rotation::inverse: component-wise dots with the columns.
inline V rotate_inverse(const double r[9], V p)
{
    return {dot(V{r[0], r[1], r[2]}, p), dot(V{r[3], r[4], r[5]}, p), dot(V{r[6], r[7], r[8]}, p)};
}

// Hexagonal prism faces (long axis +y; side face j normal (cos j pi/3, 0, sin j pi/3)).
inline V prism_normal(unsigned f)
{
    switch (f) {
    case 0: return {1, 0, 0};
    case 1: return {0.5, 0, kSqrt3 / 2};
    case 2: return {-0.5, 0, kSqrt3 / 2};
    case 3: return {-1, 0, 0};
    case 4: return {-0.5, 0, -kSqrt3 / 2};
    case 5: return {0.5, 0, -kSqrt3 / 2};
    case 6: return {0, 1, 0};
    case 7: return {0, -1, 0};
    default: return {};
    }
}
inline double prism_face_area(double R, double L, unsigned f) { return f < 6 ? R * L : (3 * kSqrt3 / 2) * R * R; }

struct KahanSum {
    double value = 0, correction = 0;
    void add(double x)
    {
        const double y = x - correction, t = value + y;
        correction = (t - value) - y;
        value = t;
    }
};

// Projected area (Kahan over faces) and the cumulative face weights used to choose the entry
// face (plain adds in face order, hex_prism.hpp:64-80).
struct FaceTable {
    double area = 0;
    double cum[8] = {};
    uint32_t mask = 0;
};
inline FaceTable prism_faces(double R, double L, V k)
{
    FaceTable t;
    KahanSum a;
    double acc = 0;
    for (unsigned f = 0; f < 8; ++f) {
        const double w = prism_face_area(R, L, f) * maxd(0, -dot(prism_normal(f), k));
        a.add(w);
        if (w > 0) {
            t.mask |= 1u << f;
            acc += w;
        }
        t.cum[f] = acc;
    }
    t.area = a.value;
    return t;
}

} // namespace icp::host
