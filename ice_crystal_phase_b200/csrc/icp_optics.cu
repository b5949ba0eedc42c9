// icp_optics.cu -- per-direction optics of the drop's wave stages on the device (sm_100a) and
// its C ABI (include/icp_b200.h, "patch optics").  Built with -fmad=false: every binary32 and
// binary64 product and sum rounds on its own and only the reference's explicit fmaf / fma
// calls are fused, so the arithmetic is the reference's host build's operation for operation.
//
// patch_optics_kernel: one thread per query direction (grid-stride over the SMs).  The thread
// walks the direction's sorted hit list (contiguous: consecutive directions read consecutive
// hit ranges) and, per hit, gathers the four corner vertices of the hit patch (68-byte records;
// the whole lattice -- 4 x 513^2 vertices, 72 MB -- stays resident in the 126 MB L2 across the
// launch), carries each corner's Jones vector(s) to the query direction's scattering frame by
// the minimum rotation, interpolates the optical path in cycles and the fields bilinearly at
// the hit's (u, v), and adds the coherent path field, the incoherent intensities and -- for
// the focal stage -- the quarter-turn-corrected field and the per-family counters into
// compensated sums, in hit order.  The reference's PatchOpticalEvaluator
// (include/rainbow/patch_optical_evaluator.hpp) defines every value and flag; folded-branch
// records are not taken (hits on NeedsRefinement patches are refinement-pending).
// Device libm (sqrt / sqrtf are correctly rounded; cosf, sinf, atan2 are CUDA's) is the only
// source of difference from the reference's host results.
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

// result flags (PatchOpticalFlags), query flags (PatchQueryFlags), focal flags (FocalOpticalFlags)
enum : uint32_t { kQuery = 1, kInput = 2, kFrame = 4, kPhase = 8, kArith = 16, kRefine = 32, kBoundary = 64,
                  kSingular = 128 };
constexpr uint32_t kErrors = kQuery | kInput | kFrame | kPhase | kArith;
constexpr uint32_t kPending = kRefine | kBoundary | kSingular;
constexpr uint32_t kQueryErrors = 1u | 2u | 4u | 256u;
enum : uint32_t { kQueryRefineHit = 8, kQueryBoundaryHit = 16, kQuerySingularHit = 128 };
enum : uint32_t { kFocalInputError = 1, kFocalInputPending = 2, kFocalDerivative = 4, kFocalGeometry = 8,
                  kFocalArith = 16 };
constexpr float kFrameTol = 0x1p-10f;
constexpr float kDegenerate = 0x1p-30f;

struct F3 {
    float x, y, z;
};
struct D3 {
    double x, y, z;
};
struct Frame {
    F3 e0, e1;
};

__device__ __forceinline__ F3 f3(const icp_vec3f& v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ float dot(F3 a, F3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
__device__ __forceinline__ double dot(D3 a, D3 b) { return fma(a.x, b.x, fma(a.y, b.y, a.z * b.z)); }
__device__ __forceinline__ F3 cross(F3 a, F3 b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ D3 cross(D3 a, D3 b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ F3 scale(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ D3 scale(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ F3 divide(F3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ D3 divide(D3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ F3 minus(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 plus(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 minus(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 wide(F3 a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ F3 unit(F3 a) { return divide(a, sqrtf(dot(a, a))); }
__device__ __forceinline__ D3 unit(D3 a) { return divide(a, sqrt(dot(a, a))); }
__device__ __forceinline__ bool finite64(double x) { return x >= -DBL_MAX && x <= DBL_MAX; }
__device__ __forceinline__ bool finite32(float x) { return x >= -FLT_MAX && x <= FLT_MAX; }
__device__ __forceinline__ bool finite(F3 a) { return finite32(a.x) && finite32(a.y) && finite32(a.z); }
__device__ __forceinline__ bool finite(const icp_field32& f)
{
    return finite32(f.x.real) && finite32(f.x.imag) && finite32(f.y.real) && finite32(f.y.imag);
}
__device__ __forceinline__ bool finite(const icp_field64& f)
{
    return finite64(f.s_real) && finite64(f.s_imag) && finite64(f.p_real) && finite64(f.p_imag);
}
__device__ __forceinline__ double nan64() { return __longlong_as_double(0x7ff8000000000000ll); }

// ------------------------------------------------------------ frames and transport
__device__ __forceinline__ bool is_unit(F3 a) { return finite(a) && fabsf(dot(a, a) - 1.0f) <= kFrameTol; }
__device__ __forceinline__ bool is_frame(F3 d, const Frame& f)
{
    if (!is_unit(f.e0) || !is_unit(f.e1)) return false;
    if (fabsf(dot(d, f.e0)) > kFrameTol || fabsf(dot(d, f.e1)) > kFrameTol || fabsf(dot(f.e0, f.e1)) > kFrameTol)
        return false;
    return dot(cross(f.e0, f.e1), d) >= 1.0f - 4.0f * kFrameTol;
}
// e0 normal to the scattering plane (the incident basis carried over at exact forward or
// backward scattering), e1 = out x e0.
__device__ bool scattering_frame(F3 inc, F3 basis, F3 out, Frame& frame)
{
    if (!is_unit(inc) || !is_unit(out) || !is_unit(basis) || fabsf(dot(inc, basis)) > kFrameTol) return false;
    F3 e0 = cross(inc, out);
    float n2 = dot(e0, e0);
    if (n2 > kDegenerate)
        e0 = divide(e0, sqrtf(n2));
    else {
        e0 = minus(basis, scale(out, dot(out, basis)));
        n2 = dot(e0, e0);
        if (!(n2 > kDegenerate)) return false;
        e0 = divide(e0, sqrtf(n2));
    }
    F3 e1 = cross(out, e0);
    const float m2 = dot(e1, e1);
    if (!(m2 > kDegenerate)) return false;
    e1 = divide(e1, sqrtf(m2));
    const Frame f{e0, e1};
    if (!is_frame(out, f)) return false;
    frame = f;
    return true;
}
// Rodrigues' formula for the minimum rotation taking a to b: v = a x b, c = a . b.
__device__ __forceinline__ D3 rotate(D3 x, D3 v, double c)
{
    const D3 vx = cross(v, x);
    return plus(plus(x, vx), divide(cross(v, vx), 1.0 + c));
}
__device__ __forceinline__ bool fits_float(double x) { return x >= -0x1.fffffep127 && x <= 0x1.fffffep127; }

// Carries `columns` Jones vectors from the source ray's frame to the target frame.
__device__ bool transport(F3 sdir, const Frame& sf, const icp_field32* src, unsigned columns, F3 tdir,
                          const Frame& tf, icp_field32* out)
{
    if (columns == 2 && (!finite(src[0]) || !finite(src[1]))) return false;
    if (!is_unit(sdir) || !is_unit(tdir) || !is_frame(sdir, sf) || !is_frame(tdir, tf)) return false;
    const D3 sw = unit(wide(sdir)), tw = unit(wide(tdir));
    const double c = dot(sw, tw);
    if (!(1.0 + c > 0x1p-30)) return false; // no unique rotation between antipodes
    const D3 v = cross(sw, tw);
    const D3 se0 = wide(sf.e0), se1 = wide(sf.e1), te0 = wide(tf.e0), te1 = wide(tf.e1);
    icp_field32 tmp[2];
    for (unsigned j = 0; j < columns; ++j) {
        const icp_field32& f = src[j];
        const D3 re = plus(scale(se0, double(f.x.real)), scale(se1, double(f.y.real)));
        const D3 im = plus(scale(se0, double(f.x.imag)), scale(se1, double(f.y.imag)));
        const D3 rt = rotate(re, v, c), it = rotate(im, v, c);
        const double xr = dot(rt, te0), xi = dot(it, te0), yr = dot(rt, te1), yi = dot(it, te1);
        if (!fits_float(xr) || !fits_float(xi) || !fits_float(yr) || !fits_float(yi)) return false;
        tmp[j] = {{float(xr), float(xi)}, {float(yr), float(yi)}};
    }
    for (unsigned j = 0; j < columns; ++j) out[j] = tmp[j];
    return true;
}

// ------------------------------------------------------------ optical path in cycles
__device__ __forceinline__ bool cycles_ok(const icp_phase_cycles& q) { return q.fraction >= 0.0f && q.fraction < 1.0f; }
__device__ __forceinline__ double cycles_diff(const icp_phase_cycles& a, const icp_phase_cycles& b)
{
    const long long whole = (long long)a.turns - (long long)b.turns;
    return double(whole) + (double(a.fraction) - double(b.fraction));
}
__device__ bool cycles_add(const icp_phase_cycles& anchor, double delta, icp_phase_cycles& out)
{
    if (!(delta > -0x1p33 && delta < 0x1p33)) return false;
    const double whole = floor(delta);
    double frac = double(anchor.fraction) + (delta - whole);
    long long turns = (long long)anchor.turns + (long long)whole;
    if (frac < 0.0) {
        --turns;
        frac += 1.0;
    }
    if (frac >= 1.0) {
        ++turns;
        frac -= 1.0;
    }
    constexpr long long lo = -2147483647LL - 1, hi = 2147483647LL;
    if (turns < lo || turns > hi) return false;
    float stored = float(frac);
    if (stored >= 1.0f) {
        ++turns;
        stored = 0.0f;
        if (turns > hi) return false;
    } else if (stored < 0.0f) {
        --turns;
        stored += 1.0f;
        if (turns < lo) return false;
    }
    out.turns = int(turns);
    out.fraction = stored == 0.0f ? 0.0f : stored;
    return cycles_ok(out);
}
// Bilinear optical path anchored at q00; the corners are returned exactly.
__device__ bool cycles_bilinear(const icp_phase_cycles* q, float u, float v, icp_phase_cycles& out)
{
    if (!cycles_ok(q[0]) || !cycles_ok(q[1]) || !cycles_ok(q[2]) || !cycles_ok(q[3]) || !(u >= 0.0f && u <= 1.0f) ||
        !(v >= 0.0f && v <= 1.0f))
        return false;
    if (u == 0.0f && v == 0.0f) { out = q[0]; return true; }
    if (u == 1.0f && v == 0.0f) { out = q[1]; return true; }
    if (u == 0.0f && v == 1.0f) { out = q[2]; return true; }
    if (u == 1.0f && v == 1.0f) { out = q[3]; return true; }
    const double du0 = cycles_diff(q[1], q[0]), du1 = cycles_diff(q[3], q[2]), dv0 = cycles_diff(q[2], q[0]);
    const double ud = u, vd = v;
    const double row = fma(ud, du1 - du0, dv0);
    return cycles_add(q[0], fma(vd, row, ud * du0), out);
}
// exp(+i 2 pi fraction) in binary32, exact at quarter turns.
__device__ bool unit_phasor(const icp_phase_cycles& q, float& re, float& im)
{
    if (!cycles_ok(q)) return false;
    const float f = q.fraction;
    if (f == 0.0f) { re = 1.0f; im = 0.0f; return true; }
    if (f == 0.25f) { re = 0.0f; im = 1.0f; return true; }
    if (f == 0.5f) { re = -1.0f; im = 0.0f; return true; }
    if (f == 0.75f) { re = 0.0f; im = -1.0f; return true; }
    const float angle = 0x1.921fb6p+2f * (f > 0.5f ? f - 1.0f : f);
    re = cosf(angle);
    im = sinf(angle);
    return true;
}

// ------------------------------------------------------------ focal quarter turns
__device__ __forceinline__ bool focal_layout_ok(const icp_focal_config& c)
{
    if (c.grid_width < 2 || c.grid_height < 2 || !(c.grid_half_extent > 0) || !(c.grid_half_extent <= FLT_MAX))
        return false;
    if ((unsigned long long)c.grid_width * c.grid_height > 0xffffffffull / 4u ||
        (unsigned long long)(c.grid_width - 1u) * (c.grid_height - 1u) > 0xffffffffull / 4u)
        return false;
    for (unsigned j = 0; j < 4; ++j)
        if (c.quarter_turn_offsets[j] > 3) return false;
    return true;
}
// Sign of the radial derivative of the scattering angle over the emitting plane at (u, v) of the
// patch's incident cell -- the centre (central differences), or a folded branch's representative
// point (differences along the cell edges interpolated to u, v): one extra quarter turn where it
// is positive (a focal line was crossed).  FocalPhase::estimate / estimate_at
// (include/rainbow/focal_phase.hpp:27-101).
__device__ uint32_t focal_estimate(const icp_outgoing_vertex* __restrict__ vertices, uint32_t vertex_count,
                                   const icp_outgoing_patch& patch, F3 incident, const icp_focal_config& c,
                                   uint32_t& family_out, uint32_t& extra_out, uint32_t& turns_out, double u = 0.5,
                                   double v = 0.5, bool at_center = true)
{
    if (!(u >= 0 && u <= 1 && v >= 0 && v <= 1) || !vertices || !focal_layout_ok(c) || !finite(incident))
        return kFocalGeometry;
    const uint32_t n = c.grid_width * c.grid_height, nx = c.grid_width - 1u, cells = nx * (c.grid_height - 1u);
    if (patch.patch_id >= 4u * cells || vertex_count < 4u * n) return kFocalGeometry;
    const uint32_t family = patch.patch_id / cells, cell = patch.patch_id % cells;
    const uint32_t ix = cell % nx, iy = cell / nx;
    const uint32_t first = family * n + iy * c.grid_width + ix;
    const uint32_t expected[4] = {first, first + 1u, first + c.grid_width, first + c.grid_width + 1u};
    const D3 wi = wide(incident);
    if (!(dot(wi, wi) > 0)) return kFocalGeometry;
    double theta[4];
    for (unsigned j = 0; j < 4; ++j) {
        if (patch.vertex_indices[j] != expected[j]) return kFocalGeometry;
        const icp_outgoing_vertex& a = vertices[expected[j]];
        const F3 dir = f3(a.direction_drop);
        if (a.status != 1u || !finite(dir)) return kFocalGeometry;
        const D3 wo = wide(dir);
        if (!(dot(wo, wo) > 0)) return kFocalGeometry;
        const D3 x = cross(wi, wo);
        theta[j] = atan2(sqrt(dot(x, x)), dot(wi, wo));
        if (!finite64(theta[j])) return kFocalGeometry;
    }
    const double e = double(c.grid_half_extent);
    const double du = 2 * e / double(c.grid_width - 1u), dv = 2 * e / double(c.grid_height - 1u);
    const double U = (2 * (double(ix) + u) / double(c.grid_width - 1u) - 1) * e;
    const double V = (2 * (double(iy) + v) / double(c.grid_height - 1u) - 1) * e;
    const double r2 = fma(U, U, V * V);
    if (!(r2 > 0)) return kFocalDerivative;
    const double gu = at_center ? ((theta[1] - theta[0]) + (theta[3] - theta[2])) / (2 * du)
                                : ((1 - v) * (theta[1] - theta[0]) + v * (theta[3] - theta[2])) / du;
    const double gv = at_center ? ((theta[2] - theta[0]) + (theta[3] - theta[1])) / (2 * dv)
                                : ((1 - u) * (theta[2] - theta[0]) + u * (theta[3] - theta[1])) / dv;
    const double num = fma(U, gu, V * gv);
    const double guard = 0x1p-46 * (fabs(U * gu) + fabs(V * gv) + 1); // cancellation guard
    if (!finite64(num) || !finite64(r2)) return kFocalGeometry;
    if (fabs(num) <= guard) return kFocalDerivative;
    if (!finite64(num / (2 * r2))) return kFocalGeometry;
    family_out = family;
    extra_out = num > 0 ? 1u : 0u;
    turns_out = (c.quarter_turn_offsets[family] + extra_out) & 3u;
    return 0;
}
__device__ __forceinline__ icp_field64 quarter_turns(const icp_field64& a, uint32_t q)
{
    switch (q & 3u) {
    case 1: return {-a.s_imag, a.s_real, -a.p_imag, a.p_real};
    case 2: return {-a.s_real, -a.s_imag, -a.p_real, -a.p_imag};
    case 3: return {a.s_imag, -a.s_real, a.p_imag, -a.p_real};
    default: return a;
    }
}

// ------------------------------------------------------------ folded patches
// A patch that needs refinement (its bilinear direction map folds: the Jacobian J(u, v) of the
// map from the cell's parameters to the sphere of directions changes sign inside the cell) is
// described by its connected sign components ("branches") instead of one solid angle
// (include/rainbow/folded_patch_geometry.hpp, folded_patch_builder.hpp): per branch its share of
// the cell's parameter area, its unsigned solid angle (adaptive Gauss-Legendre quadrature of
// |J| / |x|^3 over the component, 8 x 8 against 16 x 16 points per panel), a representative
// parameter point and, for the focal stage, the quarter turns at that point.  A hit on such a
// patch is evaluated with the branch containing its (u, v).  All binary64, fma where the
// reference fuses, so each record is the reference's host build's bit for bit.
enum : uint32_t { kFoldReady = 0, kFoldInvalidInput = 1, kFoldHemisphere = 2, kFoldNoSignChange = 4,
                  kFoldTopology = 8, kFoldUnconverged = 16, kFoldInvalidMetric = 32 };

// Gauss-Legendre nodes and weights of orders 8 and 16 on [-1, 1], non-negative half (the rule
// is symmetric), correctly rounded to binary64.
__constant__ double kGl8x[4] = {0.18343464249564978, 0.525532409916329, 0.7966664774136267, 0.9602898564975362};
__constant__ double kGl8w[4] = {0.36268378337836166, 0.3137066458778869, 0.22238103445337443, 0.10122853629037706};
__constant__ double kGl16x[8] = {0.09501250983763744, 0.2816035507792589, 0.45801677765722737, 0.6178762444026438,
                                 0.755404408355003,   0.8656312023878318, 0.9445750230732326,  0.9894009349916499};
__constant__ double kGl16w[8] = {0.18945061045506864, 0.18260341504492364, 0.16915651939500265, 0.1495959888165767,
                                 0.12462897125553407, 0.0951585116824926,  0.062253523938647456, 0.027152459411754176};
// node i (ascending) of the n-point rule
__device__ __forceinline__ void gl_point(bool high, unsigned i, double& x, double& w)
{
    const unsigned h = high ? 8u : 4u;
    const double* X = high ? kGl16x : kGl8x;
    const double* W = high ? kGl16w : kGl8w;
    const unsigned k = i < h ? h - 1u - i : i - h;
    x = i < h ? -X[k] : X[k];
    w = W[k];
}

__device__ __forceinline__ double fmix(double a, double b, double t) { return fma(t, b - a, a); }
__device__ __forceinline__ double bilinear4(const double* a, double u, double v)
{
    return fmix(fmix(a[0], a[1], u), fmix(a[2], a[3], u), v);
}
struct Fold {
    D3 c[4];        // the four corner directions, binary64
    double j[4];    // corner Jacobians (order 00, 10, 01, 11), divided by `scale`
    double scale;   // max |J| at the corners
};
__device__ __forceinline__ D3 fold_point(const Fold& g, double u, double v)
{
    return plus(scale(plus(scale(g.c[0], 1 - u), scale(g.c[1], u)), 1 - v),
                scale(plus(scale(g.c[2], 1 - u), scale(g.c[3], u)), v));
}
// det[a, b, c] with the cofactors' products rounded once (fma pairs)
__device__ __forceinline__ double det3(D3 a, D3 b, D3 c)
{
    const double yz = b.z * c.y, zx = b.x * c.z, xy = b.y * c.x;
    const double x = fma(b.y, c.z, -yz) + fma(-b.z, c.y, yz);
    const double y = fma(b.z, c.x, -zx) + fma(-b.x, c.z, zx);
    const double z = fma(b.x, c.y, -xy) + fma(-b.y, c.x, xy);
    return fma(a.x, x, fma(a.y, y, a.z * z));
}
__device__ uint32_t fold_init(Fold& g, const F3* input)
{
    for (unsigned i = 0; i < 4; ++i) {
        if (!finite(input[i])) return kFoldInvalidInput;
        g.c[i] = wide(input[i]);
        const double q = dot(g.c[i], g.c[i]);
        if (!(q > 0 && q <= 4)) return kFoldInvalidInput;
    }
    const D3 axis = plus(plus(g.c[0], g.c[1]), plus(g.c[2], g.c[3]));
    // a conservative roundoff guard for the corner sum and dot; failing it proves nothing
    for (unsigned i = 0; i < 4; ++i) {
        double bound = 0;
        for (unsigned k = 0; k < 4; ++k)
            bound += fabs(g.c[k].x * g.c[i].x) + fabs(g.c[k].y * g.c[i].y) + fabs(g.c[k].z * g.c[i].z);
        if (!(dot(axis, g.c[i]) > 0x1p-46 * bound)) return kFoldHemisphere;
    }
    const D3 eu = minus(g.c[1], g.c[0]), ev = minus(g.c[2], g.c[0]);
    g.j[0] = det3(g.c[0], eu, ev);
    g.j[1] = det3(g.c[1], eu, minus(g.c[3], g.c[1]));
    g.j[2] = det3(g.c[2], minus(g.c[3], g.c[2]), ev);
    g.j[3] = det3(g.c[3], minus(g.c[3], g.c[2]), minus(g.c[3], g.c[1]));
    g.scale = 0;
    bool pos = false, neg = false;
    for (unsigned i = 0; i < 4; ++i) {
        if (!finite64(g.j[i])) return kFoldInvalidInput;
        g.scale = fmax(g.scale, fabs(g.j[i]));
        pos |= g.j[i] > 0;
        neg |= g.j[i] < 0;
    }
    if (!(pos && neg && g.scale > 0)) return kFoldNoSignChange;
    for (unsigned i = 0; i < 4; ++i) g.j[i] /= g.scale;
    return kFoldReady;
}
// The v interval of the vertical section at u where sign J > 0 (J is linear in v there).
__device__ __forceinline__ bool fold_section(const double* a, int sign, double u, double& lo, double& hi)
{
    const double b = double(sign) * fmix(a[0], a[1], u);
    const double t = double(sign) * fmix(a[2], a[3], u);
    if (b <= 0 && t <= 0) return false;
    lo = 0;
    hi = 1;
    if (b > 0 && t > 0) return true;
    const double r = fabs(b) / (fabs(b) + fabs(t)); // in [0, 1] without cancellation
    if (b > 0) hi = r;
    else lo = r;
    return hi > lo;
}
// u values where an edge v = 0 or v = 1 changes sign, with 0 and 1, sorted and distinct.
__device__ unsigned fold_cuts(const Fold& g, double* x)
{
    unsigned n = 2;
    x[0] = 0;
    x[1] = 1;
    for (unsigned edge = 0; edge < 2; ++edge) {
        const double a = g.j[2 * edge], b = g.j[2 * edge + 1];
        if ((a < 0 && b > 0) || (a > 0 && b < 0)) x[n++] = fabs(a) / (fabs(a) + fabs(b));
    }
    for (unsigned i = 1; i < n; ++i) {
        const double t = x[i];
        unsigned k = i;
        while (k && x[k - 1] > t) {
            x[k] = x[k - 1];
            --k;
        }
        x[k] = t;
    }
    unsigned m = 1;
    for (unsigned i = 1; i < n; ++i)
        if (x[i] != x[m - 1]) x[m++] = x[i];
    return m;
}
// Connected components of J < 0 and J > 0 as runs of u slabs whose sections stay joined.
__device__ bool fold_components(const Fold& g, icp_folded_record& r)
{
    double x[4] = {0, 0, 0, 0};
    const unsigned n = fold_cuts(g, x);
    r.branch_count = 0;
    for (int sign = -1; sign <= 1; sign += 2) {
        int active = -1;
        for (unsigned i = 0; i + 1 < n; ++i) {
            const double mid = (x[i] + x[i + 1]) * 0.5;
            double lo = 0, hi = 0;
            if (!(mid > x[i] && mid < x[i + 1])) return false;
            if (!fold_section(g.j, sign, mid, lo, hi)) {
                active = -1;
                continue;
            }
            double bl = 0, bh = 0;
            const bool joined = active >= 0 && fold_section(g.j, sign, x[i], bl, bh);
            if (!joined) {
                if (r.branch_count >= 4) return false;
                active = int(r.branch_count++);
                r.branches[active].sign = sign;
                r.branches[active].u0 = x[i];
            }
            r.branches[active].u1 = x[i + 1];
        }
    }
    return r.branch_count >= 2;
}
// Branch of a folded record containing (u, v), or -1 where the sign of J is not certain.
__device__ int fold_branch_at(const icp_folded_record& r, double u, double v)
{
    if (r.flags != kFoldReady || !(u >= 0 && u <= 1 && v >= 0 && v <= 1)) return -1;
    const double b = fmix(r.jacobian[0], r.jacobian[1], u);
    const double t = fmix(r.jacobian[2], r.jacobian[3], u);
    const double jac = fmix(b, t, v);
    const double bound = (1 - u) * (1 - v) * fabs(r.jacobian[0]) + u * (1 - v) * fabs(r.jacobian[1]) +
                         (1 - u) * v * fabs(r.jacobian[2]) + u * v * fabs(r.jacobian[3]);
    if (fabs(jac) <= 0x1p-46 * bound) return -1; // a sign-uncertainty guard only
    const int sign = jac > 0 ? 1 : -1;
    for (unsigned i = 0; i < r.branch_count; ++i)
        if (r.branches[i].sign == sign && u >= r.branches[i].u0 && u <= r.branches[i].u1) return int(i);
    return -1;
}
struct Integral {
    double area, mu, mv, omega;
};
struct Panel {
    double u0, u1, z0, z1;
    unsigned depth;
};
// Tensor Gauss rule over a panel of the branch: u across [u0, u1], v = the section's
// [lo, hi] mapped from z in [z0, z1].
__device__ Integral fold_quadrature(const Fold& g, int sign, const Panel& p, bool high)
{
    const unsigned n = high ? 16u : 8u;
    const double uh = (p.u1 - p.u0) * 0.5, uc = (p.u0 + p.u1) * 0.5;
    const double zh = (p.z1 - p.z0) * 0.5, zc = (p.z0 + p.z1) * 0.5;
    Integral s{0, 0, 0, 0};
    for (unsigned i = 0; i < n; ++i) {
        double xi, wi;
        gl_point(high, i, xi, wi);
        const double u = fma(uh, xi, uc);
        double vl = 0, vh = 0;
        if (!fold_section(g.j, sign, u, vl, vh)) continue;
        const double width = vh - vl;
        for (unsigned k = 0; k < n; ++k) {
            double xk, wk;
            gl_point(high, k, xk, wk);
            const double z = fma(zh, xk, zc), v = fma(z, width, vl);
            const double w = uh * zh * wi * wk * width;
            const D3 pt = fold_point(g, u, v);
            const double q = dot(pt, pt);
            const double J = fabs(bilinear4(g.j, u, v)) * g.scale;
            s.area += w;
            s.mu += w * u;
            s.mv += w * v;
            s.omega += w * J / (q * sqrt(q));
        }
    }
    return s;
}
__device__ bool fold_integrate(const Fold& g, icp_folded_branch& b, const icp_folded_config& c, icp_folded_record& r)
{
    double cuts[4] = {0, 0, 0, 0};
    const unsigned n = fold_cuts(g, cuts);
    Integral sum{0, 0, 0, 0};
    // starting panels split where the sections' topology changes, so the root curve is smooth
    // inside each
    for (unsigned k = 0; k + 1 < n; ++k) {
        const double lo = fmax(cuts[k], b.u0), hi = fmin(cuts[k + 1], b.u1);
        if (!(hi > lo)) continue;
        Panel stack[26];
        unsigned size = 1;
        stack[0] = {lo, hi, 0, 1, 0};
        while (size) {
            const Panel p = stack[--size];
            if (++r.panels > c.maximum_panels) return false;
            const Integral low = fold_quadrature(g, b.sign, p, false), high = fold_quadrature(g, b.sign, p, true);
            if (!(high.area > 0 && high.omega > 0 && finite64(high.area) && finite64(high.omega))) return false;
            const double ea = fabs(high.area - low.area) / high.area;
            const double es = fabs(high.omega - low.omega) / high.omega;
            const double emu = fabs(high.mu - low.mu) / high.area;
            const double emv = fabs(high.mv - low.mv) / high.area;
            const double error = fmax(fmax(ea, es), fmax(emu, emv));
            if (error <= c.relative_tolerance) {
                r.largest_estimated_relative_error = fmax(r.largest_estimated_relative_error, error);
                sum.area += high.area;
                sum.mu += high.mu;
                sum.mv += high.mv;
                sum.omega += high.omega;
                continue;
            }
            if (p.depth >= c.maximum_depth || size + 2 > 26u) return false;
            if ((p.depth & 1u) == 0) { // alternate: halve u, then z
                const double m = (p.u0 + p.u1) * 0.5;
                if (!(m > p.u0 && m < p.u1)) return false;
                stack[size++] = {m, p.u1, p.z0, p.z1, p.depth + 1};
                stack[size++] = {p.u0, m, p.z0, p.z1, p.depth + 1};
            } else {
                const double m = (p.z0 + p.z1) * 0.5;
                if (!(m > p.z0 && m < p.z1)) return false;
                stack[size++] = {p.u0, p.u1, m, p.z1, p.depth + 1};
                stack[size++] = {p.u0, p.u1, p.z0, m, p.depth + 1};
            }
        }
    }
    if (!(sum.area > 0 && sum.omega > 0 && finite64(sum.omega))) return false;
    b.area_fraction = sum.area;
    b.solid_angle_sr = sum.omega;
    b.representative_u = sum.mu / sum.area;
    b.representative_v = sum.mv / sum.area;
    // the centroid of a non-convex component can lie outside it: then the section's midpoint
    double vl = 0, vh = 0;
    if (!(b.representative_u > b.u0 && b.representative_u < b.u1) ||
        !fold_section(g.j, b.sign, b.representative_u, vl, vh))
        return false;
    if (!(b.representative_v > vl && b.representative_v < vh)) b.representative_v = (vl + vh) * 0.5;
    return b.representative_v > vl && b.representative_v < vh;
}
__device__ __forceinline__ bool fold_config_ok(const icp_folded_config& c)
{
    return c.relative_tolerance >= 1e-12 && c.relative_tolerance <= 1e-3 && c.maximum_panels >= 1 &&
           c.maximum_panels <= 65536 && c.maximum_depth >= 1 && c.maximum_depth <= 24;
}
__device__ __forceinline__ void fold_blank(icp_folded_record& r, uint32_t patch_id, uint32_t compact)
{
    memset(&r, 0, sizeof r);
    r.compact_index = compact;
    r.patch_id = patch_id;
    r.flags = kFoldInvalidInput;
    for (unsigned i = 0; i < 4; ++i) r.branches[i].focal_flags = kFocalInputPending;
}
// FoldedPatchBuilder::prepare: the record of one NeedsRefinement patch (status 3).
__device__ void fold_prepare(const icp_outgoing_vertex* __restrict__ vertices, uint32_t vertex_count,
                             const icp_outgoing_patch& patch, uint32_t compact, F3 incident,
                             const icp_focal_config* focal, const icp_folded_config& config, icp_folded_record& r)
{
    fold_blank(r, patch.patch_id, compact);
    if (!vertices || patch.status != 3u || !(patch.incident_area_drop2 > 0) ||
        !finite64(double(patch.incident_area_drop2)))
        return;
    F3 corners[4];
    for (unsigned i = 0; i < 4; ++i) {
        const uint32_t id = patch.vertex_indices[i];
        if (id >= vertex_count) return;
        const icp_outgoing_vertex& a = vertices[id];
        const F3 d = f3(a.direction_drop);
        // PatchConstruction::usable_vertex
        const bool usable = finite(f3(a.position_drop)) && finite(d) && finite(f3(a.basis_x)) &&
                            fabsf(dot(d, d) - 1.0f) <= 0x1p-16f && cycles_ok(a.optical_cycles) && finite(a.field);
        if (a.status != 1u || !usable) return;
        corners[i] = d;
    }
    if (!fold_config_ok(config)) return;
    Fold g;
    r.flags = fold_init(g, corners);
    if (r.flags != kFoldReady) return;
    for (unsigned i = 0; i < 4; ++i) r.jacobian[i] = g.j[i];
    if (!fold_components(g, r)) {
        r.flags = kFoldTopology;
        return;
    }
    double area = 0;
    for (unsigned i = 0; i < r.branch_count; ++i) {
        if (!fold_integrate(g, r.branches[i], config, r)) {
            r.flags = kFoldUnconverged;
            return;
        }
        area += r.branches[i].area_fraction;
    }
    // a consistency check, not a normalisation
    if (!finite64(area) || fabs(area - 1) > 8 * config.relative_tolerance) {
        r.flags = kFoldInvalidMetric;
        return;
    }
    if (focal)
        for (unsigned i = 0; i < r.branch_count; ++i) {
            icp_folded_branch& b = r.branches[i];
            uint32_t family = 0, extra = 0, turns = 0;
            b.focal_flags = focal_estimate(vertices, vertex_count, patch, incident, *focal, family, extra, turns,
                                           b.representative_u, b.representative_v, false);
            if (b.focal_flags == 0u) {
                b.quarter_turns = turns;
                b.extra_quarter_turn = extra;
            }
        }
}

// Records by compact patch index (rainbow::FoldedPatchView).
struct FoldView {
    const uint32_t* indices;
    const icp_folded_record* records;
    uint32_t patch_count, record_count;
};
__device__ __forceinline__ bool fold_enabled(const FoldView& f) { return f.indices && f.records; }
__device__ __forceinline__ const icp_folded_record* fold_find(const FoldView& f, uint32_t compact)
{
    if (!fold_enabled(f) || compact >= f.patch_count) return nullptr;
    const uint32_t i = f.indices[compact];
    if (i >= f.record_count) return nullptr;
    const icp_folded_record* r = f.records + i;
    return r->compact_index == compact ? r : nullptr;
}

// ------------------------------------------------------------ per hit, per direction
struct Compensated {
    double s = 0, c = 0;
    __device__ __forceinline__ void add(double x)
    {
        const double n = s + x;
        c += fabs(s) >= fabs(x) ? (s - n) + x : (x - n) + s;
        s = n;
    }
    __device__ __forceinline__ double value() const { return s + c; }
};
struct FieldSum {
    Compensated sr, si, pr, pi;
    __device__ __forceinline__ void add(const icp_field64& f)
    {
        sr.add(f.s_real);
        si.add(f.s_imag);
        pr.add(f.p_real);
        pi.add(f.p_imag);
    }
    __device__ __forceinline__ icp_field64 value() const { return {sr.value(), si.value(), pr.value(), pi.value()}; }
};
struct Contribution {
    icp_field64 field[2];
    double inc_s, inc_p;
};
__device__ __forceinline__ double lerp2(double a, double b, double c, double d, double u, double v)
{
    const double lower = fma(u, b - a, a), upper = fma(u, d - c, c);
    return fma(v, upper - lower, lower);
}

__device__ uint32_t hit_optics(const icp_optics_input& in, const icp_outgoing_patch& patch, const icp_query_hit& hit,
                               F3 dir, const Frame& target, Contribution& out, const icp_folded_record* folded,
                               const icp_folded_branch*& used)
{
    used = nullptr;
    if (!in.vertices || (hit.flags & ~(1u | 2u | 4u)) != 0u || hit.patch_id != patch.patch_id || hit.root_index > 1u ||
        !(hit.u >= 0.0f && hit.u <= 1.0f && hit.v >= 0.0f && hit.v <= 1.0f) || !(hit.t > 0.0f && finite32(hit.t)) ||
        !(hit.residual >= 0.0f && finite32(hit.residual)))
        return kInput;
    uint32_t pending = 0;
    const icp_folded_branch* branch = nullptr;
    if (patch.status == 3u) {
        // a folded patch: the branch of the hit's (u, v), when a ready record exists
        if (!folded || folded->patch_id != patch.patch_id || folded->compact_index != hit.compact_index ||
            folded->flags != kFoldReady)
            pending |= kRefine;
        else {
            const int b = fold_branch_at(*folded, double(hit.u), double(hit.v));
            if (b < 0) pending |= kSingular;
            else branch = &folded->branches[b];
        }
    } else if (patch.status != 1u && patch.status != 2u)
        return kInput;
    if (hit.flags & 1u) pending |= kBoundary;
    if (hit.flags & 2u) pending |= kSingular;
    if (pending) return pending;
    const double area = branch ? double(patch.incident_area_drop2) * branch->area_fraction
                               : double(patch.incident_area_drop2);
    const double omega = branch ? branch->solid_angle_sr : fabs(double(patch.signed_solid_angle_sr));
    if (!(area > 0.0 && finite64(area) && omega > 0.0 && finite64(omega))) return kInput;
    const unsigned columns = in.second_input_fields ? 2u : 1u;
    const double weight = in.second_input_fields ? 0.5 : 1.0;
    icp_field32 moved[2][4];
    icp_phase_cycles paths[4];
    for (unsigned k = 0; k < 4; ++k) {
        const uint32_t idx = patch.vertex_indices[k];
        if (idx >= in.vertex_count) return kInput;
        const icp_outgoing_vertex& vx = in.vertices[idx];
        const F3 dirv = f3(vx.direction_drop), basis = f3(vx.basis_x);
        if (vx.status != 1u || !finite(f3(vx.position_drop)) || !finite(dirv) || !finite(basis) || !finite(vx.field))
            return kInput;
        if (!cycles_ok(vx.optical_cycles)) return kPhase;
        const F3 second = cross(dirv, basis);
        const D3 s2 = wide(second);
        const double len2 = dot(s2, s2);
        if (!(len2 > 0.0 && finite64(len2))) return kFrame;
        const Frame source{basis, unit(second)};
        icp_field32 src[2] = {vx.field, vx.field};
        if (in.second_input_fields) {
            src[1] = in.second_input_fields[idx];
            if (!finite(src[0]) || !finite(src[1])) return kInput;
        }
        icp_field32 got[2];
        if (!transport(dirv, source, src, columns, dir, target, got)) return kFrame;
        moved[0][k] = got[0];
        moved[1][k] = columns == 2 ? got[1] : got[0];
        paths[k] = vx.optical_cycles;
    }
    icp_phase_cycles path;
    if (!cycles_bilinear(paths, hit.u, hit.v, path)) return kPhase;
    float pre, pim;
    if (!unit_phasor(path, pre, pim)) return kPhase;
    const double amplitude = sqrt(area / omega);
    const double c = pre, s = pim, u = hit.u, v = hit.v;
    Contribution cand{};
    for (unsigned j = 0; j < columns; ++j) {
        const icp_field32* f = moved[j];
        const double sr = amplitude * lerp2(f[0].x.real, f[1].x.real, f[2].x.real, f[3].x.real, u, v);
        const double si = amplitude * lerp2(f[0].x.imag, f[1].x.imag, f[2].x.imag, f[3].x.imag, u, v);
        const double pr = amplitude * lerp2(f[0].y.real, f[1].y.real, f[2].y.real, f[3].y.real, u, v);
        const double pi = amplitude * lerp2(f[0].y.imag, f[1].y.imag, f[2].y.imag, f[3].y.imag, u, v);
        cand.inc_s += weight * fma(sr, sr, si * si);
        cand.inc_p += weight * fma(pr, pr, pi * pi);
        cand.field[j] = {fma(sr, c, -si * s), fma(sr, s, si * c), fma(pr, c, -pi * s), fma(pr, s, pi * c)};
    }
    if (!finite64(cand.inc_s) || !finite64(cand.inc_p) || !finite(cand.field[0]) || !finite(cand.field[1]))
        return kArith;
    out = cand;
    used = branch;
    return 0;
}

__device__ __forceinline__ void unavailable(icp_optical_result& r)
{
    r.path_field = {nan64(), nan64(), nan64(), nan64()};
    r.path_field_second = r.path_field;
    r.incoherent_s = r.incoherent_p = r.path_s = r.path_p = nan64();
}
__device__ __forceinline__ void unavailable(icp_focal_sample& r)
{
    for (unsigned k = 0; k < 4; ++k) r.field[k] = r.field_second[k] = nan64();
    r.intensity_s = r.intensity_p = nan64();
}
__device__ __forceinline__ bool hit_before(const icp_query_hit& a, const icp_query_hit& b)
{
    if (a.patch_id != b.patch_id) return a.patch_id < b.patch_id;
    if (a.compact_index != b.compact_index) return a.compact_index < b.compact_index;
    return a.root_index < b.root_index;
}

__device__ void direction_optics(const icp_optics_input& in, uint32_t index, const icp_focal_config* fc,
                                 icp_optical_result& res, icp_focal_sample* focal_out, const FoldView& folded)
{
    res = icp_optical_result{};
    res.first_problem_patch_id = 0xffffffffu;
    const bool dual = in.input_polarization == 1u;
    const unsigned columns = dual ? 2u : 1u;
    const double weight = dual ? 0.5 : 1.0;
    if (focal_out) {
        *focal_out = icp_focal_sample{};
        focal_out->first_problem_patch_id = 0xffffffffu;
        focal_out->flags = kFocalInputError;
        unavailable(*focal_out);
    }
    if ((in.input_polarization != 0u && !dual) ||
        (dual && (!in.second_input_fields || in.second_input_count != in.vertex_count)) ||
        (!dual && (in.second_input_fields || in.second_input_count != 0u)) || index >= in.direction_count ||
        !in.directions || !in.offsets || !in.summaries) {
        res.flags = kInput;
        unavailable(res);
        return;
    }
    const icp_query_summary sm = in.summaries[index];
    res.hit_count = sm.hit_count;
    res.query_flags = sm.flags;
    if (sm.flags & kQueryErrors) {
        res.flags = kQuery;
        res.first_problem_patch_id = sm.first_problem_patch_id;
        res.rejected_hits = sm.hit_count;
        unavailable(res);
        return;
    }
    const uint64_t begin = in.offsets[index], end = in.offsets[index + 1u];
    if (begin > end || end > in.hit_storage_count || uint64_t(sm.hit_count) > end - begin ||
        uint64_t(sm.candidate_count) != end - begin || (sm.hit_count != 0u && (!in.hits || !in.patches || !in.vertices))) {
        res.flags = kInput;
        res.rejected_hits = sm.hit_count;
        unavailable(res);
        return;
    }
    // a refinement hit stays pending unless folded records are supplied, and then only where a
    // record accounts for it (checked after the loop)
    if ((sm.flags & kQueryRefineHit) && !fold_enabled(folded)) res.flags |= kRefine;
    if (sm.flags & kQueryBoundaryHit) res.flags |= kBoundary;
    if (sm.flags & kQuerySingularHit) res.flags |= kSingular;
    const F3 dir = f3(in.directions[index]);
    Frame target;
    if (!scattering_frame(f3(in.incident_direction), f3(in.incident_basis_x), dir, target)) {
        res.flags |= kFrame;
        res.rejected_hits = sm.hit_count;
        unavailable(res);
        return;
    }
    FieldSum path[2], turned[2];
    Compensated inc_s, inc_p, envelope[4];
    const bool with_focal = fc && focal_out;
    icp_focal_sample focal{};
    focal.first_problem_patch_id = 0xffffffffu;
    if (with_focal && !focal_layout_ok(*fc)) focal.flags |= kFocalGeometry;
    uint32_t recorded_nonregular = 0;
    for (uint32_t i = 0; i < sm.hit_count; ++i) {
        const icp_query_hit hit = in.hits[begin + i];
        uint32_t flags;
        Contribution ct{};
        const icp_folded_branch* used = nullptr;
        if (i != 0u && !hit_before(in.hits[begin + i - 1u], hit))
            flags = kInput; // the query sorts its hits and removes duplicates
        else if (hit.compact_index >= in.patch_count)
            flags = kInput;
        else {
            const icp_outgoing_patch& patch = in.patches[hit.compact_index];
            recorded_nonregular += patch.status == 3u;
            flags = hit_optics(in, patch, hit, dir, target, ct, fold_find(folded, hit.compact_index), used);
        }
        if (flags) {
            res.flags |= flags;
            ++res.rejected_hits;
            res.refinement_hits += (flags & kRefine) != 0u;
            res.boundary_hits += (flags & kBoundary) != 0u;
            res.singular_hits += (flags & kSingular) != 0u;
            if (hit.patch_id < res.first_problem_patch_id) res.first_problem_patch_id = hit.patch_id;
            continue;
        }
        ++res.evaluated_hits;
        res.folded_hits += used != nullptr;
        for (unsigned j = 0; j < columns; ++j) path[j].add(ct.field[j]);
        inc_s.add(ct.inc_s);
        inc_p.add(ct.inc_p);
        if (with_focal) {
            uint32_t family = 0, extra = 0, turns = 0, code;
            if (used) { // the branch's quarter turns, estimated at its representative point
                code = used->focal_flags;
                if (focal_layout_ok(*fc)) {
                    const uint32_t cells = (fc->grid_width - 1u) * (fc->grid_height - 1u);
                    family = hit.patch_id / cells;
                    if (family >= 4) code |= kFocalGeometry;
                    turns = used->quarter_turns;
                    extra = used->extra_quarter_turn;
                } else
                    code |= kFocalGeometry;
            } else
                code = focal_estimate(in.vertices, in.vertex_count, in.patches[hit.compact_index],
                                      f3(in.incident_direction), *fc, family, extra, turns);
            if (code) {
                focal.flags |= code;
                if (hit.patch_id < focal.first_problem_patch_id) focal.first_problem_patch_id = hit.patch_id;
            } else {
                for (unsigned j = 0; j < columns; ++j) turned[j].add(quarter_turns(ct.field[j], turns));
                envelope[family].add(ct.inc_s + ct.inc_p);
                ++focal.family_hits[family];
                ++focal.corrected_hits;
                focal.extra_quarter_turn_hits += extra;
            }
        }
    }
    if (fold_enabled(folded) && (sm.flags & kQueryRefineHit)) {
        if (recorded_nonregular == 0u) res.flags |= kRefine;
        if (recorded_nonregular != sm.refinement_hits) res.flags |= kInput;
    }
    res.path_field = path[0].value();
    res.path_field_second = path[1].value();
    res.incoherent_s = inc_s.value();
    res.incoherent_p = inc_p.value();
    for (unsigned j = 0; j < columns; ++j) {
        const icp_field64 f = path[j].value();
        res.path_s += weight * fma(f.s_real, f.s_real, f.s_imag * f.s_imag);
        res.path_p += weight * fma(f.p_real, f.p_real, f.p_imag * f.p_imag);
    }
    if (!finite(res.path_field) || !finite(res.path_field_second) || !finite64(res.incoherent_s) ||
        !finite64(res.incoherent_p) || !finite64(res.path_s) || !finite64(res.path_p))
        res.flags |= kArith;
    if (res.flags & kErrors) unavailable(res);
    if (with_focal) {
        if (res.flags & kErrors) focal.flags |= kFocalInputError;
        if (res.flags & kPending) focal.flags |= kFocalInputPending;
        if (res.first_problem_patch_id < focal.first_problem_patch_id)
            focal.first_problem_patch_id = res.first_problem_patch_id;
        const icp_field64 g0 = turned[0].value(), g1 = turned[1].value();
        focal.field[0] = g0.s_real, focal.field[1] = g0.s_imag, focal.field[2] = g0.p_real, focal.field[3] = g0.p_imag;
        focal.field_second[0] = g1.s_real, focal.field_second[1] = g1.s_imag;
        focal.field_second[2] = g1.p_real, focal.field_second[3] = g1.p_imag;
        for (unsigned j = 0; j < columns; ++j) {
            const icp_field64& f = j == 0 ? g0 : g1;
            focal.intensity_s += weight * fma(f.s_real, f.s_real, f.s_imag * f.s_imag);
            focal.intensity_p += weight * fma(f.p_real, f.p_real, f.p_imag * f.p_imag);
        }
        for (unsigned k = 0; k < 4; ++k) focal.family_incoherent[k] = envelope[k].value();
        if (!finite(g0) || !finite(g1) || !finite64(focal.intensity_s + focal.intensity_p)) focal.flags |= kFocalArith;
        if (focal.flags) unavailable(focal);
        *focal_out = focal;
    }
}

__global__ void __launch_bounds__(kThreads) patch_optics_kernel(const icp_optics_input in, const icp_focal_config fc,
                                                                int with_focal, const FoldView folded,
                                                                icp_optical_result* __restrict__ results,
                                                                icp_focal_sample* __restrict__ focal)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < in.direction_count; i += stride) {
        icp_optical_result r;
        if (with_focal) {
            icp_focal_sample f;
            direction_optics(in, i, &fc, r, &f, folded);
            focal[i] = f;
        } else
            direction_optics(in, i, nullptr, r, nullptr, folded);
        results[i] = r;
    }
}

// ------------------------------------------------------------ folded records: slots and build
// The NeedsRefinement patches get record slots in compact-index order (a block count, one
// scan, a ballot rank), so the records' order does not depend on scheduling.
constexpr unsigned kFoldThreads = 256;
__global__ void __launch_bounds__(kFoldThreads) fold_count_kernel(const icp_outgoing_patch* __restrict__ patches,
                                                                   uint32_t patch_count, uint32_t* __restrict__ counts)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const int flag = i < patch_count && patches[i].status == 3u;
    const int n = __syncthreads_count(flag);
    if (threadIdx.x == 0) counts[blockIdx.x] = uint32_t(n);
}
// exclusive scan of `n` block counts in place (one block), the total into *total
__global__ void __launch_bounds__(1024) fold_scan_kernel(uint32_t* __restrict__ counts, uint32_t n,
                                                         uint32_t* __restrict__ total)
{
    __shared__ uint32_t warp_sums[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (uint32_t base = 0; base < n; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t x = i < n ? counts[i] : 0u;
        uint32_t incl = x;
        for (unsigned o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) warp_sums[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = lane < (blockDim.x >> 5) ? warp_sums[lane] : 0u;
            for (unsigned o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            warp_sums[lane] = w; // inclusive over warps
        }
        __syncthreads();
        const uint32_t before = (warp ? warp_sums[warp - 1] : 0u) + carry;
        if (i < n) counts[i] = before + incl - x;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = before + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}
__global__ void __launch_bounds__(kFoldThreads) fold_slot_kernel(const icp_outgoing_patch* __restrict__ patches,
                                                                  uint32_t patch_count, const uint32_t* __restrict__ offsets,
                                                                  uint32_t* __restrict__ indices, uint32_t* __restrict__ list)
{
    __shared__ uint32_t warp_counts[kFoldThreads / 32];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool flag = i < patch_count && patches[i].status == 3u;
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned ballot = __ballot_sync(0xffffffffu, flag);
    if (lane == 0) warp_counts[warp] = __popc(ballot);
    __syncthreads();
    uint32_t rank = __popc(ballot & ((1u << lane) - 1u));
    for (unsigned w = 0; w < warp; ++w) rank += warp_counts[w];
    if (i < patch_count) {
        const uint32_t slot = offsets[blockIdx.x] + rank;
        indices[i] = flag ? slot : 0xffffffffu;
        if (flag) list[slot] = i;
    }
}
// one thread per record: the quadrature's panel count varies, so the records are dense and
// the launch covers only them.  acc: [0] prepared, [1] unresolved, [2] branches, [3] focal-
// pending branches, [4] largest estimated error (bits of a non-negative double)
__global__ void __launch_bounds__(64) fold_prepare_kernel(const icp_outgoing_vertex* __restrict__ vertices,
                                                          uint32_t vertex_count, const icp_outgoing_patch* __restrict__ patches,
                                                          const uint32_t* __restrict__ list, uint32_t count, F3 incident,
                                                          icp_focal_config focal, int with_focal, icp_folded_config config,
                                                          icp_folded_record* __restrict__ records,
                                                          unsigned long long* __restrict__ acc)
{
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= count) return;
    const uint32_t compact = list[slot];
    icp_folded_record r;
    fold_prepare(vertices, vertex_count, patches[compact], compact, incident, with_focal ? &focal : nullptr, config, r);
    records[slot] = r;
    if (r.flags == kFoldReady) {
        atomicAdd(&acc[0], 1ull);
        atomicAdd(&acc[2], (unsigned long long)r.branch_count);
        unsigned long long pend = 0;
        for (unsigned b = 0; with_focal && b < r.branch_count; ++b) pend += r.branches[b].focal_flags != 0u;
        if (pend) atomicAdd(&acc[3], pend);
        atomicMax(&acc[4], (unsigned long long)__double_as_longlong(r.largest_estimated_relative_error + 0.0));
    } else
        atomicAdd(&acc[1], 1ull);
}

// ------------------------------------------------------------ stage density and audit
__global__ void __launch_bounds__(256) stage_density_kernel(uint32_t stage, const icp_optical_result* __restrict__ optical,
                                                            const icp_focal_sample* __restrict__ focal,
                                                            const icp_diffraction_result* __restrict__ diffraction,
                                                            uint64_t count, double* __restrict__ density,
                                                            unsigned long long* __restrict__ acc)
{
    // acc: [0] max (bits of a non-negative double), [1] invalid, [2] incomplete, [3] underresolved,
    //      [4] first problem
    unsigned long long invalid = 0, incomplete_n = 0, under_n = 0, first = ~0ull, maxbits = 0;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride) {
        const icp_optical_result& o = optical[i];
        bool incomplete = (o.flags & (kErrors | kPending)) != 0u || o.rejected_hits != 0u || o.evaluated_hits != o.hit_count;
        bool under = false;
        double d;
        if (stage == ICP_STAGE_INCOHERENT)
            d = o.incoherent_s + o.incoherent_p;
        else if (stage == ICP_STAGE_PATH)
            d = o.path_s + o.path_p;
        else {
            incomplete = incomplete || focal[i].flags != 0u;
            if (stage == ICP_STAGE_FOCAL)
                d = focal[i].intensity_s + focal[i].intensity_p;
            else {
                const icp_diffraction_result& r = diffraction[i];
                incomplete = incomplete || (r.flags & (ICP_DIFFRACTION_INPUT_UNAVAILABLE | ICP_DIFFRACTION_STENCIL_UNAVAILABLE |
                                                       ICP_DIFFRACTION_DETECTION_UNAVAILABLE | ICP_DIFFRACTION_INVALID_DATA)) != 0u;
                under = (r.flags & ICP_DIFFRACTION_UNDERRESOLVED) != 0u;
                d = r.intensity_s + r.intensity_p;
            }
        }
        density[i] = d;
        const bool bad = !finite64(d) || d < 0;
        invalid += bad;
        incomplete_n += incomplete;
        under_n += under;
        if ((bad || incomplete || under) && i < first) first = i;
        if (!bad) {
            const unsigned long long bits = (unsigned long long)__double_as_longlong(d + 0.0); // -0 -> +0
            if (bits > maxbits) maxbits = bits;
        }
    }
    for (unsigned off = 16; off; off >>= 1) {
        invalid += __shfl_down_sync(0xffffffffu, invalid, off);
        incomplete_n += __shfl_down_sync(0xffffffffu, incomplete_n, off);
        under_n += __shfl_down_sync(0xffffffffu, under_n, off);
        const unsigned long long f = __shfl_down_sync(0xffffffffu, first, off);
        const unsigned long long m = __shfl_down_sync(0xffffffffu, maxbits, off);
        first = f < first ? f : first;
        maxbits = m > maxbits ? m : maxbits;
    }
    if ((threadIdx.x & 31u) == 0) {
        if (maxbits) atomicMax(&acc[0], maxbits);
        if (invalid) atomicAdd(&acc[1], invalid);
        if (incomplete_n) atomicAdd(&acc[2], incomplete_n);
        if (under_n) atomicAdd(&acc[3], under_n);
        if (first != ~0ull) atomicMin(&acc[4], first);
    }
}

} // namespace

extern "C" int icp_stage_density(icp_context* ctx, uint32_t stage, const icp_optical_result* d_optical,
                                 const icp_focal_sample* d_focal, const icp_diffraction_result* d_diffraction,
                                 uint64_t count, double* d_density, icp_density_report* report)
{
    if (!ctx || !d_optical || !d_density || !report || stage < ICP_STAGE_INCOHERENT || stage > ICP_STAGE_DIFFRACTION ||
        (stage >= ICP_STAGE_FOCAL && !d_focal) || (stage == ICP_STAGE_DIFFRACTION && !d_diffraction))
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_stage_density: invalid stage or null argument");
    ICP_CUDA(cudaSetDevice(ctx->device));
    ICP_CUDA(ctx->stage_audit.ensure(5 * sizeof(unsigned long long)));
    auto* acc = static_cast<unsigned long long*>(ctx->stage_audit.ptr);
    const unsigned long long init[5] = {0ull, 0ull, 0ull, 0ull, ~0ull};
    ICP_CUDA(cudaMemcpyAsync(acc, init, sizeof init, cudaMemcpyHostToDevice, ctx->stream));
    if (count) {
        const uint64_t need = (count + 255) / 256, cap = uint64_t(ctx->sms > 0 ? ctx->sms : 148) * 8u;
        stage_density_kernel<<<unsigned(need < cap ? need : cap), 256, 0, ctx->stream>>>(stage, d_optical, d_focal,
                                                                                        d_diffraction, count, d_density, acc);
        ICP_CUDA(cudaGetLastError());
        count_launch();
    }
    unsigned long long got[5];
    ICP_CUDA(cudaMemcpyAsync(got, acc, sizeof got, cudaMemcpyDeviceToHost, ctx->stream));
    ICP_CUDA(cudaStreamSynchronize(ctx->stream));
    double m;
    std::memcpy(&m, &got[0], sizeof m);
    *report = {m, got[1], got[2], got[3], got[4]};
    return ok();
}

extern "C" int icp_patch_optics_folded(icp_context* ctx, const icp_optics_input* input, icp_optical_result* d_results,
                                       const icp_focal_config* focal, icp_focal_sample* d_focal,
                                       const icp_folded_view* folded)
{
    if (!ctx || !input || !d_results || (focal && !d_focal))
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_patch_optics: null argument");
    if (folded && (!folded->record_indices != !folded->records))
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_patch_optics: a folded view needs both its index and record arrays");
    if (input->direction_count == 0) return ok();
    if (input->direction_count > 0x7fffffffu) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_patch_optics: too many directions");
    ICP_CUDA(cudaSetDevice(ctx->device));
    const uint64_t need = (uint64_t(input->direction_count) + kThreads - 1) / kThreads;
    const uint64_t cap = uint64_t(ctx->sms > 0 ? ctx->sms : 148) * 16u;
    const unsigned blocks = unsigned(need < cap ? need : cap);
    const icp_focal_config fc = focal ? *focal : icp_focal_config{};
    FoldView view{nullptr, nullptr, 0u, 0u};
    if (folded) view = {folded->record_indices, folded->records, folded->patch_count, folded->record_count};
    patch_optics_kernel<<<blocks, kThreads, 0, ctx->stream>>>(*input, fc, focal ? 1 : 0, view, d_results, d_focal);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    ICP_CUDA(cudaStreamSynchronize(ctx->stream));
    return ok();
}

extern "C" int icp_patch_optics(icp_context* ctx, const icp_optics_input* input, icp_optical_result* d_results,
                                const icp_focal_config* focal, icp_focal_sample* d_focal)
{
    return icp_patch_optics_folded(ctx, input, d_results, focal, d_focal, nullptr);
}

extern "C" int icp_folded_prepare(icp_context* ctx, const icp_outgoing_vertex* d_vertices, uint32_t vertex_count,
                                  const icp_outgoing_patch* d_patches, uint32_t patch_count, const float incident[3],
                                  const icp_focal_config* focal, const icp_folded_config* config,
                                  uint32_t* d_record_indices, icp_folded_record* d_records, uint32_t capacity,
                                  uint32_t* record_count, icp_folded_stats* stats)
{
    if (!ctx || !d_vertices || !d_patches || !incident || !d_record_indices || !record_count)
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_folded_prepare: null argument");
    icp_folded_config cfg{1e-8, 2048u, 20u};
    if (config) cfg = *config;
    if (!(cfg.relative_tolerance >= 1e-12 && cfg.relative_tolerance <= 1e-3 && cfg.maximum_panels >= 1 &&
          cfg.maximum_panels <= 65536 && cfg.maximum_depth >= 1 && cfg.maximum_depth <= 24))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid folded-patch quadrature settings.");
    *record_count = 0;
    if (stats) std::memset(stats, 0, sizeof *stats);
    if (patch_count == 0) return ok();
    ICP_CUDA(cudaSetDevice(ctx->device));
    const uint32_t blocks = (patch_count + kFoldThreads - 1) / kFoldThreads;
    // scratch: block counts / offsets, the total, the candidate list, the statistics
    const size_t counts_bytes = sizeof(uint32_t) * (size_t(blocks) + 1);
    const size_t list_off = (counts_bytes + 255) / 256 * 256;
    const size_t acc_off = list_off + (sizeof(uint32_t) * size_t(patch_count) + 255) / 256 * 256;
    ICP_CUDA(ctx->folded.ensure(acc_off + 5 * sizeof(unsigned long long)));
    char* base = static_cast<char*>(ctx->folded.ptr);
    auto* counts = reinterpret_cast<uint32_t*>(base);
    uint32_t* total = counts + blocks;
    auto* list = reinterpret_cast<uint32_t*>(base + list_off);
    auto* acc = reinterpret_cast<unsigned long long*>(base + acc_off);
    fold_count_kernel<<<blocks, kFoldThreads, 0, ctx->stream>>>(d_patches, patch_count, counts);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    fold_scan_kernel<<<1, 1024, 0, ctx->stream>>>(counts, blocks, total);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    fold_slot_kernel<<<blocks, kFoldThreads, 0, ctx->stream>>>(d_patches, patch_count, counts, d_record_indices, list);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    uint32_t n = 0;
    ICP_CUDA(cudaMemcpyAsync(&n, total, sizeof n, cudaMemcpyDeviceToHost, ctx->stream));
    ICP_CUDA(cudaStreamSynchronize(ctx->stream));
    *record_count = n;
    if (stats) stats->candidates = n;
    if (n == 0) return ok();
    if (!d_records || capacity < n)
        return fail(ICP_ERR_CAPACITY, "icp_folded_prepare: %u folded-patch records need room, capacity is %u", n, capacity);
    ICP_CUDA(cudaMemsetAsync(acc, 0, 5 * sizeof(unsigned long long), ctx->stream));
    const icp_focal_config fc = focal ? *focal : icp_focal_config{};
    fold_prepare_kernel<<<(n + 63) / 64, 64, 0, ctx->stream>>>(d_vertices, vertex_count, d_patches, list, n,
                                                               F3{incident[0], incident[1], incident[2]}, fc,
                                                               focal ? 1 : 0, cfg, d_records, acc);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    unsigned long long h[5];
    ICP_CUDA(cudaMemcpyAsync(h, acc, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    ICP_CUDA(cudaStreamSynchronize(ctx->stream));
    if (stats) {
        stats->prepared = uint32_t(h[0]);
        stats->unresolved = uint32_t(h[1]);
        stats->branch_count = uint32_t(h[2]);
        stats->focal_pending_branches = uint32_t(h[3]);
        std::memcpy(&stats->largest_estimated_relative_error, &h[4], sizeof(double));
    }
    return ok();
}
