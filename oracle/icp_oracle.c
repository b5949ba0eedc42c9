/*
 * icp_oracle.c -- CPU restatement of the reference phase-function path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product
 * path; nothing in the product links, loads or calls it.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
 *
 * It restates, in plain C (binary64, no FMA contraction, same operation
 * order), the algorithm of the reference hex-prism Monte Carlo path of
 * Somatic-Cell/ice-crystal-phase:
 *   counter RNG            hex_trace/include/ice_crystal/math.hpp:136-146
 *   vectors / frames       hex_trace/include/ice_crystal/math.hpp:23-133
 *   prism geometry         hex_trace/include/ice_crystal/hex_prism.hpp:10-175
 *   Fresnel flux split     hex_trace/include/ice_crystal/flux_interface.hpp:13-88
 *   linear R/T chain       hex_trace/include/ice_crystal/hex_trace_core.hpp:155-259
 *   (u,phi) binning        hex_phase/include/ice_crystal/phase_math.hpp:37-81
 *   Kahan mass histogram   hex_phase/src/phase_table.cpp:39-103
 *   CPU CDF builder        hex_phase/src/phase_table.cpp:104-187
 *   u edges                include/rainbow/phase_cdf_math.hpp:16-32
 *   quaternion rotation    hex_phase/src/phase_table.cpp:11-21
 *   Table-II diffraction   include/rainbow/rainbow_diffraction.hpp:16-174
 *   patch optics           include/rainbow/patch_optical_evaluator.hpp:26-326 (+ transport,
 *                          phase cycles, focal phase)
 *   patch construction     include/rainbow/patch_geometry.hpp:75-172
 *   ray / patch hits       include/rainbow/bilinear_patch_intersection.hpp:58-314
 *   all-hit query          shaders/entry/patch_query.cu, include/rainbow/patch_query_data.hpp:43-128
 * Parity is pinned: tests compare this restatement bit-for-bit with the
 * reference sources compiled from their own files into oracle/_ref
 * (oracle/build_ref.sh) and with fixtures under tests/golden/.  The query's box test is
 * the one part with no reference counterpart to pin (the reference leaves it to OptiX).
 *
 * Build: oracle/build_oracle.sh (gcc -O2 -ffp-contract=off -fno-fast-math).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ICPO_PI 3.141592653589793238462643383279502884
#define ICPO_SQRT3 1.732050807568877293527446341505872367
#define ICPO_EPS DBL_EPSILON

/* ---------------------------------------------------------------- scalars */
static int fin(double x) { return x >= -DBL_MAX && x <= DBL_MAX; }
static double mx(double a, double b) { return a > b ? a : b; }

typedef struct { double x, y, z; } v3;
static v3 v_add(v3 a, v3 b) { v3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static v3 v_sub(v3 a, v3 b) { v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static v3 v_neg(v3 a) { v3 r = {-a.x, -a.y, -a.z}; return r; }
static v3 v_mul(v3 a, double s) { v3 r = {a.x * s, a.y * s, a.z * s}; return r; }
static v3 v_div(v3 a, double s) { v3 r = {a.x / s, a.y / s, a.z / s}; return r; }
static double v_dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 v_cross(v3 a, v3 b)
{
    v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static int v_fin(v3 a) { return fin(a.x) && fin(a.y) && fin(a.z); }
static double v_maxabs(v3 a) { return mx(fabs(a.x), mx(fabs(a.y), fabs(a.z))); }

/* math.hpp:38-47: scale by the largest component first, then divide by the norm. */
static int v_normalize(v3 a, v3* out)
{
    double s = v_maxabs(a), n;
    if (!(s > 0) || !fin(s)) return 0;
    a = v_div(a, s);
    n = sqrt(v_dot(a, a));
    if (!(n > 0) || !fin(n)) return 0;
    *out = v_div(a, n);
    return v_fin(*out);
}
static int v_is_unit(v3 a) { return v_fin(a) && fabs(v_dot(a, a) - 1.0) <= 128 * ICPO_EPS; }

typedef struct { v3 e0, e1; } frame_t;
/* math.hpp:53-59 */
static int frame_valid(frame_t f, v3 k)
{
    return v_is_unit(k) && v_is_unit(f.e0) && v_is_unit(f.e1) &&
           fabs(v_dot(k, f.e0)) <= 128 * ICPO_EPS && fabs(v_dot(k, f.e1)) <= 128 * ICPO_EPS &&
           v_maxabs(v_sub(v_cross(k, f.e0), f.e1)) <= 256 * ICPO_EPS;
}
/* math.hpp:61-69: helper axis = the coordinate axis least aligned with k. */
static int make_frame(v3 k, frame_t* f)
{
    double ax, ay, az;
    v3 a;
    if (!v_is_unit(k)) return 0;
    ax = fabs(k.x); ay = fabs(k.y); az = fabs(k.z);
    if (ax <= ay && ax <= az) { a.x = 1; a.y = 0; a.z = 0; }
    else if (ay <= az) { a.x = 0; a.y = 1; a.z = 0; }
    else { a.x = 0; a.y = 0; a.z = 1; }
    if (!v_normalize(v_sub(a, v_mul(k, v_dot(k, a))), &f->e0)) return 0;
    if (!v_normalize(v_cross(k, f->e0), &f->e1)) return 0;
    return frame_valid(*f, k);
}

/* math.hpp:70-78 */
typedef struct { double re, im; } cplx;
static cplx c_add(cplx a, cplx b) { cplx r = {a.re + b.re, a.im + b.im}; return r; }
static cplx c_muld(cplx a, double b) { cplx r = {a.re * b, a.im * b}; return r; }
static cplx c_mul(cplx a, cplx b)
{
    cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}
static double c_norm2(cplx a) { return a.re * a.re + a.im * a.im; }

/* math.hpp:79-109: two response columns (unit incident fields), rows in the transverse frame. */
typedef struct { cplx x, y; } field_t;
typedef struct { field_t col[2]; } jones_t;
static jones_t jones_identity(void)
{
    jones_t j;
    memset(&j, 0, sizeof j);
    j.col[0].x.re = 1;
    j.col[1].y.re = 1;
    return j;
}
static double jones_power(const jones_t* j)
{
    return 0.5 * (c_norm2(j->col[0].x) + c_norm2(j->col[0].y) + c_norm2(j->col[1].x) + c_norm2(j->col[1].y));
}
static int jones_finite(const jones_t* j)
{
    int i;
    for (i = 0; i < 2; ++i)
        if (!fin(j->col[i].x.re) || !fin(j->col[i].x.im) || !fin(j->col[i].y.re) || !fin(j->col[i].y.im)) return 0;
    return 1;
}
static int jones_nonzero(const jones_t* j)
{
    int i;
    for (i = 0; i < 2; ++i)
        if (j->col[i].x.re != 0 || j->col[i].x.im != 0 || j->col[i].y.re != 0 || j->col[i].y.im != 0) return 1;
    return 0;
}
/* math.hpp:110-119 */
static jones_t change_frame(const jones_t* j, frame_t o, frame_t n)
{
    jones_t r;
    int c;
    for (c = 0; c < 2; ++c) {
        r.col[c].x = c_add(c_muld(j->col[c].x, v_dot(o.e0, n.e0)), c_muld(j->col[c].y, v_dot(o.e1, n.e0)));
        r.col[c].y = c_add(c_muld(j->col[c].x, v_dot(o.e0, n.e1)), c_muld(j->col[c].y, v_dot(o.e1, n.e1)));
    }
    return r;
}
/* math.hpp:120-124 */
static jones_t scale_rows(jones_t j, cplx s, cplx p)
{
    int c;
    for (c = 0; c < 2; ++c) {
        j.col[c].x = c_mul(j.col[c].x, s);
        j.col[c].y = c_mul(j.col[c].y, p);
    }
    return j;
}

/* math.hpp:125-133: Kahan sum with a separate correction term. */
typedef struct { double value, correction; } ksum;
static void ks_add(ksum* s, double x)
{
    double y = x - s->correction, t = s->value + y;
    s->correction = (t - s->value) - y;
    s->value = t;
}

/* math.hpp:136-146: SplitMix64 finaliser over a golden-ratio counter; 52-bit midpoints. */
static uint64_t mix64(uint64_t x)
{
    x = (x ^ (x >> 30)) * UINT64_C(0xbf58476d1ce4e5b9);
    x = (x ^ (x >> 27)) * UINT64_C(0x94d049bb133111eb);
    return x ^ (x >> 31);
}
double icpo_sample_uniform(uint64_t seed, uint64_t id, unsigned dim)
{
    uint64_t x = mix64(seed + UINT64_C(0x9e3779b97f4a7c15) * (3 * id + dim + 1));
    return ((double)(x >> 12) + 0.5) * 0x1p-52;
}

/* ----------------------------------------------------------- hex prism */
/* hex_prism.hpp:10-52: circumradius R, full length L, long axis +y; coordinates are x/R. */
typedef struct { double R, L; } prism_t;
static double pr_half(prism_t h) { return 0.5 * (h.L / h.R); }
static int pr_valid(prism_t h)
{
    return fin(h.R) && fin(h.L) && h.R > 0 && h.L > 0 && fin(pr_half(h)) && pr_half(h) > 0 &&
           fin(h.R * h.R) && h.R * h.R > 0 && fin(h.R * h.L) && h.R * h.L > 0;
}
static v3 pr_normal(unsigned f)
{
    v3 r = {0, 0, 0};
    switch (f) {
    case 0: r.x = 1; break;
    case 1: r.x = 0.5; r.z = ICPO_SQRT3 / 2; break;
    case 2: r.x = -0.5; r.z = ICPO_SQRT3 / 2; break;
    case 3: r.x = -1; break;
    case 4: r.x = -0.5; r.z = -ICPO_SQRT3 / 2; break;
    case 5: r.x = 0.5; r.z = -ICPO_SQRT3 / 2; break;
    case 6: r.y = 1; break;
    case 7: r.y = -1; break;
    default: break;
    }
    return r;
}
static v3 pr_vertex(unsigned f)
{
    v3 r = {0, 0, 0};
    switch (f % 6) {
    case 0: r.x = ICPO_SQRT3 / 2; r.z = 0.5; break;
    case 1: r.z = 1; break;
    case 2: r.x = -ICPO_SQRT3 / 2; r.z = 0.5; break;
    case 3: r.x = -ICPO_SQRT3 / 2; r.z = -0.5; break;
    case 4: r.z = -1; break;
    default: r.x = ICPO_SQRT3 / 2; r.z = -0.5; break;
    }
    return r;
}
static double pr_offset(prism_t h, unsigned f) { return f < 6 ? ICPO_SQRT3 / 2 : pr_half(h); }
static double pr_face_area(prism_t h, unsigned f) { return f < 6 ? h.R * h.L : (3 * ICPO_SQRT3 / 2) * h.R * h.R; }
double icpo_hex_projected_area(double R, double L, const double k[3])
{
    prism_t h = {R, L};
    v3 kk = {k[0], k[1], k[2]};
    ksum a = {0, 0};
    unsigned f;
    for (f = 0; f < 8; ++f) ks_add(&a, pr_face_area(h, f) * mx(0, -v_dot(pr_normal(f), kk)));
    return a.value;
}
static double pr_projected(prism_t h, v3 k)
{
    double kk[3] = {k.x, k.y, k.z};
    return icpo_hex_projected_area(h.R, h.L, kk);
}
/* hex_prism.hpp:54-57 */
static double geom_tol(prism_t h, v3 p, double t)
{
    return 128 * ICPO_EPS * mx(1, mx(pr_half(h), mx(v_maxabs(p), fabs(t))));
}

typedef struct { v3 pos; unsigned face; int valid; } entry_t;
/* hex_prism.hpp:64-98: face chosen in proportion to projected face area. */
static entry_t sample_entry(prism_t h, v3 k, double u0, double u1, double u2)
{
    entry_t s;
    double a, target, acc = 0;
    unsigned last = 8, f;
    memset(&s, 0, sizeof s);
    s.face = 8;
    if (!pr_valid(h) || !v_is_unit(k) || !(u0 >= 0 && u0 < 1 && u1 >= 0 && u1 < 1 && u2 >= 0 && u2 < 1)) return s;
    a = pr_projected(h, k);
    if (!(a > 0) || !fin(a)) return s;
    target = u0 * a;
    for (f = 0; f < 8; ++f) {
        double w = pr_face_area(h, f) * mx(0, -v_dot(pr_normal(f), k));
        if (!(w > 0)) continue;
        last = f;
        acc += w;
        if (target < acc) { s.face = f; break; }
    }
    if (s.face == 8) s.face = last;
    if (s.face == 8) return s;
    if (s.face < 6) {
        v3 n = pr_normal(s.face), tangent = {-n.z, 0, n.x}, axial = {0, (2 * u2 - 1) * pr_half(h), 0};
        s.pos = v_add(v_add(v_mul(n, ICPO_SQRT3 / 2), v_mul(tangent, u1 - 0.5)), axial);
    } else {
        double sector = 6 * u1, r;
        unsigned j = (unsigned)sector;
        r = sqrt(sector - (double)j);
        s.pos = v_mul(v_add(v_mul(pr_vertex(j), 1 - u2), v_mul(pr_vertex(j + 1), u2)), r);
        s.pos.y = (s.face == 6 ? 1 : -1) * pr_half(h);
    }
    s.valid = v_fin(s.pos);
    return s;
}

enum { HIT_REGULAR = 0, HIT_MISS = 1, HIT_AMBIGUOUS = 2, HIT_INVALID = 3 };
typedef struct { v3 pos; double t; unsigned face; int status; } hit_t;
/* hex_prism.hpp:108-120 */
static int strict_face_point(prism_t h, v3 p, unsigned face)
{
    double tol;
    unsigned f;
    if (face >= 8 || !v_fin(p)) return 0;
    tol = geom_tol(h, p, 0);
    for (f = 0; f < 8; ++f) {
        double gap = pr_offset(h, f) - v_dot(pr_normal(f), p);
        if (f == face) { if (fabs(gap) > tol) return 0; }
        else if (!(gap > tol)) return 0;
    }
    return 1;
}
/* hex_prism.hpp:123-147: nearest exit plane; an edge/vertex tie is reported as ambiguous. */
static hit_t next_boundary(prism_t h, v3 p, v3 d, unsigned start)
{
    hit_t hit;
    double best = DBL_MAX, second = DBL_MAX, tol;
    unsigned f;
    memset(&hit, 0, sizeof hit);
    hit.face = 8;
    hit.status = HIT_INVALID;
    if (!pr_valid(h) || !v_is_unit(d) || start >= 8) return hit;
    if (!strict_face_point(h, p, start)) { hit.status = HIT_AMBIGUOUS; return hit; }
    if (v_dot(pr_normal(start), d) > 128 * ICPO_EPS) return hit;
    for (f = 0; f < 8; ++f) {
        double cosine, t;
        if (f == start) continue;
        cosine = v_dot(pr_normal(f), d);
        if (!(cosine > 0)) continue;
        t = (pr_offset(h, f) - v_dot(pr_normal(f), p)) / cosine;
        if (!(t > 0) || !fin(t)) continue;
        if (t < best) { second = best; best = t; hit.face = f; }
        else if (t < second) second = t;
    }
    if (hit.face == 8) return hit;
    hit.t = best;
    hit.pos = v_add(p, v_mul(d, best));
    tol = geom_tol(h, hit.pos, best);
    if (second - best <= tol || !strict_face_point(h, hit.pos, hit.face)) hit.status = HIT_AMBIGUOUS;
    else hit.status = HIT_REGULAR;
    return hit;
}

/* ------------------------------------------------------ Fresnel (flux) */
typedef struct { v3 d; frame_t fr; jones_t j; } fray_t;
typedef struct { fray_t refl, trans; double balance; int valid, has_t, tir; } branches_t;
/* flux_interface.hpp:13-19 */
static cplx tir_phase(double a, double b)
{
    double s = mx(fabs(a), fabs(b)), den;
    cplx r;
    a /= s;
    b /= s;
    den = a * a + b * b;
    r.re = (a * a - b * b) / den;
    r.im = -2 * a * b / den;
    return r;
}
/* flux_interface.hpp:26-88: s/p split in flux normalisation; n points into the incident medium.
 * drop = 1 adds the drop interface's conventions (include/rainbow/dielectric_interface.hpp:
 * 86-91): a cosine down to -2^-19 is clamped to zero, and below sin^2 = 2^-40 the s axis is the
 * incident frame's e0.  It also re-orthogonalises s against the incident and each outgoing
 * direction (a no-op in exact arithmetic): near normal incidence d x n loses ~1e-16/sin of
 * its direction, which on a curved surface would otherwise fail the 128-ulp frame test. */
static v3 orthogonal_to(v3 s, v3 d)
{
    v3 o;
    if (!v_normalize(v_sub(s, v_mul(d, v_dot(d, s))), &o)) return s;
    return o;
}
static branches_t split_flux_graze(const fray_t* ray, v3 n, double ni, double nt, int drop)
{
    const double graze = drop ? 0x1p-19 : 0.0;
    branches_t b;
    double ci, scale, sine, ns, a, c, eta, st, before, after;
    v3 s, scaled, pin;
    jones_t j;
    frame_t spf;
    cplx rs = {0, 0}, rp = {0, 0};
    memset(&b, 0, sizeof b);
    if (!frame_valid(ray->fr, ray->d) || !v_is_unit(n) || !jones_finite(&ray->j) ||
        !(ni > 0 && nt > 0 && fin(ni) && fin(nt)))
        return b;
    ci = -v_dot(ray->d, n);
    if (ci < -graze || ci > 1 + 128 * ICPO_EPS) return b;
    if (ci < 0) ci = 0;
    if (ci > 1) ci = 1;
    if (ni == nt) {
        b.trans = *ray;
        b.has_t = 1;
        b.refl.d = v_add(ray->d, v_mul(n, 2 * ci));
        if (!v_normalize(b.refl.d, &b.refl.d)) return b;
        if (!make_frame(b.refl.d, &b.refl.fr)) return b;
        b.valid = 1;
        return b;
    }
    s = v_cross(ray->d, n);
    scale = v_maxabs(s);
    if (scale > 0) scaled = v_div(s, scale);
    else { scaled.x = 0; scaled.y = 0; scaled.z = 0; }
    sine = scale * sqrt(v_dot(scaled, scaled));
    if (drop) {
        if (sine * sine > 0x1p-40) { if (!v_normalize(s, &s)) return b; }
        else s = ray->fr.e0;
        s = orthogonal_to(s, ray->d);
    } else if (sine > 0) { if (!v_normalize(s, &s)) return b; }
    else s = ray->fr.e0;
    if (!v_normalize(v_cross(ray->d, s), &pin)) return b;
    spf.e0 = s;
    spf.e1 = pin;
    j = change_frame(&ray->j, ray->fr, spf);
    ns = mx(ni, nt);
    a = ni / ns;
    c = nt / ns;
    eta = a / c;
    if (!fin(eta) || !(a > 0 && c > 0)) return b;
    st = eta * sine;
    if (!fin(st)) return b;
    if (!v_normalize(v_add(ray->d, v_mul(n, 2 * ci)), &b.refl.d)) return b;
    b.refl.fr.e0 = drop ? orthogonal_to(s, b.refl.d) : s;
    if (!v_normalize(v_cross(b.refl.d, b.refl.fr.e0), &b.refl.fr.e1)) return b;
    if (st > 1) {
        double inverse = 1 / st, beta = st * sqrt((1 - inverse) * (1 + inverse));
        rs = tir_phase(a * ci, c * beta);
        rp = tir_phase(c * ci, a * beta);
        b.tir = 1;
    } else {
        double ct = sqrt((1 - st) * (1 + st)), ds = a * ci + c * ct, dp = c * ci + a * ct, numerator, ts, tp;
        cplx cts, ctp;
        if (!(ds > 0 && dp > 0)) return b;
        rs.re = (a * ci - c * ct) / ds;
        rp.re = (c * ci - a * ct) / dp;
        numerator = 2 * sqrt(a * ci) * sqrt(c * ct);
        ts = numerator / ds;
        tp = numerator / dp;
        cts.re = ts; cts.im = 0;
        ctp.re = tp; ctp.im = 0;
        b.trans.j = scale_rows(j, cts, ctp);
        if (!v_normalize(v_sub(v_mul(v_add(ray->d, v_mul(n, ci)), eta), v_mul(n, ct)), &b.trans.d)) return b;
        b.trans.fr.e0 = drop ? orthogonal_to(s, b.trans.d) : s;
        if (!v_normalize(v_cross(b.trans.d, b.trans.fr.e0), &b.trans.fr.e1)) return b;
        b.has_t = 1;
    }
    b.refl.j = scale_rows(j, rs, rp);
    before = jones_power(&ray->j);
    after = jones_power(&b.refl.j) + (b.has_t ? jones_power(&b.trans.j) : 0);
    b.balance = after - before;
    b.valid = frame_valid(b.refl.fr, b.refl.d) && jones_finite(&b.refl.j) &&
              (!b.has_t || (frame_valid(b.trans.fr, b.trans.d) && jones_finite(&b.trans.j))) &&
              fin(b.balance) && fabs(b.balance) <= 2048 * ICPO_EPS * mx(before, DBL_MIN);
    return b;
}
static branches_t split_flux(const fray_t* ray, v3 n, double ni, double nt)
{
    return split_flux_graze(ray, n, ni, nt, 0);
}

/* ----------------------------------------------------------- ray chain */
/* Status codes follow hex_trace_core.hpp:97-102. */
enum {
    ST_EXHAUSTED = 0, ST_TAIL = 1, ST_LIMIT = 2, ST_AMBIGUOUS = 3,
    ST_INVALID = 4, ST_NUMERICAL = 5, ST_OVERFLOW = 6, ST_REPLAY = 7
};

typedef struct {
    prism_t prism;
    v3 k;
    frame_t kf;
    double n_ext, n_int, tail;
    uint64_t seed, total;
    uint32_t max_hits;
} trace_cfg_t;

/* One emitted exit; the histogram consumes only its direction and power. */
typedef struct { v3 d; double power; } exit_t;

typedef struct {
    double escaped, unresolved, balance, max_iface;
    uint64_t outputs;
    uint32_t hits, tir;
    int status;
} ray_audit_t;

typedef void (*emit_fn)(void* user, v3 d, double power);

/* hex_trace_core.hpp:155-162 */
static int cfg_valid(const trace_cfg_t* c)
{
    double a = pr_projected(c->prism, c->k);
    return pr_valid(c->prism) && frame_valid(c->kf, c->k) && fin(c->n_ext) && fin(c->n_int) && c->n_ext > 0 &&
           c->n_int > 0 && fin(c->tail) && c->tail >= 0 && c->tail < 1 && c->total > 0 && c->max_hits > 0 &&
           fin(a) && a > 0;
}
static ray_audit_t finish_audit(ray_audit_t a, const ksum* esc, double residual, int status)
{
    a.escaped = esc->value;
    a.unresolved = residual;
    a.balance = esc->value + residual - 1;
    a.status = status;
    return a;
}
/* hex_trace_core.hpp:169-184 */
static int emit_exit(emit_fn emit, void* user, ray_audit_t* a, ksum* esc, const trace_cfg_t* c, const fray_t* ray, v3 pos)
{
    double power = jones_power(&ray->j);
    v3 pmm;
    if (!fin(power) || power < 0 || (!power && jones_nonzero(&ray->j))) return ST_NUMERICAL;
    if (power == 0) return ST_EXHAUSTED;
    pmm = v_mul(pos, c->prism.R);
    if (!v_fin(pmm)) return ST_NUMERICAL;
    if (emit) emit(user, ray->d, power);
    ks_add(esc, power);
    ++a->outputs;
    return ST_EXHAUSTED;
}
/* hex_trace_core.hpp:190-252: exterior R once, then T at every internal hit while R continues. */
static ray_audit_t trace_from_entry(const trace_cfg_t* c, uint64_t id, entry_t e, emit_fn emit, void* user)
{
    ray_audit_t a;
    ksum esc = {0, 0}, length = {0, 0};
    fray_t inc, ray;
    branches_t sp;
    v3 p;
    unsigned cur, encounter;
    int em;
    double remaining;
    memset(&a, 0, sizeof a);
    a.unresolved = 1;
    a.status = ST_INVALID;
    if (!cfg_valid(c) || id >= c->total || !e.valid || e.face >= 8) return finish_audit(a, &esc, 1, ST_INVALID);
    if (!strict_face_point(c->prism, e.pos, e.face)) return finish_audit(a, &esc, 1, ST_AMBIGUOUS);
    if (!(v_dot(pr_normal(e.face), c->k) < 0)) return finish_audit(a, &esc, 1, ST_INVALID);
    inc.d = c->k;
    inc.fr = c->kf;
    inc.j = jones_identity();
    sp = split_flux(&inc, pr_normal(e.face), c->n_ext, c->n_int);
    if (!sp.valid) return finish_audit(a, &esc, 1, ST_NUMERICAL);
    a.max_iface = fabs(sp.balance);
    em = emit_exit(emit, user, &a, &esc, c, &sp.refl, e.pos);
    if (em != ST_EXHAUSTED) return finish_audit(a, &esc, 1, em);
    if (!sp.has_t) { a.tir = 1; return finish_audit(a, &esc, 0, ST_EXHAUSTED); }
    ray = sp.trans;
    p = e.pos;
    cur = e.face;
    for (encounter = 0; encounter < c->max_hits; ++encounter) {
        double power = jones_power(&ray.j), segment;
        hit_t hit;
        if (!fin(power) || power < 0 || (!power && jones_nonzero(&ray.j))) return finish_audit(a, &esc, power, ST_NUMERICAL);
        if (power == 0) return finish_audit(a, &esc, 0, ST_EXHAUSTED);
        if (power <= c->tail) return finish_audit(a, &esc, power, ST_TAIL);
        hit = next_boundary(c->prism, p, ray.d, cur);
        if (hit.status != HIT_REGULAR)
            return finish_audit(a, &esc, power, hit.status == HIT_AMBIGUOUS ? ST_AMBIGUOUS : ST_NUMERICAL);
        segment = hit.t * c->prism.R;
        if (!fin(segment) || segment < 0) return finish_audit(a, &esc, power, ST_NUMERICAL);
        ks_add(&length, segment);
        if (!fin(length.value)) return finish_audit(a, &esc, power, ST_NUMERICAL);
        sp = split_flux(&ray, v_neg(pr_normal(hit.face)), c->n_int, c->n_ext);
        if (!sp.valid) return finish_audit(a, &esc, power, ST_NUMERICAL);
        ++a.hits;
        if (sp.tir) ++a.tir;
        a.max_iface = mx(a.max_iface, fabs(sp.balance));
        if (sp.has_t) {
            em = emit_exit(emit, user, &a, &esc, c, &sp.trans, hit.pos);
            if (em != ST_EXHAUSTED) return finish_audit(a, &esc, power, em);
        }
        ray = sp.refl;
        p = hit.pos;
        cur = hit.face;
    }
    remaining = jones_power(&ray.j);
    if (!fin(remaining) || remaining < 0 || (!remaining && jones_nonzero(&ray.j)))
        return finish_audit(a, &esc, remaining, ST_NUMERICAL);
    return finish_audit(a, &esc, remaining,
                        remaining == 0 ? ST_EXHAUSTED : (remaining <= c->tail ? ST_TAIL : ST_LIMIT));
}
/* hex_trace_core.hpp:253-259 */
static ray_audit_t trace_sample(const trace_cfg_t* c, uint64_t id, emit_fn emit, void* user)
{
    entry_t e = sample_entry(c->prism, c->k, icpo_sample_uniform(c->seed, id, 0), icpo_sample_uniform(c->seed, id, 1),
                             icpo_sample_uniform(c->seed, id, 2));
    return trace_from_entry(c, id, e, emit, user);
}

/* ------------------------------------------------------------- binning */
typedef struct {
    const double* edges;
    v3 ki;
    frame_t fr;
    uint32_t nt, np;
} grid_t;
typedef struct { uint64_t index; double mu; int pole, valid, snapped; } bin_t;

/* phase_math.hpp:37-81: u row by binary search on the saved edges, phi column via atan2,
 * canonical half-open assignment within a 64-epsilon roundoff window. */
static bin_t phase_bin(const grid_t* g, v3 d)
{
    bin_t b;
    double x, y, z, n, mu, s, u, phi, v, index, nearest;
    uint32_t lo, hi, j;
    unsigned cand;
    memset(&b, 0, sizeof b);
    if (!g->edges || !g->nt || !g->np || !v_is_unit(d)) return b;
    x = v_dot(g->fr.e0, d);
    y = v_dot(g->fr.e1, d);
    z = v_dot(g->ki, d);
    n = sqrt(x * x + y * y + z * z);
    if (!(n > 0) || !fin(n) || fabs(n - 1) > 512 * ICPO_EPS) return b;
    mu = z / n;
    s = hypot(x, y) / n;
    b.mu = mu;
    if (s <= 256 * ICPO_EPS) { b.pole = mu >= 0 ? 1 : -1; b.valid = 1; return b; }
    u = mu >= 0 ? (0.5 * s * s) / (1 + mu) : 1 - (0.5 * s * s) / (1 - mu);
    if (!(u >= 0 && u <= 1)) return b;
    lo = 0;
    hi = g->nt;
    while (lo + 1 < hi) {
        uint32_t mid = lo + (hi - lo) / 2;
        if (u >= g->edges[mid]) lo = mid; else hi = mid;
    }
    for (cand = 0; cand < 2; ++cand) {
        uint32_t e = lo + cand;
        double width, tol;
        if (e == 0 || e >= g->nt) continue;
        width = fmin(g->edges[e] - g->edges[e - 1], g->edges[e + 1] - g->edges[e]);
        tol = fmin(64 * ICPO_EPS * fmax(fabs(u), fabs(g->edges[e])), 1e-7 * width);
        if (fabs(u - g->edges[e]) <= tol) { b.snapped = (u != g->edges[e]); lo = e; break; }
    }
    phi = atan2(y, x);
    if (phi >= ICPO_PI) phi -= 2 * ICPO_PI;
    v = (phi + ICPO_PI) / (2 * ICPO_PI);
    index = v * g->np;
    nearest = floor(index + 0.5);
    if (fabs(index - nearest) <= fmin(64 * ICPO_EPS * g->np, 1e-7)) {
        b.snapped = b.snapped || (index != nearest);
        index = nearest;
    }
    j = (uint32_t)index;
    if (j == g->np) j = 0;
    if (j >= g->np) return b;
    b.index = (uint64_t)lo * g->np + j;
    b.valid = 1;
    return b;
}

/* include/rainbow/phase_cdf_math.hpp:16-32: symmetric sin^2 edges with exact endpoints. */
int icpo_u_edges(uint32_t n, double* edges)
{
    uint32_t i;
    if (n == 0) return -1;
    edges[0] = 0;
    edges[n] = 1;
    for (i = 1; i < n; ++i) {
        uint32_t k = i < n - i ? i : n - i;
        double s = sin((0.5 * ICPO_PI) * (double)k / (double)n);
        edges[i] = i <= n / 2u ? s * s : 1.0 - s * s;
    }
    for (i = 0; i < n; ++i)
        if (!(edges[i + 1] > edges[i])) return -2;
    return 0;
}

/* hex_phase/src/phase_table.cpp:11-21: active Hamilton quaternion (w,x,y,z); columns body->ensemble. */
typedef struct { v3 x, y, z; } rot_t;
static v3 rot_apply(const rot_t* r, v3 p) { return v_add(v_add(v_mul(r->x, p.x), v_mul(r->y, p.y)), v_mul(r->z, p.z)); }
static v3 rot_inverse(const rot_t* r, v3 p)
{
    v3 o = {v_dot(r->x, p), v_dot(r->y, p), v_dot(r->z, p)};
    return o;
}
static int rot_valid(const rot_t* r)
{
    return v_is_unit(r->x) && v_is_unit(r->y) && v_is_unit(r->z) && fabs(v_dot(r->x, r->y)) <= 128 * ICPO_EPS &&
           v_maxabs(v_sub(v_cross(r->x, r->y), r->z)) <= 256 * ICPO_EPS;
}
int icpo_rotation_from_quaternion(double w, double x, double y, double z, double out[9])
{
    double n = w * w + x * x + y * y + z * z, k;
    rot_t r;
    if (!fin(n) || fabs(n - 1) > 2e-12) return -1;
    k = 1 / sqrt(n);
    w *= k; x *= k; y *= k; z *= k;
    r.x.x = 1 - 2 * (y * y + z * z); r.x.y = 2 * (x * y + w * z); r.x.z = 2 * (x * z - w * y);
    r.y.x = 2 * (x * y - w * z); r.y.y = 1 - 2 * (x * x + z * z); r.y.z = 2 * (y * z + w * x);
    r.z.x = 2 * (x * z + w * y); r.z.y = 2 * (y * z - w * x); r.z.z = 1 - 2 * (x * x + y * y);
    if (!rot_valid(&r)) return -2;
    /* column-major: out[0..2] = x column, out[3..5] = y column, out[6..8] = z column */
    out[0] = r.x.x; out[1] = r.x.y; out[2] = r.x.z;
    out[3] = r.y.x; out[4] = r.y.y; out[5] = r.y.z;
    out[6] = r.z.x; out[7] = r.z.y; out[8] = r.z.z;
    return 0;
}

/* math.hpp:61-69 exported for host-side frame conventions (ki must already be unit). */
int icpo_make_frame(const double k_in[3], double k_out[3], double e0[3], double e1[3])
{
    v3 k = {k_in[0], k_in[1], k_in[2]}, kn;
    frame_t f;
    if (!v_normalize(k, &kn)) return -1;
    if (!make_frame(kn, &f)) return -2;
    k_out[0] = kn.x; k_out[1] = kn.y; k_out[2] = kn.z;
    e0[0] = f.e0.x; e0[1] = f.e0.y; e0[2] = f.e0.z;
    e1[0] = f.e1.x; e1[1] = f.e1.y; e1[2] = f.e1.z;
    return 0;
}

/* ---------------------------------------------------- mass histogram */
/* Accumulator state (phase_table.cpp:39-62); cells are Kahan pairs (value, correction). */
typedef struct {
    grid_t grid;
    ksum* cells;
    ksum point_mass, point_axial, forward, backward;
    uint64_t count, snapped;
    int error;
    rot_t rot;
    double scale;
} hist_t;

static void hist_emit(void* user, v3 d, double power)
{
    hist_t* h = (hist_t*)user;
    double w = h->scale * power;
    bin_t b;
    if (h->error) return;
    if (!(power > 0) || !fin(power) || !(w > 0) || !fin(w)) { h->error = 1; return; }
    b = phase_bin(&h->grid, rot_apply(&h->rot, d));
    if (!b.valid) { h->error = 2; return; }
    ++h->count;
    h->snapped += b.snapped;
    ks_add(&h->point_mass, w);
    ks_add(&h->point_axial, w * b.mu);
    if (b.pole > 0) ks_add(&h->forward, w);
    else if (b.pole < 0) ks_add(&h->backward, w);
    else ks_add(&h->cells[b.index], w);
}

/*
 * Public hex entry: trace rays [first, first+count) of one orientation node and
 * add their exits to an existing Kahan histogram (cells: 2*nt*np doubles).
 *
 * node[] layout (doubles): R, L, n_ext, n_int, tail, normalised orientation weight.
 *   The body-frame incident direction is the grid axis under the inverse rotation and the
 *   per-ray area weight is weight * Aproj / samples (generate_hex_phase.cpp:101-102).
 * grid_frame[] layout: ki(3), e0(3), e1(3) of the ensemble grid.
 * rot[] column-major body->ensemble rotation (9).
 * stats[] (inout, doubles): point_mass(v,c), point_axial(v,c), forward(v,c), backward(v,c),
 *   escaped_sum, unresolved_sum, max_balance, max_iface, [14..]=batch escaped kahan value/corr,...
 * counts[] (inout, uint64): samples, snapped, outputs, rays, status[8]
 * Audits follow the reference CLI: per batch of batch_size rays a Kahan summary
 * (hex_trace/src/hex_trace.cpp:72-88) is merged with plain adds (:89-100).
 */
static rot_t rot_from(const double* r9)
{
    rot_t r;
    r.x.x = r9[0]; r.x.y = r9[1]; r.x.z = r9[2];
    r.y.x = r9[3]; r.y.y = r9[4]; r.y.z = r9[5];
    r.z.x = r9[6]; r.z.y = r9[7]; r.z.z = r9[8];
    return r;
}
/* node_trace_settings + node_area (hex_phase/src/phase_generate.cpp:240-249, hex_trace.cpp:16-24):
 * the grid axis rotated into the body frame, normalised, its frame and projected area. */
static int node_setup(double R, double L, const double* r9, const double* grid_ki, v3* k, frame_t* kf, double* area)
{
    rot_t r = rot_from(r9);
    v3 gk = {grid_ki[0], grid_ki[1], grid_ki[2]};
    prism_t p = {R, L};
    if (!v_normalize(rot_inverse(&r, gk), k) || !make_frame(*k, kf)) return -1;
    *area = pr_projected(p, *k);
    return 0;
}
double icpo_hex_node_area(double R, double L, const double* r9, const double* grid_ki)
{
    v3 k;
    frame_t kf;
    double a;
    if (node_setup(R, L, r9, grid_ki, &k, &kf, &a)) return -1;
    return a;
}
int icpo_hex_accumulate(const double* node, uint64_t seed, uint64_t total, uint32_t max_hits,
                        const double* edges, uint32_t nt, uint32_t np, const double* grid_frame,
                        const double* rot, uint64_t first, uint64_t count, uint64_t batch_size,
                        double* cells, double* stats, uint64_t* counts, double balance_tol)
{
    trace_cfg_t c;
    hist_t h;
    double area;
    uint64_t i, b0;
    memset(&c, 0, sizeof c);
    memset(&h, 0, sizeof h);
    c.prism.R = node[0];
    c.prism.L = node[1];
    if (node_setup(node[0], node[1], rot, grid_frame, &c.k, &c.kf, &area)) return -1;
    c.n_ext = node[2];
    c.n_int = node[3];
    c.tail = node[4];
    c.seed = seed;
    c.total = total;
    c.max_hits = max_hits;
    if (!cfg_valid(&c)) return -2;
    h.grid.edges = edges;
    h.grid.nt = nt;
    h.grid.np = np;
    h.grid.ki.x = grid_frame[0]; h.grid.ki.y = grid_frame[1]; h.grid.ki.z = grid_frame[2];
    h.grid.fr.e0.x = grid_frame[3]; h.grid.fr.e0.y = grid_frame[4]; h.grid.fr.e0.z = grid_frame[5];
    h.grid.fr.e1.x = grid_frame[6]; h.grid.fr.e1.y = grid_frame[7]; h.grid.fr.e1.z = grid_frame[8];
    h.rot = rot_from(rot);
    h.scale = node[5] * area / (double)total;
    h.cells = (ksum*)cells;
    h.point_mass.value = stats[0]; h.point_mass.correction = stats[1];
    h.point_axial.value = stats[2]; h.point_axial.correction = stats[3];
    h.forward.value = stats[4]; h.forward.correction = stats[5];
    h.backward.value = stats[6]; h.backward.correction = stats[7];
    h.count = counts[0];
    h.snapped = counts[1];
    if (first + count > total || batch_size == 0) return -3;
    for (b0 = first; b0 < first + count; b0 += batch_size) {
        uint64_t b1 = b0 + batch_size < first + count ? b0 + batch_size : first + count;
        ksum esc = {0, 0}, tail = {0, 0};
        double maxbal = 0, maxif = 0;
        int accepted = 1;
        for (i = b0; i < b1; ++i) {
            ray_audit_t a = trace_sample(&c, i, hist_emit, &h);
            if (h.error) return -10 - h.error;
            counts[2] += a.outputs;
            counts[3] += 1;
            if ((unsigned)a.status < 8) counts[4 + a.status] += 1;
            ks_add(&esc, a.escaped);
            ks_add(&tail, a.unresolved);
            maxbal = mx(maxbal, fabs(a.balance));
            maxif = mx(maxif, a.max_iface);
            accepted = accepted && (a.status == ST_EXHAUSTED || a.status == ST_TAIL) && fin(a.escaped) &&
                       fin(a.unresolved) && a.escaped >= 0 && a.unresolved >= 0 && fin(a.balance) &&
                       fabs(a.balance) <= balance_tol && fin(a.max_iface) && a.max_iface >= 0 &&
                       a.max_iface <= balance_tol;
        }
        /* record_batch_audit: scale * batch sum, Kahan over batches (phase_generate.cpp:258-263) */
        {
            ksum ea = {stats[14], stats[15]}, ua = {stats[16], stats[17]};
            ks_add(&ea, h.scale * esc.value);
            ks_add(&ua, h.scale * tail.value);
            stats[14] = ea.value; stats[15] = ea.correction;
            stats[16] = ua.value; stats[17] = ua.correction;
        }
        stats[8] += esc.value;
        stats[9] += tail.value;
        stats[10] = mx(stats[10], maxbal);
        stats[11] = mx(stats[11], maxif);
        if (!accepted) counts[12] += 1;
    }
    stats[0] = h.point_mass.value; stats[1] = h.point_mass.correction;
    stats[2] = h.point_axial.value; stats[3] = h.point_axial.correction;
    stats[4] = h.forward.value; stats[5] = h.forward.correction;
    stats[6] = h.backward.value; stats[7] = h.backward.correction;
    counts[0] = h.count;
    counts[1] = h.snapped;
    return 0;
}

/*
 * Per-ray dump for kernel-level parity: for each ray, its status, outputs, escaped and
 * unresolved power, and the first max_out exits (body-frame direction + power).
 */
typedef struct { double* out; uint32_t cap, n; } dump_t;
static void dump_emit(void* user, v3 d, double power)
{
    dump_t* q = (dump_t*)user;
    if (q->n < q->cap) {
        q->out[4 * q->n + 0] = d.x;
        q->out[4 * q->n + 1] = d.y;
        q->out[4 * q->n + 2] = d.z;
        q->out[4 * q->n + 3] = power;
    }
    q->n++;
}
int icpo_hex_trace_rays(const double* node, uint64_t seed, uint64_t total, uint32_t max_hits, uint64_t first,
                        uint64_t count, uint32_t max_out, double* ray_info, double* exits)
{
    trace_cfg_t c;
    v3 kin;
    uint64_t i;
    memset(&c, 0, sizeof c);
    c.prism.R = node[0];
    c.prism.L = node[1];
    kin.x = node[2]; kin.y = node[3]; kin.z = node[4];
    if (!v_normalize(kin, &c.k) || !make_frame(c.k, &c.kf)) return -1;
    c.n_ext = node[5];
    c.n_int = node[6];
    c.tail = node[7];
    c.seed = seed;
    c.total = total;
    c.max_hits = max_hits;
    for (i = 0; i < count; ++i) {
        dump_t q;
        ray_audit_t a;
        q.out = exits + (size_t)i * max_out * 4;
        q.cap = max_out;
        q.n = 0;
        a = trace_sample(&c, first + i, dump_emit, &q);
        ray_info[6 * i + 0] = a.status;
        ray_info[6 * i + 1] = (double)a.outputs;
        ray_info[6 * i + 2] = a.escaped;
        ray_info[6 * i + 3] = a.unresolved;
        ray_info[6 * i + 4] = a.hits;
        ray_info[6 * i + 5] = a.max_iface;
    }
    return 0;
}

/*
 * Deterministic atlas node (hex_atlas/src/atlas.cpp:140-153, atlas::trace_cpu): every quadrature
 * ray traced from its given entry (trace_from_entry), its exits binned into a per-ray Kahan
 * histogram by the atlas mass sink (hex_atlas/include/ice_crystal/atlas.hpp:51-72: weight x power
 * per exit; an exit on a pole adds weight x power / np to every cell of the end row), then each
 * touched cell of the ray added to the node's Kahan histogram, in ray order.
 *
 * k3, e03, e13: the trace direction and its frame (also the binning frame).  rays[5n]: face,
 * x, y, z (units of the circumradius), weight (mm^2).  cells[nt*np] (out), stats[8] (out):
 * escaped_mm2, unresolved_mm2 (weight x per-ray sums, Kahan in ray order), rays, outputs,
 * max |balance|, max interface balance, first rejected ray (-1 none), its status.
 * Returns 0, -1 invalid setup, -2 out of memory.
 */
int icpo_atlas_node(double R, double L, double n_ext, double n_int, double tail, uint32_t max_hits, const double* k3,
                    const double* e03, const double* e13, const double* rays, uint64_t n, const double* edges,
                    uint32_t nt, uint32_t np, double balance_tol, double* cells, double* stats);

typedef struct {
    grid_t grid;
    ksum* ray_cells;
    unsigned char* touched;
    uint64_t* list;
    uint64_t listed;
    double weight;
    int error;
} atlas_sink_t;

static void atlas_add(atlas_sink_t* s, uint64_t cell, double w)
{
    if (!s->touched[cell]) {
        s->touched[cell] = 1;
        s->list[s->listed++] = cell;
    }
    ks_add(&s->ray_cells[cell], w);
}
static void atlas_emit(void* user, v3 d, double power)
{
    atlas_sink_t* s = (atlas_sink_t*)user;
    double w = s->weight * power;
    bin_t b;
    uint32_t row, j;
    if (s->error) return;
    if (!(w > 0) || !fin(w)) { s->error = 1; return; }
    b = phase_bin(&s->grid, d);
    if (!b.valid) { s->error = 2; return; }
    if (!b.pole) { atlas_add(s, b.index, w); return; }
    row = b.pole > 0 ? 0 : s->grid.nt - 1;
    for (j = 0; j < s->grid.np; ++j) atlas_add(s, (uint64_t)row * s->grid.np + j, w / s->grid.np);
}
int icpo_atlas_node(double R, double L, double n_ext, double n_int, double tail, uint32_t max_hits, const double* k3,
                    const double* e03, const double* e13, const double* rays, uint64_t n, const double* edges,
                    uint32_t nt, uint32_t np, double balance_tol, double* cells, double* stats)
{
    trace_cfg_t c;
    atlas_sink_t s;
    ksum* acc;
    ksum esc = {0, 0}, unres = {0, 0};
    uint64_t r, q, C = (uint64_t)nt * np;
    memset(&c, 0, sizeof c);
    memset(&s, 0, sizeof s);
    c.prism.R = R;
    c.prism.L = L;
    c.k.x = k3[0]; c.k.y = k3[1]; c.k.z = k3[2];
    c.kf.e0.x = e03[0]; c.kf.e0.y = e03[1]; c.kf.e0.z = e03[2];
    c.kf.e1.x = e13[0]; c.kf.e1.y = e13[1]; c.kf.e1.z = e13[2];
    c.n_ext = n_ext;
    c.n_int = n_int;
    c.tail = tail;
    c.total = n;
    c.max_hits = max_hits;
    if (!cfg_valid(&c) || !n || !nt || !np) return -1;
    s.grid.edges = edges;
    s.grid.ki = c.k;
    s.grid.fr = c.kf;
    s.grid.nt = nt;
    s.grid.np = np;
    acc = (ksum*)calloc(C, sizeof(ksum));
    s.ray_cells = (ksum*)calloc(C, sizeof(ksum));
    s.touched = (unsigned char*)calloc(C, 1);
    s.list = (uint64_t*)malloc(C * sizeof(uint64_t));
    if (!acc || !s.ray_cells || !s.touched || !s.list) {
        free(acc); free(s.ray_cells); free(s.touched); free(s.list);
        return -2;
    }
    stats[2] = (double)n;
    stats[3] = 0;
    stats[4] = stats[5] = 0;
    stats[6] = -1;
    stats[7] = 0;
    for (r = 0; r < n; ++r) {
        entry_t e;
        ray_audit_t a;
        const double* q5 = rays + 5 * r;
        e.face = (unsigned)q5[0];
        e.pos.x = q5[1]; e.pos.y = q5[2]; e.pos.z = q5[3];
        e.valid = 1;
        s.weight = q5[4];
        s.listed = 0;
        s.error = 0;
        a = trace_from_entry(&c, r, e, atlas_emit, &s);
        if (s.error) a.status = ST_OVERFLOW;
        stats[3] += (double)a.outputs;
        stats[4] = mx(stats[4], fabs(a.balance));
        stats[5] = mx(stats[5], a.max_iface);
        if (stats[6] < 0 && !((a.status == ST_EXHAUSTED || a.status == ST_TAIL) && fin(a.max_iface) &&
                              a.max_iface <= balance_tol && fabs(a.balance) <= balance_tol)) {
            stats[6] = (double)r;
            stats[7] = (double)a.status;
        }
        ks_add(&esc, s.weight * a.escaped);
        ks_add(&unres, s.weight * a.unresolved);
        for (q = 0; q < s.listed; ++q) {
            const uint64_t cell = s.list[q];
            if (s.ray_cells[cell].value > 0) ks_add(&acc[cell], s.ray_cells[cell].value);
            s.ray_cells[cell].value = 0;
            s.ray_cells[cell].correction = 0;
            s.touched[cell] = 0;
        }
    }
    for (q = 0; q < C; ++q) cells[q] = acc[q].value;
    stats[0] = esc.value;
    stats[1] = unres.value;
    free(acc); free(s.ray_cells); free(s.touched); free(s.list);
    return 0;
}

/* PhaseMassAccumulator::masses (phase_table.cpp:63-76): pole mass spread uniformly
 * over the first / last row, added into the Kahan pair of each cell. */
int icpo_masses(const double* cells, uint32_t nt, uint32_t np, const double* stats, double* out)
{
    double f = stats[4] / np, b = stats[6] / np;
    size_t k, n = (size_t)nt * np;
    if ((stats[4] > 0 && !(f > 0)) || (stats[6] > 0 && !(b > 0))) return -1;
    for (k = 0; k < n; ++k) {
        ksum s = {cells[2 * k], cells[2 * k + 1]};
        size_t i = k / np;
        if (i == 0) ks_add(&s, f);
        if (i + 1 == nt) ks_add(&s, b);
        out[k] = s.value;
    }
    return 0;
}

/* measure_mass (phase_table.cpp:79-93) */
int icpo_measure_mass(const double* edges, uint32_t nt, uint32_t np, const double* mass, double out[2])
{
    ksum total = {0, 0}, axial = {0, 0};
    size_t k, n = (size_t)nt * np;
    for (k = 0; k < n; ++k) {
        double w = mass[k];
        size_t i = k / np;
        if (!fin(w) || w < 0) return -1;
        ks_add(&total, w);
        ks_add(&axial, w * (1 - edges[i] - edges[i + 1]));
    }
    if (!(total.value > 0) || !fin(total.value) || !fin(axial.value)) return -2;
    out[0] = total.value;
    out[1] = axial.value;
    return 0;
}

/*
 * build_host_cdf (phase_table.cpp:111-187): conservative aggregation of a fine
 * (nt x np) mass grid into (ct x cp), ordered binary64 column scans, ordered
 * marginal scan, normalisation with u-edge fallback for empty columns, audits.
 * report[]: g_source, g_stored, coarsening_tv, cdf_mass, l1, lost_mass,
 *           max_cell_error, aggregation_relative_error, lost_cells.
 * Returns 0, or a negative code for the reference's exception sites.
 */
int icpo_build_cdf(const double* edges, uint32_t nt, uint32_t np, const double* mass, uint32_t ct, uint32_t cp,
                   double max_l1, double max_lost, double max_tv, double* phi, double* theta, double* cedges,
                   double* report)
{
    double fine[2], stored[2], largest, total;
    ksum* sums;
    double* coarse;
    double* columns;
    uint32_t dt, dp, i, j;
    ksum tv = {0, 0}, l1 = {0, 0}, lost = {0, 0}, recovered = {0, 0}, axial = {0, 0};
    size_t k;
    int rc = 0;
    if (!fin(max_l1) || max_l1 < 0 || max_l1 > 2 || !fin(max_lost) || max_lost < 0 || max_lost > 1 ||
        !fin(max_tv) || max_tv < 0 || max_tv > 1)
        return -1;
    if (icpo_measure_mass(edges, nt, np, mass, fine)) return -2;
    if (!ct || !cp || ct > nt || cp > np || nt % ct || np % cp) return -3;
    dt = nt / ct;
    dp = np / cp;
    for (i = 0; i <= ct; ++i) cedges[i] = edges[(size_t)i * dt];
    sums = (ksum*)calloc((size_t)ct * cp, sizeof(ksum));
    coarse = (double*)malloc(sizeof(double) * (size_t)ct * cp);
    columns = (double*)malloc(sizeof(double) * cp);
    if (!sums || !coarse || !columns) { rc = -4; goto done; }
    for (i = 0; i < nt; ++i)
        for (j = 0; j < np; ++j) ks_add(&sums[(size_t)(i / dt) * cp + j / dp], mass[(size_t)i * np + j]);
    for (k = 0; k < (size_t)ct * cp; ++k) coarse[k] = sums[k].value;
    if (icpo_measure_mass(cedges, ct, cp, coarse, stored)) { rc = -2; goto done; }
    report[0] = fine[1] / fine[0];
    report[7] = fabs(stored[0] / fine[0] - 1);
    for (i = 0; i < nt; ++i)
        for (j = 0; j < np; ++j) {
            uint32_t ci = i / dt, cj = j / dp;
            double fraction = (edges[i + 1] - edges[i]) / (cedges[ci + 1] - cedges[ci]) / dp;
            ks_add(&tv, fabs(mass[(size_t)i * np + j] / fine[0] - coarse[(size_t)ci * cp + cj] / stored[0] * fraction));
        }
    report[2] = 0.5 * tv.value;
    if (!fin(report[2]) || report[2] > max_tv || report[7] > 1e-12) { rc = -5; goto done; }
    largest = coarse[0];
    for (k = 1; k < (size_t)ct * cp; ++k)
        if (coarse[k] > largest) largest = coarse[k];
    phi[0] = 0;
    for (j = 0; j < cp; ++j) {
        size_t base = (size_t)j * (ct + 1);
        double s = 0;
        theta[base] = 0;
        for (i = 0; i < ct; ++i) {
            double w = coarse[(size_t)i * cp + j] / largest;
            if (coarse[(size_t)i * cp + j] > 0 && !(w > 0)) { rc = -6; goto done; }
            s += w;
            theta[base + i + 1] = s;
        }
        columns[j] = s;
        phi[j + 1] = phi[j] + s;
    }
    total = phi[cp];
    if (!(total > 0) || !fin(total)) { rc = -7; goto done; }
    for (j = 0; j < cp; ++j) {
        size_t base = (size_t)j * (ct + 1);
        for (i = 1; i < ct; ++i) theta[base + i] = columns[j] > 0 ? theta[base + i] / columns[j] : cedges[i];
        theta[base + ct] = 1;
    }
    for (j = 1; j < cp; ++j) phi[j] /= total;
    phi[cp] = 1;
    report[6] = 0;
    report[8] = 0;
    for (j = 0; j < cp; ++j)
        for (i = 0; i < ct; ++i) {
            size_t base = (size_t)j * (ct + 1) + i;
            double q = (phi[j + 1] - phi[j]) * (theta[base + 1] - theta[base]);
            double p = coarse[(size_t)i * cp + j] / stored[0], err;
            if (!fin(q) || q < 0 || phi[j + 1] < phi[j] || theta[base + 1] < theta[base]) { rc = -8; goto done; }
            if (coarse[(size_t)i * cp + j] > 0 && !(p > 0)) { rc = -9; goto done; }
            err = fabs(p - q);
            ks_add(&l1, err);
            if (err > report[6]) report[6] = err;
            if (p > 0 && q == 0) { ks_add(&lost, p); report[8] += 1; }
            ks_add(&recovered, q);
            ks_add(&axial, q * (1 - cedges[i] - cedges[i + 1]));
        }
    report[4] = l1.value;
    report[5] = lost.value;
    report[3] = recovered.value;
    report[1] = axial.value / recovered.value;
    if (report[4] > max_l1 || report[5] > max_lost || fabs(report[3] - 1) > 1e-10 || !fin(report[1]) ||
        !(report[1] > -1 && report[1] < 1))
        rc = -10;
done:
    free(sums);
    free(coarse);
    free(columns);
    return rc;
}

/* ============================================================ water drops */
/*
 * Axisymmetric drop in units of its equal-volume radius a: r/a = 1 + sum_n c_n T_n(mu),
 * mu = -p.y/|p| (include/rainbow/raindrop_shape.hpp:70-100).  The ray chain is the prism's
 * linear R/T chain (hex_trace_core.hpp:190-252) with the drop surface as the boundary; its
 * first four exits are RaindropPathTracer::trace_impl's families R, TT, TRT, TRRT
 * (include/rainbow/raindrop_paths.hpp:41-107).  The reference intersects with an interval
 * bracket stack plus safeguarded Newton (raindrop_intersection.hpp:203-382); this oracle
 * brackets the same root by sampling the chord of the bounding sphere (a golden-section
 * minimum of the convex gauge |p|/R(mu) decides near-silhouette lines) and polishes it with
 * bracketed Newton.  Rays start on a disk of radius `disk` perpendicular to k, `back` before
 * the centre, drawn with the counter RNG (math.hpp:136-146) in place of the reference's
 * deterministic vertex lattice (raindrop_paths.hpp:52-58).
 *
 * drop[] layout (doubles): c[0..7], r_center, r_out, r_in, sphere, disk, back, n_ext, n_int,
 *   tail, scale (mm^2 per unit exit power), radius_mm.
 * frame9[]: k(3), e0(3), e1(3) -- the incident direction and the sampling / grid frame.
 */
typedef struct {
    double c[8];
    double r_center, r_out, r_in, disk, back;
    int sphere;
} drop_t;

typedef struct {
    drop_t shape;
    v3 k;
    frame_t kf;
    double n_ext, n_int, tail, scale, radius_mm;
    uint64_t seed, total;
    uint32_t max_hits;
} drop_cfg_t;

#define DR_SAMPLES 24

static double dr_radius(const drop_t* s, double mu, double* deriv)
{
    double prev = 1, cur = mu, dprev = 0, dcur = 1, r = 1 + s->c[0] + s->c[1] * mu, d = s->c[1];
    int n;
    for (n = 2; n < 8; ++n) {
        double next = 2 * mu * cur - prev, dnext = 2 * cur + 2 * mu * dcur - dprev;
        r += s->c[n] * next;
        d += s->c[n] * dnext;
        prev = cur;
        cur = next;
        dprev = dcur;
        dcur = dnext;
    }
    *deriv = d;
    return r;
}
/* outward unit normal: gradient of |p| - R(mu) (raindrop_shape.hpp:92-100) */
static int dr_normal(const drop_t* s, v3 p, v3* n)
{
    double r = sqrt(v_dot(p, p)), dR;
    v3 u, g, down = {0, -1, 0};
    if (!(r > 0) || !fin(r)) return 0;
    u = v_div(p, r);
    if (s->sphere) return v_normalize(u, n);
    dr_radius(s, -u.y, &dR);
    g = v_sub(u, v_mul(v_sub(down, v_mul(u, -u.y)), dR / r));
    return v_normalize(g, n);
}
/* f(t) = |o + t d| - R(mu) and df/dt; deep inside only its sign matters (raindrop_shape.hpp:86-91) */
static double dr_f(const drop_t* s, v3 o, v3 d, double t, double* df)
{
    v3 p = v_add(o, v_mul(d, t));
    double r = sqrt(v_dot(p, p)), mu, dR, R, rd, dmu;
    if (r < 0.25 * s->r_in) {
        *df = r > 0 ? v_dot(p, d) / r : 0;
        return r - s->r_in;
    }
    rd = v_dot(p, d) / r;
    mu = -p.y / r;
    R = dr_radius(s, mu, &dR);
    dmu = (-d.y - mu * rd) / r;
    *df = rd - dR * dmu;
    return r - R;
}
static double dr_gauge(const drop_t* s, v3 o, v3 d, double t)
{
    v3 p = v_add(o, v_mul(d, t));
    double r = sqrt(v_dot(p, p)), dR;
    if (!(r > 0)) return 0;
    return r / dr_radius(s, -p.y / r, &dR);
}
/* minimum of the convex gauge on [a, b] by golden-section search */
static double dr_gauge_min(const drop_t* s, v3 o, v3 d, double a, double b)
{
    const double g = 0.6180339887498949;
    double x1 = b - g * (b - a), x2 = a + g * (b - a);
    double f1 = dr_gauge(s, o, d, x1), f2 = dr_gauge(s, o, d, x2);
    int it;
    for (it = 0; it < 200 && b - a > 4 * ICPO_EPS * mx(1, fabs(a)); ++it) {
        if (f1 <= f2) {
            b = x2; x2 = x1; f2 = f1;
            x1 = b - g * (b - a);
            f1 = dr_gauge(s, o, d, x1);
        } else {
            a = x1; x1 = x2; f1 = f2;
            x2 = a + g * (b - a);
            f2 = dr_gauge(s, o, d, x2);
        }
    }
    return f1 <= f2 ? x1 : x2;
}
/* bracketed Newton on [a, b], f(a) and f(b) of opposite signs (bisection when Newton leaves it) */
static double dr_refine(const drop_t* s, v3 o, v3 d, double a, double fa, double b)
{
    double t = 0.5 * (a + b);
    int it;
    for (it = 0; it < 300; ++it) {
        double df, f = dr_f(s, o, d, t, &df), tn, lo, hi;
        if (f == 0) return t;
        if ((f < 0) == (fa < 0)) { a = t; fa = f; }
        else b = t;
        lo = a < b ? a : b;
        hi = a < b ? b : a;
        tn = t - f / df;
        if (!(tn > lo && tn < hi)) tn = 0.5 * (lo + hi);
        if (fabs(tn - t) <= 2 * ICPO_EPS * mx(1, fabs(t)) || hi - lo <= 4 * ICPO_EPS * mx(1, fabs(t))) return tn;
        t = tn;
    }
    return t;
}
static int dr_sphere_roots(v3 p, v3 d, double rad, double* t0, double* t1)
{
    double b = v_dot(p, d), c = v_dot(p, p) - rad * rad, disc = b * b - c, q;
    if (!(disc >= 0)) return 0;
    q = sqrt(disc);
    *t0 = -b - q;
    *t1 = -b + q;
    return 1;
}
/* first surface point along an exterior line; 0 on a miss */
static int dr_entry(const drop_t* s, v3 o, v3 d, double* t)
{
    double t0, t1, prev, fprev, df, tm;
    int i;
    if (s->sphere) {
        if (!dr_sphere_roots(o, d, s->r_center, &t0, &t1) || t0 < 0) return 0;
        *t = t0;
        return 1;
    }
    if (!dr_sphere_roots(o, d, s->r_out, &t0, &t1)) return 0;
    if (t0 < 0) t0 = 0;
    prev = t0;
    fprev = dr_f(s, o, d, prev, &df);
    for (i = 1; i <= DR_SAMPLES; ++i) {
        double ti = t0 + (t1 - t0) * i / DR_SAMPLES, fi = dr_f(s, o, d, ti, &df);
        if (fi < 0) { *t = dr_refine(s, o, d, prev, fprev, ti); return 1; }
        prev = ti;
        fprev = fi;
    }
    tm = dr_gauge_min(s, o, d, t0, t1);
    if (!(dr_gauge(s, o, d, tm) < 1)) return 0;
    *t = dr_refine(s, o, d, t0, dr_f(s, o, d, t0, &df), tm);
    return 1;
}
/* far end of an interior chord that starts on the surface at p */
static double dr_exit(const drop_t* s, v3 p, v3 d)
{
    double t0, t1, df, tm, prev;
    int i;
    if (s->sphere) {
        if (!dr_sphere_roots(p, d, s->r_center, &t0, &t1)) return 0;
        return t1 > 0 ? t1 : 0;
    }
    if (!dr_sphere_roots(p, d, s->r_out, &t0, &t1) || !(t1 > 0)) return 0;
    prev = t1;
    for (i = DR_SAMPLES - 1; i >= 1; --i) {
        double ti = t1 * i / DR_SAMPLES, fi = dr_f(s, p, d, ti, &df);
        if (fi < 0) return dr_refine(s, p, d, prev, dr_f(s, p, d, prev, &df), ti);
        prev = ti;
    }
    tm = dr_gauge_min(s, p, d, 0, t1);
    if (!(dr_gauge(s, p, d, tm) < 1)) return 0;
    return dr_refine(s, p, d, t1, dr_f(s, p, d, t1, &df), tm);
}

typedef void (*drop_emit_fn)(void* user, v3 d, double power, uint32_t hit);

static int drop_emit(drop_emit_fn emit, void* user, ray_audit_t* a, ksum* esc, const drop_cfg_t* c,
                     const fray_t* ray, v3 pos, uint32_t hit)
{
    double power = jones_power(&ray->j);
    if (!fin(power) || power < 0 || (!power && jones_nonzero(&ray->j))) return ST_NUMERICAL;
    if (power == 0) return ST_EXHAUSTED;
    if (!v_fin(v_mul(pos, c->radius_mm))) return ST_NUMERICAL;
    if (emit) emit(user, ray->d, power, hit);
    ks_add(esc, power);
    ++a->outputs;
    return ST_EXHAUSTED;
}
/* chain from the entry point pos of a ray travelling along k (frame kf) */
static ray_audit_t drop_from_entry(const drop_cfg_t* c, v3 pos, v3 k, frame_t kf, drop_emit_fn emit, void* user)
{
    ray_audit_t a;
    ksum esc = {0, 0};
    fray_t inc, ray;
    branches_t sp;
    v3 p, n;
    unsigned encounter;
    int em;
    double remaining;
    memset(&a, 0, sizeof a);
    if (!dr_normal(&c->shape, pos, &n)) return finish_audit(a, &esc, 1, ST_NUMERICAL);
    inc.d = k;
    inc.fr = kf;
    inc.j = jones_identity();
    sp = split_flux_graze(&inc, n, c->n_ext, c->n_int, 1);
    if (!sp.valid) return finish_audit(a, &esc, 1, ST_NUMERICAL);
    a.max_iface = fabs(sp.balance);
    em = drop_emit(emit, user, &a, &esc, c, &sp.refl, pos, 0);
    if (em != ST_EXHAUSTED) return finish_audit(a, &esc, 1, em);
    if (!sp.has_t) { a.tir = 1; return finish_audit(a, &esc, 0, ST_EXHAUSTED); }
    ray = sp.trans;
    p = pos;
    for (encounter = 0; encounter < c->max_hits; ++encounter) {
        double power = jones_power(&ray.j), t;
        if (!fin(power) || power < 0 || (!power && jones_nonzero(&ray.j))) return finish_audit(a, &esc, power, ST_NUMERICAL);
        if (power == 0) return finish_audit(a, &esc, 0, ST_EXHAUSTED);
        if (power <= c->tail) return finish_audit(a, &esc, power, ST_TAIL);
        t = dr_exit(&c->shape, p, ray.d);
        p = v_add(p, v_mul(ray.d, t));
        if (!fin(t) || !dr_normal(&c->shape, p, &n)) return finish_audit(a, &esc, power, ST_NUMERICAL);
        sp = split_flux_graze(&ray, v_neg(n), c->n_int, c->n_ext, 1);
        if (!sp.valid) return finish_audit(a, &esc, power, ST_NUMERICAL);
        ++a.hits;
        if (sp.tir) ++a.tir;
        a.max_iface = mx(a.max_iface, fabs(sp.balance));
        if (sp.has_t) {
            em = drop_emit(emit, user, &a, &esc, c, &sp.trans, p, a.hits);
            if (em != ST_EXHAUSTED) return finish_audit(a, &esc, power, em);
        }
        ray = sp.refl;
    }
    remaining = jones_power(&ray.j);
    if (!fin(remaining) || remaining < 0 || (!remaining && jones_nonzero(&ray.j)))
        return finish_audit(a, &esc, remaining, ST_NUMERICAL);
    return finish_audit(a, &esc, remaining,
                        remaining == 0 ? ST_EXHAUSTED : (remaining <= c->tail ? ST_TAIL : ST_LIMIT));
}
/* ray `id`: point on the sampling disk, entry along k; *missed = 1 when the line misses */
static ray_audit_t drop_sample(const drop_cfg_t* c, uint64_t id, drop_emit_fn emit, void* user, int* missed)
{
    ray_audit_t a;
    ksum none = {0, 0};
    double u0 = icpo_sample_uniform(c->seed, id, 0), u1 = icpo_sample_uniform(c->seed, id, 1);
    double rad = c->shape.disk * sqrt(u0), sn = sin(ICPO_PI * (2 * u1)), cs = cos(ICPO_PI * (2 * u1)), t;
    v3 o = v_sub(v_add(v_mul(c->kf.e0, rad * cs), v_mul(c->kf.e1, rad * sn)), v_mul(c->k, c->shape.back));
    *missed = 0;
    if (!dr_entry(&c->shape, o, c->k, &t)) {
        memset(&a, 0, sizeof a);
        *missed = 1;
        return finish_audit(a, &none, 0, ST_EXHAUSTED);
    }
    return drop_from_entry(c, v_add(o, v_mul(c->k, t)), c->k, c->kf, emit, user);
}
static int drop_setup(const double* drop, const double* frame9, uint64_t seed, uint64_t total, uint32_t max_hits,
                      drop_cfg_t* c)
{
    int i;
    memset(c, 0, sizeof *c);
    for (i = 0; i < 8; ++i) c->shape.c[i] = drop[i];
    c->shape.r_center = drop[8];
    c->shape.r_out = drop[9];
    c->shape.r_in = drop[10];
    c->shape.sphere = drop[11] != 0;
    c->shape.disk = drop[12];
    c->shape.back = drop[13];
    c->n_ext = drop[14];
    c->n_int = drop[15];
    c->tail = drop[16];
    c->scale = drop[17];
    c->radius_mm = drop[18];
    c->k.x = frame9[0]; c->k.y = frame9[1]; c->k.z = frame9[2];
    c->kf.e0.x = frame9[3]; c->kf.e0.y = frame9[4]; c->kf.e0.z = frame9[5];
    c->kf.e1.x = frame9[6]; c->kf.e1.y = frame9[7]; c->kf.e1.z = frame9[8];
    c->seed = seed;
    c->total = total;
    c->max_hits = max_hits;
    if (!frame_valid(c->kf, c->k) || !(c->n_ext > 0 && c->n_int > 0) || !(c->tail >= 0 && c->tail < 1) ||
        !max_hits || !(c->shape.r_out >= c->shape.r_center) || !(c->shape.r_in > 0) || !(c->shape.disk > 0))
        return -1;
    return 0;
}

static void drop_hist_emit(void* user, v3 d, double power, uint32_t hit)
{
    (void)hit;
    hist_emit(user, d, power);
}
/*
 * Traces rays [first, first+count) of a drop record into a Kahan histogram (cells: 2*nt*np).
 * stats[] (inout): point_mass(v,c), point_axial(v,c), forward(v,c), backward(v,c),
 *   escaped(v,c), unresolved(v,c), max_balance, max_iface  -- powers in units of one ray.
 * counts[] (inout): binned exits, snapped, outputs, rays, status[8], missed, encounters.
 */
int icpo_drop_accumulate(const double* drop, const double* frame9, uint64_t seed, uint64_t total, uint32_t max_hits,
                         const double* edges, uint32_t nt, uint32_t np, uint64_t first, uint64_t count,
                         double* cells, double* stats, uint64_t* counts)
{
    drop_cfg_t c;
    hist_t h;
    uint64_t i;
    ksum esc, unres;
    if (drop_setup(drop, frame9, seed, total, max_hits, &c)) return -1;
    if (first + count > total) return -3;
    memset(&h, 0, sizeof h);
    h.grid.edges = edges;
    h.grid.nt = nt;
    h.grid.np = np;
    h.grid.ki = c.k;
    h.grid.fr = c.kf;
    h.rot.x.x = 1; h.rot.y.y = 1; h.rot.z.z = 1;
    h.scale = c.scale;
    h.cells = (ksum*)cells;
    h.point_mass.value = stats[0]; h.point_mass.correction = stats[1];
    h.point_axial.value = stats[2]; h.point_axial.correction = stats[3];
    h.forward.value = stats[4]; h.forward.correction = stats[5];
    h.backward.value = stats[6]; h.backward.correction = stats[7];
    esc.value = stats[8]; esc.correction = stats[9];
    unres.value = stats[10]; unres.correction = stats[11];
    h.count = counts[0];
    h.snapped = counts[1];
    for (i = first; i < first + count; ++i) {
        int missed;
        ray_audit_t a = drop_sample(&c, i, drop_hist_emit, &h, &missed);
        if (h.error) return -10 - h.error;
        counts[3] += 1;
        if (missed) { counts[12] += 1; continue; }
        counts[2] += a.outputs;
        if ((unsigned)a.status < 8) counts[4 + a.status] += 1;
        counts[13] += a.hits;
        ks_add(&esc, a.escaped);
        ks_add(&unres, a.unresolved);
        stats[12] = mx(stats[12], fabs(a.balance));
        stats[13] = mx(stats[13], a.max_iface);
    }
    stats[0] = h.point_mass.value; stats[1] = h.point_mass.correction;
    stats[2] = h.point_axial.value; stats[3] = h.point_axial.correction;
    stats[4] = h.forward.value; stats[5] = h.forward.correction;
    stats[6] = h.backward.value; stats[7] = h.backward.correction;
    stats[8] = esc.value; stats[9] = esc.correction;
    stats[10] = unres.value; stats[11] = unres.correction;
    counts[0] = h.count;
    counts[1] = h.snapped;
    return 0;
}

/* per-ray dump: ray_info[8] = status, outputs, escaped, unresolved, hits, max_iface, missed, tir;
 * exits[5 per exit] = direction(3), power, interaction index (0 = entry reflection) */
typedef struct { double* out; uint32_t cap, n; } drop_dump_t;
static void drop_dump_emit(void* user, v3 d, double power, uint32_t hit)
{
    drop_dump_t* q = (drop_dump_t*)user;
    if (q->n < q->cap) {
        double* e = q->out + 5 * (size_t)q->n;
        e[0] = d.x; e[1] = d.y; e[2] = d.z; e[3] = power; e[4] = hit;
    }
    q->n++;
}
static void drop_info(double* info, ray_audit_t a, int missed)
{
    info[0] = a.status;
    info[1] = (double)a.outputs;
    info[2] = a.escaped;
    info[3] = a.unresolved;
    info[4] = a.hits;
    info[5] = a.max_iface;
    info[6] = missed;
    info[7] = a.tir;
}
int icpo_drop_trace_rays(const double* drop, const double* frame9, uint64_t seed, uint64_t total, uint32_t max_hits,
                         uint64_t first, uint64_t count, uint32_t max_out, double* ray_info, double* exits)
{
    drop_cfg_t c;
    uint64_t i;
    if (drop_setup(drop, frame9, seed, total, max_hits, &c)) return -1;
    for (i = 0; i < count; ++i) {
        drop_dump_t q;
        int missed;
        ray_audit_t a;
        q.out = exits + (size_t)i * max_out * 5;
        q.cap = max_out;
        q.n = 0;
        a = drop_sample(&c, first + i, drop_dump_emit, &q, &missed);
        drop_info(ray_info + 8 * i, a, missed);
    }
    return 0;
}
/* one ray from an exterior origin o along unit k with polarisation frame vector e0 */
int icpo_drop_trace_from(const double* drop, const double* o3, const double* k3, const double* e03, uint32_t max_hits,
                         uint32_t max_out, double* ray_info, double* exits)
{
    drop_cfg_t c;
    double frame9[9], t;
    v3 o = {o3[0], o3[1], o3[2]}, k = {k3[0], k3[1], k3[2]}, e0 = {e03[0], e03[1], e03[2]}, e1 = v_cross(k, e0);
    drop_dump_t q;
    ray_audit_t a;
    frame9[0] = k.x; frame9[1] = k.y; frame9[2] = k.z;
    frame9[3] = e0.x; frame9[4] = e0.y; frame9[5] = e0.z;
    frame9[6] = e1.x; frame9[7] = e1.y; frame9[8] = e1.z;
    if (drop_setup(drop, frame9, 0, 1, max_hits, &c)) return -1;
    q.out = exits;
    q.cap = max_out;
    q.n = 0;
    if (!dr_entry(&c.shape, o, k, &t)) {
        ksum none = {0, 0};
        memset(&a, 0, sizeof a);
        drop_info(ray_info, finish_audit(a, &none, 0, ST_EXHAUSTED), 1);
        return 0;
    }
    a = drop_from_entry(&c, v_add(o, v_mul(k, t)), k, c.kf, drop_dump_emit, &q);
    drop_info(ray_info, a, 0);
    return 0;
}
/* boundary query: entry from an exterior point (inside = 0) or chord exit from a surface
 * point (inside = 1); out[8] = hit, t, position(3), outward normal(3) */
int icpo_drop_intersect(const double* drop, const double* o3, const double* d3, int inside, double* out)
{
    drop_cfg_t c;
    static const double frame9[9] = {1, 0, 0, 0, 0, 1, 0, -1, 0};
    v3 o = {o3[0], o3[1], o3[2]}, d = {d3[0], d3[1], d3[2]}, p, n;
    double t = 0;
    int hit;
    if (drop_setup(drop, frame9, 0, 1, 1, &c)) return -1;
    if (inside) {
        t = dr_exit(&c.shape, o, d);
        hit = 1;
    } else {
        hit = dr_entry(&c.shape, o, d, &t);
    }
    memset(out, 0, 8 * sizeof(double));
    out[0] = hit;
    if (!hit) return 0;
    p = v_add(o, v_mul(d, t));
    if (!dr_normal(&c.shape, p, &n)) return -2;
    out[1] = t;
    out[2] = p.x; out[3] = p.y; out[4] = p.z;
    out[5] = n.x; out[6] = n.y; out[7] = n.z;
    return 0;
}
/* Incident frame of an inclination alpha: ki = (cos a, -sin a, 0) rounded to binary32 and
 * normalised there, e0 from the z helper axis (x when |k_z| >= 0.9) in binary32
 * (apps/generate_phase.cpp:209-217, include/rainbow/raindrop_settings.hpp:37-38,
 * include/rainbow/vec3.hpp:20-36, 60-65), then promoted and re-orthonormalised in binary64
 * (apps/generate_phase.cpp:242-245). */
static float f_dot(float ax, float ay, float az, float bx, float by, float bz)
{
    return fmaf(ax, bx, fmaf(ay, by, az * bz));
}
int icpo_drop_frame(double inclination_deg, double* k, double* e0, double* e1)
{
    double a = inclination_deg * ICPO_PI / 180.0, kd[3], ed[3], n, d;
    float kx = (float)cos(a), ky = (float)-sin(a), kz = 0.0f, len, hx, hz, w, ex, ey, ez;
    int i;
    len = sqrtf(f_dot(kx, ky, kz, kx, ky, kz));
    kx /= len; ky /= len; kz /= len;
    hx = fabsf(kz) < 0.9f ? 0.0f : 1.0f;
    hz = fabsf(kz) < 0.9f ? 1.0f : 0.0f;
    w = f_dot(kx, ky, kz, hx, 0.0f, hz);
    ex = hx - kx * w; ey = 0.0f - ky * w; ez = hz - kz * w;
    len = sqrtf(f_dot(ex, ey, ez, ex, ey, ez));
    ex /= len; ey /= len; ez /= len;
    kd[0] = kx; kd[1] = ky; kd[2] = kz;
    n = sqrt(kd[0] * kd[0] + kd[1] * kd[1] + kd[2] * kd[2]);
    if (!(n > 0)) return -1;
    for (i = 0; i < 3; ++i) kd[i] /= n;
    ed[0] = ex; ed[1] = ey; ed[2] = ez;
    d = ed[0] * kd[0] + ed[1] * kd[1] + ed[2] * kd[2];
    for (i = 0; i < 3; ++i) ed[i] -= d * kd[i];
    n = sqrt(ed[0] * ed[0] + ed[1] * ed[1] + ed[2] * ed[2]);
    if (!(n > 0)) return -1;
    for (i = 0; i < 3; ++i) { k[i] = kd[i]; e0[i] = ed[i] / n; }
    e1[0] = k[1] * e0[2] - k[2] * e0[1];
    e1[1] = k[2] * e0[0] - k[0] * e0[2];
    e1[2] = k[0] * e0[1] - k[1] * e0[0];
    return 0;
}

/* --------------------------------------------------- Table-II rainbow diffraction
 * Restates RainbowDiffraction (include/rainbow/rainbow_diffraction.hpp): the Table-II width
 * lookup (:16-28), the configuration check (:29-39), the transition labels of the edge below
 * each query direction (:40-56), the local spherical Gaussian (:57-139), the haversine
 * distance (:140-145) and the longitude window of a spherical cap (:166-174).  Binary64,
 * the reference's operation order and the same libm calls, so the results equal the header's
 * compiled on the same host bit for bit.  The focal records have the 144-byte layout of
 * rainbow::FocalOpticalResult (include/rainbow/wave_optics_data.hpp:27-40). */
typedef struct {
    double field[4];
    double s, p;
    double fam_inc[4];
    uint32_t fam_hits[4];
    uint32_t corrected, extra;
    uint32_t flags, first_problem;
    double field2[4];
} rb_focal;
typedef struct {
    double s, p, sigma, blend;
    uint32_t flags, kind;
} rb_result;
typedef struct {
    double s, c;
} rb_sum;

#define RB_TOL 0x1p-44 /* closed-cap cutoff slack (rainbow_diffraction.hpp:14) */
enum { RB_PRIMARY = 1, RB_SECONDARY = 2, RB_UNKNOWN = 4 };
enum { RB_FILTERED = 1, RB_UNDER = 2, RB_INPUT = 4, RB_STENCIL = 8, RB_DETECT = 16, RB_INVALID = 32 };

int icpo_rainbow_table_sigma(float radius, double* out)
{
    static const float radii[10] = {0.1f, 0.2f, 0.3f, 0.4f, 0.5f, 0.6f, 0.7f, 0.8f, 0.9f, 1.0f};
    static const double widths[10] = {0.70, 0.45, 0.30, 0.25, 0.22, 0.20, 0.18, 0.17, 0.16, 0.15};
    if (!(radius >= radii[0] && radius <= radii[9])) return 0;
    for (unsigned j = 0; j < 10; ++j) {
        if (radius == radii[j]) {
            *out = widths[j];
            return 1;
        }
        if (j > 0 && radius < radii[j]) {
            const double f = ((double)radius - radii[j - 1]) / ((double)radii[j] - radii[j - 1]);
            *out = fma(f, widths[j] - widths[j - 1], widths[j - 1]);
            return 1;
        }
    }
    return 0;
}

/* cfg = {primary sigma (rad), support (sigmas), transition contrast, inner blend (sigmas)} */
int icpo_rainbow_config_ok(uint32_t nt, uint32_t np, const double* cfg)
{
    return nt >= 2u && np >= 1u && nt <= 32767u && np <= 32767u && cfg[0] > 0 && fin(cfg[0]) && cfg[1] >= 2 &&
           cfg[1] <= 8 && cfg[3] >= 0 && cfg[3] < cfg[1] && 2 * cfg[0] * cfg[1] < ICPO_PI && cfg[2] >= 0 && cfg[2] < 1;
}

static int rb_sample_ok(const rb_focal* r) { return r->flags == 0 && r->s >= 0 && r->p >= 0 && fin(r->s + r->p); }

void icpo_rainbow_detect(const rb_focal* f, uint32_t nt, uint32_t np, const double* cfg, uint32_t* edges)
{
    const uint64_t n = (uint64_t)nt * np;
    const int ok = icpo_rainbow_config_ok(nt, np, cfg);
    for (uint64_t i = 0; i < n; ++i) {
        uint32_t e = 0;
        if (!ok)
            e = RB_UNKNOWN;
        else if (i / np + 1 != nt) { /* the last row has no edge below it */
            const rb_focal* a = f + i;
            const rb_focal* b = a + np;
            if (!rb_sample_ok(a) || !rb_sample_ok(b))
                e = RB_UNKNOWN;
            else {
                const double x = a->s + a->p, y = b->s + b->p, peak = fmax(x, y);
                if (peak > 0 && fin(peak) && !(fabs(y - x) / peak < cfg[2])) {
                    /* entering TRT support with increasing theta / leaving TRRT support */
                    if (a->fam_hits[2] == 0 && b->fam_hits[2] > 0 && b->fam_inc[2] > 0) e |= RB_PRIMARY;
                    if (a->fam_hits[3] > 0 && b->fam_hits[3] == 0 && a->fam_inc[3] > 0) e |= RB_SECONDARY;
                }
            }
        }
        edges[i] = e;
    }
}

static int rb_wrap(int a, int n)
{
    const int r = a % n;
    return r < 0 ? r + n : r;
}
double icpo_rainbow_distance(double a, double b, double phi)
{
    const double u = sin(0.5 * (a - b)), v = sin(0.5 * phi);
    const double h = fma(sin(a) * sin(b), v * v, u * u);
    return 2 * asin(sqrt(fmin(1.0, fmax(0.0, h))));
}
/* Half-width in columns of the longitude window of the cap of `radius` around colatitude t
 * on row colatitude r; -1 when the row misses the cap, nc when the cap wraps the row. */
static int rb_window(double t, double r, double radius, double dp, int nc)
{
    if (fabs(t - r) > radius + RB_TOL) return -1;
    const double a = sin(t) * sin(r), b = cos(t) * cos(r);
    if (!(a > 0)) return nc;
    const double x = (cos(radius) - b) / a;
    if (x <= -1) return nc;
    if (x >= 1) return 1;
    const int w = (int)ceil(acos(x) / dp) + 1;
    return nc < w ? nc : w;
}
static void rb_add(rb_sum* z, double x)
{
    const double n = z->s + x;
    z->c += fabs(z->s) >= fabs(x) ? (z->s - n) + x : (x - n) + z->s;
    z->s = n;
}
static void rb_unavailable(rb_result* r) { r->s = r->p = NAN; }

static rb_result rb_filter_one(const rb_focal* f, const uint32_t* edges, int nr, int nc, const double* cfg, int ok,
                               uint32_t index)
{
    rb_result out = {0, 0, 0, 0, 0, 0};
    if (!ok) {
        out.flags = RB_INVALID;
        rb_unavailable(&out);
        return out;
    }
    const rb_focal* c0 = f + index;
    if (!rb_sample_ok(c0)) {
        out.flags = RB_INPUT;
        rb_unavailable(&out);
        return out;
    }
    out.s = c0->s;
    out.p = c0->p;
    const int row = (int)(index / (uint32_t)nc), col = (int)(index % (uint32_t)nc);
    const double dt = ICPO_PI / (double)nr, dp = 2 * ICPO_PI / (double)nc, t = (row + 0.5) * dt;
    const double support = cfg[1];
    /* nearest labelled edge within twice the primary support, in units of its own sigma */
    const double search = 2 * cfg[0] * support;
    int lo = (int)floor((t - search) / dt) - 1, hi = (int)ceil((t + search) / dt);
    if (lo < 0) lo = 0;
    if (hi > nr - 2) hi = nr - 2;
    double best = support + 1;
    for (int rr = lo; rr <= hi; ++rr) {
        const double tr = (rr + 1.0) * dt; /* the edge lies between rows rr and rr + 1 */
        const int w = rb_window(t, tr, search, dp, nc);
        if (w < 0) continue;
        const int count = nc < 2 * w + 1 ? nc : 2 * w + 1, start = count == nc ? 0 : col - w;
        for (int j = 0; j < count; ++j) {
            const int cc = rb_wrap(start + j, nc);
            const double d = icpo_rainbow_distance(t, tr, (cc - col) * dp);
            if (d > search + RB_TOL) continue;
            const uint32_t e = edges[(uint32_t)rr * (uint32_t)nc + (uint32_t)cc];
            if (e & RB_UNKNOWN) out.flags |= RB_DETECT;
            for (uint32_t kind = RB_PRIMARY; kind <= RB_SECONDARY; kind *= 2u) {
                if (!(e & kind)) continue;
                const double sigma = cfg[0] * (kind == RB_SECONDARY ? 2 : 1);
                const double dist = d / sigma;
                if (dist < support && (dist < best - 1e-12 || (fabs(dist - best) <= 1e-12 && kind < out.kind))) {
                    best = dist;
                    out.sigma = sigma;
                    out.kind = kind;
                }
            }
        }
    }
    if (out.flags & RB_DETECT) {
        rb_unavailable(&out);
        return out;
    }
    if (out.kind == 0) return out;
    const double sigma = out.sigma;
    if (dt > 0.5 * sigma || sin(t) * dp > 0.5 * sigma) out.flags |= RB_UNDER;
    out.blend = 1;
    if (best > cfg[3]) {
        const double x = (best - cfg[3]) / (support - cfg[3]);
        out.blend = 1 - x * x * (3 - 2 * x);
    }
    /* solid-angle weighted Gaussian over the cap of support x sigma, compensated sums */
    const double radius = support * sigma;
    int lower = (int)floor((t - radius) / dt) - 1, upper = (int)ceil((t + radius) / dt);
    if (lower < 0) lower = 0;
    if (upper > nr - 1) upper = nr - 1;
    rb_sum ws = {0, 0}, ss = {0, 0}, sp = {0, 0};
    for (int rr = lower; rr <= upper; ++rr) {
        const double tr = (rr + 0.5) * dt;
        const int w = rb_window(t, tr, radius, dp, nc);
        if (w < 0) continue;
        const int count = nc < 2 * w + 1 ? nc : 2 * w + 1, start = count == nc ? 0 : col - w;
        const double area = 2 * sin(tr) * sin(0.5 * dt) * dp;
        for (int j = 0; j < count; ++j) {
            const int cc = rb_wrap(start + j, nc);
            const double d = icpo_rainbow_distance(t, tr, (cc - col) * dp);
            if (d > radius + RB_TOL) continue;
            const rb_focal* q = f + (uint32_t)rr * (uint32_t)nc + (uint32_t)cc;
            if (!rb_sample_ok(q)) {
                out.flags |= RB_STENCIL;
                continue;
            }
            const double weight = exp(-0.5 * (d / sigma) * (d / sigma)) * area;
            rb_add(&ws, weight);
            rb_add(&ss, weight * q->s);
            rb_add(&sp, weight * q->p);
        }
    }
    if (out.flags & RB_STENCIL) {
        rb_unavailable(&out);
        return out;
    }
    const double total = ws.s + ws.c;
    if (!(total > 0) || !fin(total)) {
        out.flags |= RB_INVALID;
        rb_unavailable(&out);
        return out;
    }
    /* constant-preserving local normalisation, blended toward the unfiltered value */
    out.s = fma(out.blend, (ss.s + ss.c) / total - c0->s, c0->s);
    out.p = fma(out.blend, (sp.s + sp.c) / total - c0->p, c0->p);
    if (!(out.s >= 0 && out.p >= 0) || !fin(out.s + out.p)) {
        out.flags |= RB_INVALID;
        rb_unavailable(&out);
        return out;
    }
    out.flags |= RB_FILTERED;
    return out;
}

void icpo_rainbow_filter(const rb_focal* f, const uint32_t* edges, uint32_t nt, uint32_t np, const double* cfg,
                         rb_result* out)
{
    const int ok = icpo_rainbow_config_ok(nt, np, cfg);
    const uint64_t n = (uint64_t)nt * np;
    for (uint64_t i = 0; i < n; ++i) out[i] = rb_filter_one(f, edges, (int)nt, (int)np, cfg, ok, (uint32_t)i);
}

/* The filter at `count` chosen directions only (bounded CPU time on large grids). */
void icpo_rainbow_filter_at(const rb_focal* f, const uint32_t* edges, uint32_t nt, uint32_t np, const double* cfg,
                            const uint64_t* index, uint64_t count, rb_result* out)
{
    const int ok = icpo_rainbow_config_ok(nt, np, cfg);
    for (uint64_t k = 0; k < count; ++k)
        out[k] = rb_filter_one(f, edges, (int)nt, (int)np, cfg, ok, (uint32_t)index[k]);
}

/* ------------------------------------------------------------- patch optics
 * Restates the reference's per-direction optics of the drop's wave stages:
 *   PatchOpticalEvaluator::evaluate_patch / evaluate_direction
 *                          include/rainbow/patch_optical_evaluator.hpp:26-326 (no folded view)
 *   scattering frame, minimum-rotation transport
 *                          include/rainbow/polarization_transport.hpp:24-229
 *   optical-path cycles    include/rainbow/phase_cycles.hpp:20-97, phase_interpolation.hpp:22-151
 *   focal quarter turns    include/rainbow/focal_phase.hpp:18-104
 *   float vectors          include/rainbow/vec3.hpp:11-66 (explicit fmaf dots, plain crosses)
 * Binary32 and binary64 as the reference writes them, no contraction, same libm calls, so the
 * results equal the reference's headers compiled on the same host bit for bit.  Record layouts
 * are the reference's (OutgoingVertex 68 B, OutgoingPatch / PatchQueryHit / PatchQuerySummary
 * 32 B, PatchOpticalResult 136 B, FocalOpticalResult 144 B). */
typedef struct { float x, y, z; } pf3;
typedef struct { double x, y, z; } pd3;
typedef struct { float re, im; } pc32;
typedef struct { pc32 x, y; } pfield;
typedef struct { int32_t turns; float fraction; } pcycles;
typedef struct {
    pf3 position, direction, basis;
    pfield field;
    pcycles cycles;
    uint32_t status, diagnostics;
} pvertex;
typedef struct {
    uint32_t v[4];
    uint32_t patch_id, status;
    float solid_angle, area;
} ppatch;
typedef struct {
    uint32_t compact, patch_id, root, flags;
    float u, v, t, residual;
} phit;
typedef struct {
    uint32_t candidates, hits, regular, refinement, boundary, flags, first_problem, reserved;
} psummary;
typedef struct { double sr, si, pr, pi; } pf64;
typedef struct {
    pf64 path;
    double inc_s, inc_p, path_s, path_p;
    uint32_t hits, evaluated, rejected, refinement, boundary, singular, flags, query_flags, first_problem, folded;
    pf64 path2;
} poptical;
typedef struct { pf3 e0, e1; } pframe;
typedef struct {
    const pvertex* vertices;
    const ppatch* patches;
    const pf3* directions;
    const uint64_t* offsets;
    const psummary* summaries;
    const phit* hits;
    const pfield* second;
    uint64_t hit_storage;
    uint32_t vertex_count, patch_count, direction_count, second_count;
    pf3 incident, incident_basis;
    uint32_t polarization, reserved;
} pinput;
typedef struct {
    uint32_t width, height;
    float half_extent;
    uint32_t reserved;
    uint32_t offsets[4];
} pfocal_cfg;

enum { PO_QUERY = 1, PO_INPUT = 2, PO_FRAME = 4, PO_PHASE = 8, PO_ARITH = 16, PO_REFINE = 32, PO_BOUNDARY = 64,
       PO_SINGULAR = 128 };
#define PO_ERRORS (PO_QUERY | PO_INPUT | PO_FRAME | PO_PHASE | PO_ARITH)
#define PO_PENDING (PO_REFINE | PO_BOUNDARY | PO_SINGULAR)
enum { PQ_REFINE_HIT = 8, PQ_BOUNDARY_HIT = 16, PQ_SINGULAR_HIT = 128 };
#define PQ_ERRORS (1u | 2u | 4u | 256u)
enum { FO_INPUT_ERROR = 1, FO_INPUT_PENDING = 2, FO_DERIVATIVE = 4, FO_GEOMETRY = 8, FO_ARITH = 16 };
#define PT_TOL 0x1p-10f   /* unit / orthogonality tolerance of frames */
#define PT_DEGEN 0x1p-30f /* degenerate cross product                 */

static float f3_dot(pf3 a, pf3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
static pf3 f3_cross(pf3 a, pf3 b)
{
    pf3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static pf3 f3_scale(pf3 a, float s) { pf3 r = {a.x * s, a.y * s, a.z * s}; return r; }
static pf3 f3_div(pf3 a, float s) { pf3 r = {a.x / s, a.y / s, a.z / s}; return r; }
static pf3 f3_sub(pf3 a, pf3 b) { pf3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static int f3_fin(pf3 a)
{
    const float m = 0x1.fffffep127f;
    return a.x >= -m && a.x <= m && a.y >= -m && a.y <= m && a.z >= -m && a.z <= m;
}
static pf3 f3_unit(pf3 a) { return f3_div(a, sqrtf(f3_dot(a, a))); }
static pd3 f3_wide(pf3 a) { pd3 r = {a.x, a.y, a.z}; return r; }
static double d3_dot(pd3 a, pd3 b) { return fma(a.x, b.x, fma(a.y, b.y, a.z * b.z)); }
static pd3 d3_cross(pd3 a, pd3 b)
{
    pd3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static pd3 d3_scale(pd3 a, double s) { pd3 r = {a.x * s, a.y * s, a.z * s}; return r; }
static pd3 d3_div(pd3 a, double s) { pd3 r = {a.x / s, a.y / s, a.z / s}; return r; }
static pd3 d3_add(pd3 a, pd3 b) { pd3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static pd3 d3_unit(pd3 a) { return d3_div(a, sqrt(d3_dot(a, a))); }

static int pt_unit(pf3 a) { return f3_fin(a) && fabsf(f3_dot(a, a) - 1.0f) <= PT_TOL; }
static int pt_frame(pf3 d, pframe f)
{
    if (!pt_unit(f.e0) || !pt_unit(f.e1)) return 0;
    if (fabsf(f3_dot(d, f.e0)) > PT_TOL || fabsf(f3_dot(d, f.e1)) > PT_TOL || fabsf(f3_dot(f.e0, f.e1)) > PT_TOL)
        return 0;
    return f3_dot(f3_cross(f.e0, f.e1), d) >= 1.0f - 4.0f * PT_TOL;
}
/* e0 normal to the scattering plane (or the incident basis carried over at exact forward /
 * backward scattering), e1 = out x e0. */
static int pt_scattering_frame(pf3 inc, pf3 basis, pf3 out, pframe* frame)
{
    if (!pt_unit(inc) || !pt_unit(out) || !pt_unit(basis) || fabsf(f3_dot(inc, basis)) > PT_TOL) return 0;
    pf3 e0 = f3_cross(inc, out);
    float n2 = f3_dot(e0, e0);
    if (n2 > PT_DEGEN)
        e0 = f3_div(e0, sqrtf(n2));
    else {
        e0 = f3_sub(basis, f3_scale(out, f3_dot(out, basis)));
        n2 = f3_dot(e0, e0);
        if (!(n2 > PT_DEGEN)) return 0;
        e0 = f3_div(e0, sqrtf(n2));
    }
    pf3 e1 = f3_cross(out, e0);
    const float m2 = f3_dot(e1, e1);
    if (!(m2 > PT_DEGEN)) return 0;
    e1 = f3_div(e1, sqrtf(m2));
    const pframe f = {e0, e1};
    if (!pt_frame(out, f)) return 0;
    *frame = f;
    return 1;
}
/* Rodrigues' rotation by the minimum rotation taking a to b (v = a x b, c = a.b). */
static pd3 pt_rotate(pd3 x, pd3 a, pd3 b, double c)
{
    const pd3 v = d3_cross(a, b), vx = d3_cross(v, x);
    return d3_add(d3_add(x, vx), d3_div(d3_cross(v, vx), 1.0 + c));
}
static int pt_fits(double x) { return x >= -0x1.fffffep127 && x <= 0x1.fffffep127; }
static int pfield_fin(pfield f)
{
    return fin(f.x.re) && fin(f.x.im) && fin(f.y.re) && fin(f.y.im);
}
static int pfield_fin32(pfield f)
{
    const float m = 0x1.fffffep127f;
    return f.x.re >= -m && f.x.re <= m && f.x.im >= -m && f.x.im <= m && f.y.re >= -m && f.y.re <= m &&
           f.y.im >= -m && f.y.im <= m;
}
/* One Jones column carried from the source frame to the target frame (the shared geometry
 * is set up by the caller). */
static int pt_carry(pfield f, pd3 se0, pd3 se1, pd3 sw, pd3 tw, double c, pd3 te0, pd3 te1, pfield* out)
{
    const pd3 re = d3_add(d3_scale(se0, (double)f.x.re), d3_scale(se1, (double)f.y.re));
    const pd3 im = d3_add(d3_scale(se0, (double)f.x.im), d3_scale(se1, (double)f.y.im));
    const pd3 rt = pt_rotate(re, sw, tw, c), it = pt_rotate(im, sw, tw, c);
    const double xr = d3_dot(rt, te0), xi = d3_dot(it, te0), yr = d3_dot(rt, te1), yi = d3_dot(it, te1);
    if (!pt_fits(xr) || !pt_fits(xi) || !pt_fits(yr) || !pt_fits(yi)) return 0;
    out->x.re = (float)xr;
    out->x.im = (float)xi;
    out->y.re = (float)yr;
    out->y.im = (float)yi;
    return 1;
}
/* try_transport (columns = 1) and try_transport_response (columns = 2). */
static int pt_transport(pf3 sdir, pframe sf, const pfield* src, unsigned columns, pf3 tdir, pframe tf, pfield* out)
{
    if (columns == 2 && (!pfield_fin32(src[0]) || !pfield_fin32(src[1]))) return 0;
    if (!pt_unit(sdir) || !pt_unit(tdir) || !pt_frame(sdir, sf) || !pt_frame(tdir, tf)) return 0;
    const pd3 sw = d3_unit(f3_wide(sdir)), tw = d3_unit(f3_wide(tdir));
    const double c = d3_dot(sw, tw);
    if (!(1.0 + c > 0x1p-30)) return 0;
    const pd3 se0 = f3_wide(sf.e0), se1 = f3_wide(sf.e1), te0 = f3_wide(tf.e0), te1 = f3_wide(tf.e1);
    pfield tmp[2];
    for (unsigned j = 0; j < columns; ++j)
        if (!pt_carry(src[j], se0, se1, sw, tw, c, te0, te1, &tmp[j])) return 0;
    for (unsigned j = 0; j < columns; ++j) out[j] = tmp[j];
    return 1;
}

static int cyc_ok(pcycles q) { return q.fraction >= 0.0f && q.fraction < 1.0f; }
static double cyc_diff(pcycles a, pcycles b)
{
    const int64_t whole = (int64_t)a.turns - (int64_t)b.turns;
    return (double)whole + ((double)a.fraction - (double)b.fraction);
}
/* anchor + delta cycles, fraction carried into [0, 1) (phase_interpolation.hpp:96-151) */
static int cyc_add(pcycles anchor, double delta, pcycles* out)
{
    if (!(delta > -0x1p33 && delta < 0x1p33)) return 0;
    const double whole = floor(delta);
    double frac = (double)anchor.fraction + (delta - whole);
    int64_t turns = (int64_t)anchor.turns + (int64_t)whole;
    if (frac < 0.0) {
        --turns;
        frac += 1.0;
    }
    if (frac >= 1.0) {
        ++turns;
        frac -= 1.0;
    }
    if (turns < -2147483647LL - 1 || turns > 2147483647LL) return 0;
    float stored = (float)frac;
    if (stored >= 1.0f) {
        ++turns;
        stored = 0.0f;
        if (turns > 2147483647LL) return 0;
    } else if (stored < 0.0f) {
        --turns;
        stored += 1.0f;
        if (turns < -2147483647LL - 1) return 0;
    }
    out->turns = (int32_t)turns;
    out->fraction = stored == 0.0f ? 0.0f : stored;
    return cyc_ok(*out);
}
/* bilinear optical path from the four corners, anchored at q00 (corners returned exactly) */
static int cyc_bilinear(pcycles q00, pcycles q10, pcycles q01, pcycles q11, float u, float v, pcycles* out)
{
    if (!cyc_ok(q00) || !cyc_ok(q10) || !cyc_ok(q01) || !cyc_ok(q11) || !(u >= 0.0f && u <= 1.0f) ||
        !(v >= 0.0f && v <= 1.0f))
        return 0;
    if (u == 0.0f && v == 0.0f) { *out = q00; return 1; }
    if (u == 1.0f && v == 0.0f) { *out = q10; return 1; }
    if (u == 0.0f && v == 1.0f) { *out = q01; return 1; }
    if (u == 1.0f && v == 1.0f) { *out = q11; return 1; }
    const double du0 = cyc_diff(q10, q00), du1 = cyc_diff(q11, q01), dv0 = cyc_diff(q01, q00);
    const double ud = (double)u, vd = (double)v;
    const double row = fma(ud, du1 - du0, dv0);
    return cyc_add(q00, fma(vd, row, ud * du0), out);
}
/* exp(+i 2 pi fraction) in binary32; exact quarter turns */
static int cyc_phasor(pcycles q, pc32* out)
{
    if (!cyc_ok(q)) return 0;
    const float f = q.fraction;
    if (f == 0.0f) { out->re = 1.0f; out->im = 0.0f; return 1; }
    if (f == 0.25f) { out->re = 0.0f; out->im = 1.0f; return 1; }
    if (f == 0.5f) { out->re = -1.0f; out->im = 0.0f; return 1; }
    if (f == 0.75f) { out->re = 0.0f; out->im = -1.0f; return 1; }
    const float reduced = f > 0.5f ? f - 1.0f : f;
    const float angle = 0x1.921fb6p+2f * reduced;
    out->re = cosf(angle);
    out->im = sinf(angle);
    return 1;
}

static int focal_layout_ok(const pfocal_cfg* c)
{
    if (c->width < 2 || c->height < 2 || !(c->half_extent > 0) || !(c->half_extent <= 0x1.fffffep127f)) return 0;
    if ((uint64_t)c->width * c->height > 0xffffffffull / 4u ||
        (uint64_t)(c->width - 1u) * (c->height - 1u) > 0xffffffffull / 4u)
        return 0;
    for (unsigned j = 0; j < 4; ++j)
        if (c->offsets[j] > 3) return 0;
    return 1;
}
/* Sign of the radial derivative of the scattering angle at the cell centre, in emitting-plane
 * coordinates (focal_phase.hpp:57-98, at_center): one extra quarter turn when it is positive. */
static uint32_t focal_estimate(const pvertex* vertices, uint32_t vertex_count, const ppatch* patch, pf3 incident,
                               const pfocal_cfg* c, uint32_t* family_out, uint32_t* extra_out, uint32_t* turns_out)
{
    if (!vertices || !focal_layout_ok(c) || !f3_fin(incident)) return FO_GEOMETRY;
    const uint32_t n = c->width * c->height, nx = c->width - 1u, cells = nx * (c->height - 1u);
    if (patch->patch_id >= 4u * cells || vertex_count < 4u * n) return FO_GEOMETRY;
    const uint32_t family = patch->patch_id / cells, cell = patch->patch_id % cells;
    const uint32_t ix = cell % nx, iy = cell / nx;
    const uint32_t first = family * n + iy * c->width + ix;
    const uint32_t expected[4] = {first, first + 1u, first + c->width, first + c->width + 1u};
    const pd3 wi = f3_wide(incident);
    if (!(d3_dot(wi, wi) > 0)) return FO_GEOMETRY;
    double theta[4];
    for (unsigned j = 0; j < 4; ++j) {
        if (patch->v[j] != expected[j]) return FO_GEOMETRY;
        const pvertex* a = vertices + expected[j];
        if (a->status != 1u || !f3_fin(a->direction)) return FO_GEOMETRY;
        const pd3 wo = f3_wide(a->direction);
        if (!(d3_dot(wo, wo) > 0)) return FO_GEOMETRY;
        const pd3 x = d3_cross(wi, wo);
        theta[j] = atan2(sqrt(d3_dot(x, x)), d3_dot(wi, wo));
        if (!fin(theta[j])) return FO_GEOMETRY;
    }
    const double e = (double)c->half_extent;
    const double du = 2 * e / (double)(c->width - 1u), dv = 2 * e / (double)(c->height - 1u);
    const double U = (2 * ((double)ix + 0.5) / (double)(c->width - 1u) - 1) * e;
    const double V = (2 * ((double)iy + 0.5) / (double)(c->height - 1u) - 1) * e;
    const double r2 = fma(U, U, V * V);
    if (!(r2 > 0)) return FO_DERIVATIVE;
    const double gu = ((theta[1] - theta[0]) + (theta[3] - theta[2])) / (2 * du);
    const double gv = ((theta[2] - theta[0]) + (theta[3] - theta[1])) / (2 * dv);
    const double num = fma(U, gu, V * gv);
    const double guard = 0x1p-46 * (fabs(U * gu) + fabs(V * gv) + 1);
    if (!fin(num) || !fin(r2)) return FO_GEOMETRY;
    if (fabs(num) <= guard) return FO_DERIVATIVE;
    if (!fin(num / (2 * r2))) return FO_GEOMETRY;
    *family_out = family;
    *extra_out = num > 0 ? 1u : 0u;
    *turns_out = (c->offsets[family] + *extra_out) & 3u;
    return 0;
}
static pf64 focal_turn(pf64 a, uint32_t q)
{
    pf64 r = a;
    switch (q & 3u) {
    case 1: r.sr = -a.si; r.si = a.sr; r.pr = -a.pi; r.pi = a.pr; break;
    case 2: r.sr = -a.sr; r.si = -a.si; r.pr = -a.pr; r.pi = -a.pi; break;
    case 3: r.sr = a.si; r.si = -a.sr; r.pr = a.pi; r.pi = -a.pr; break;
    default: break;
    }
    return r;
}

typedef struct {
    pf64 field[2];
    double inc_s, inc_p;
} pcontrib;
static double lerp2(double a, double b, double c, double d, double u, double v)
{
    const double lower = fma(u, b - a, a), upper = fma(u, d - c, c);
    return fma(v, upper - lower, lower);
}
static int pf64_fin(pf64 f) { return fin(f.sr) && fin(f.si) && fin(f.pr) && fin(f.pi); }

static uint32_t optics_patch(const pinput* in, const ppatch* patch, const phit* hit, pf3 dir, pframe target,
                             pcontrib* out)
{
    if (!in->vertices || (hit->flags & ~(1u | 2u | 4u)) != 0u || hit->patch_id != patch->patch_id || hit->root > 1u ||
        !(hit->u >= 0.0f && hit->u <= 1.0f && hit->v >= 0.0f && hit->v <= 1.0f) || !(hit->t > 0.0f && fin(hit->t)) ||
        !(hit->residual >= 0.0f && fin(hit->residual)))
        return PO_INPUT;
    uint32_t pending = 0;
    if (patch->status == 3u)
        pending |= PO_REFINE; /* no folded records */
    else if (patch->status != 1u && patch->status != 2u)
        return PO_INPUT;
    if (hit->flags & 1u) pending |= PO_BOUNDARY;
    if (hit->flags & 2u) pending |= PO_SINGULAR;
    if (pending) return pending;
    const double area = (double)patch->area, omega = fabs((double)patch->solid_angle);
    if (!(area > 0.0 && fin(area) && omega > 0.0 && fin(omega))) return PO_INPUT;
    const unsigned columns = in->second ? 2u : 1u;
    const double weight = in->second ? 0.5 : 1.0;
    pfield moved[2][4];
    pcycles paths[4];
    for (unsigned k = 0; k < 4; ++k) {
        const uint32_t idx = patch->v[k];
        if (idx >= in->vertex_count) return PO_INPUT;
        const pvertex* vx = in->vertices + idx;
        if (vx->status != 1u || !f3_fin(vx->position) || !f3_fin(vx->direction) || !f3_fin(vx->basis) ||
            !pfield_fin(vx->field))
            return PO_INPUT;
        if (!cyc_ok(vx->cycles)) return PO_PHASE;
        const pf3 second = f3_cross(vx->direction, vx->basis);
        const pd3 s2 = f3_wide(second);
        const double len2 = d3_dot(s2, s2);
        if (!(len2 > 0.0 && fin(len2))) return PO_FRAME;
        const pframe source = {vx->basis, f3_unit(second)};
        pfield src[2] = {vx->field, vx->field};
        pfield got[2];
        if (in->second) {
            src[1] = in->second[idx];
            if (!pfield_fin32(src[0]) || !pfield_fin32(src[1])) return PO_INPUT;
        }
        if (!pt_transport(vx->direction, source, src, columns, dir, target, got)) return PO_FRAME;
        moved[0][k] = got[0];
        if (columns == 2) moved[1][k] = got[1];
        paths[k] = vx->cycles;
    }
    pcycles path;
    if (!cyc_bilinear(paths[0], paths[1], paths[2], paths[3], hit->u, hit->v, &path)) return PO_PHASE;
    pc32 phasor;
    if (!cyc_phasor(path, &phasor)) return PO_PHASE;
    const double amplitude = sqrt(area / omega);
    const double c = (double)phasor.re, s = (double)phasor.im;
    pcontrib cand;
    memset(&cand, 0, sizeof cand);
    for (unsigned j = 0; j < columns; ++j) {
        const pfield* f = moved[j];
        const double u = hit->u, v = hit->v;
        const double sr = amplitude * lerp2(f[0].x.re, f[1].x.re, f[2].x.re, f[3].x.re, u, v);
        const double si = amplitude * lerp2(f[0].x.im, f[1].x.im, f[2].x.im, f[3].x.im, u, v);
        const double pr = amplitude * lerp2(f[0].y.re, f[1].y.re, f[2].y.re, f[3].y.re, u, v);
        const double pi = amplitude * lerp2(f[0].y.im, f[1].y.im, f[2].y.im, f[3].y.im, u, v);
        cand.inc_s += weight * fma(sr, sr, si * si);
        cand.inc_p += weight * fma(pr, pr, pi * pi);
        cand.field[j].sr = fma(sr, c, -si * s);
        cand.field[j].si = fma(sr, s, si * c);
        cand.field[j].pr = fma(pr, c, -pi * s);
        cand.field[j].pi = fma(pr, s, pi * c);
    }
    if (!fin(cand.inc_s) || !fin(cand.inc_p) || !pf64_fin(cand.field[0]) || !pf64_fin(cand.field[1]))
        return PO_ARITH;
    *out = cand;
    return 0;
}

static void optical_nan(poptical* r)
{
    r->path.sr = r->path.si = r->path.pr = r->path.pi = NAN;
    r->path2 = r->path;
    r->inc_s = r->inc_p = r->path_s = r->path_p = NAN;
}
static void focal_nan(rb_focal* r)
{
    for (unsigned k = 0; k < 4; ++k) r->field[k] = r->field2[k] = NAN;
    r->s = r->p = NAN;
}
static int hit_before(const phit* a, const phit* b)
{
    if (a->patch_id != b->patch_id) return a->patch_id < b->patch_id;
    if (a->compact != b->compact) return a->compact < b->compact;
    return a->root < b->root;
}

static poptical optics_direction(const pinput* in, uint32_t index, const pfocal_cfg* fc, rb_focal* focal_out)
{
    poptical res;
    memset(&res, 0, sizeof res);
    res.first_problem = 0xffffffffu;
    const int dual = in->polarization == 1u;
    const unsigned columns = dual ? 2u : 1u;
    const double weight = dual ? 0.5 : 1.0;
    if (focal_out) {
        memset(focal_out, 0, sizeof *focal_out);
        focal_out->first_problem = 0xffffffffu;
        focal_out->flags = FO_INPUT_ERROR;
        focal_nan(focal_out);
    }
    if ((in->polarization != 0u && !dual) || (dual && (!in->second || in->second_count != in->vertex_count)) ||
        (!dual && (in->second || in->second_count != 0u)) || index >= in->direction_count || !in->directions ||
        !in->offsets || !in->summaries) {
        res.flags = PO_INPUT;
        optical_nan(&res);
        return res;
    }
    const psummary* sm = in->summaries + index;
    res.hits = sm->hits;
    res.query_flags = sm->flags;
    if (sm->flags & PQ_ERRORS) {
        res.flags = PO_QUERY;
        res.first_problem = sm->first_problem;
        res.rejected = sm->hits;
        optical_nan(&res);
        return res;
    }
    const uint64_t begin = in->offsets[index], end = in->offsets[index + 1u];
    if (begin > end || end > in->hit_storage || (uint64_t)sm->hits > end - begin ||
        (uint64_t)sm->candidates != end - begin || (sm->hits != 0u && (!in->hits || !in->patches || !in->vertices))) {
        res.flags = PO_INPUT;
        res.rejected = sm->hits;
        optical_nan(&res);
        return res;
    }
    if (sm->flags & PQ_REFINE_HIT) res.flags |= PO_REFINE;
    if (sm->flags & PQ_BOUNDARY_HIT) res.flags |= PO_BOUNDARY;
    if (sm->flags & PQ_SINGULAR_HIT) res.flags |= PO_SINGULAR;
    pframe target;
    if (!pt_scattering_frame(in->incident, in->incident_basis, in->directions[index], &target)) {
        res.flags |= PO_FRAME;
        res.rejected = sm->hits;
        optical_nan(&res);
        return res;
    }
    rb_sum sr[2], si[2], pr[2], pi[2], inc_s, inc_p, fsr[2], fsi[2], fpr[2], fpi[2], env[4];
    memset(sr, 0, sizeof sr); memset(si, 0, sizeof si); memset(pr, 0, sizeof pr); memset(pi, 0, sizeof pi);
    memset(fsr, 0, sizeof fsr); memset(fsi, 0, sizeof fsi); memset(fpr, 0, sizeof fpr); memset(fpi, 0, sizeof fpi);
    memset(env, 0, sizeof env);
    memset(&inc_s, 0, sizeof inc_s);
    memset(&inc_p, 0, sizeof inc_p);
    const int with_focal = fc && focal_out;
    rb_focal focal;
    memset(&focal, 0, sizeof focal);
    focal.first_problem = 0xffffffffu;
    if (with_focal && !focal_layout_ok(fc)) focal.flags |= FO_GEOMETRY;
    for (uint32_t i = 0; i < sm->hits; ++i) {
        const phit* hit = in->hits + begin + i;
        uint32_t flags = 0;
        pcontrib ct;
        memset(&ct, 0, sizeof ct);
        if (i != 0u && !hit_before(hit - 1, hit))
            flags = PO_INPUT; /* the query sorts the hits and removes duplicates */
        else if (hit->compact >= in->patch_count)
            flags = PO_INPUT;
        else
            flags = optics_patch(in, in->patches + hit->compact, hit, in->directions[index], target, &ct);
        if (flags) {
            res.flags |= flags;
            ++res.rejected;
            res.refinement += (flags & PO_REFINE) != 0u;
            res.boundary += (flags & PO_BOUNDARY) != 0u;
            res.singular += (flags & PO_SINGULAR) != 0u;
            if (hit->patch_id < res.first_problem) res.first_problem = hit->patch_id;
            continue;
        }
        ++res.evaluated;
        for (unsigned j = 0; j < columns; ++j) {
            rb_add(&sr[j], ct.field[j].sr);
            rb_add(&si[j], ct.field[j].si);
            rb_add(&pr[j], ct.field[j].pr);
            rb_add(&pi[j], ct.field[j].pi);
        }
        rb_add(&inc_s, ct.inc_s);
        rb_add(&inc_p, ct.inc_p);
        if (with_focal) {
            uint32_t family = 0, extra = 0, turns = 0;
            const uint32_t code = focal_estimate(in->vertices, in->vertex_count, in->patches + hit->compact,
                                                 in->incident, fc, &family, &extra, &turns);
            if (code) {
                focal.flags |= code;
                if (hit->patch_id < focal.first_problem) focal.first_problem = hit->patch_id;
            } else {
                for (unsigned j = 0; j < columns; ++j) {
                    const pf64 f = focal_turn(ct.field[j], turns);
                    rb_add(&fsr[j], f.sr);
                    rb_add(&fsi[j], f.si);
                    rb_add(&fpr[j], f.pr);
                    rb_add(&fpi[j], f.pi);
                }
                rb_add(&env[family], ct.inc_s + ct.inc_p);
                ++focal.fam_hits[family];
                ++focal.corrected;
                focal.extra += extra;
            }
        }
    }
    const pf64 f0 = {sr[0].s + sr[0].c, si[0].s + si[0].c, pr[0].s + pr[0].c, pi[0].s + pi[0].c};
    const pf64 f1 = {sr[1].s + sr[1].c, si[1].s + si[1].c, pr[1].s + pr[1].c, pi[1].s + pi[1].c};
    res.path = f0;
    res.path2 = f1;
    res.inc_s = inc_s.s + inc_s.c;
    res.inc_p = inc_p.s + inc_p.c;
    for (unsigned j = 0; j < columns; ++j) {
        const pf64 f = j == 0 ? f0 : f1;
        res.path_s += weight * fma(f.sr, f.sr, f.si * f.si);
        res.path_p += weight * fma(f.pr, f.pr, f.pi * f.pi);
    }
    if (!pf64_fin(res.path) || !pf64_fin(res.path2) || !fin(res.inc_s) || !fin(res.inc_p) || !fin(res.path_s) ||
        !fin(res.path_p))
        res.flags |= PO_ARITH;
    if (res.flags & PO_ERRORS) optical_nan(&res);
    if (with_focal) {
        if (res.flags & PO_ERRORS) focal.flags |= FO_INPUT_ERROR;
        if (res.flags & PO_PENDING) focal.flags |= FO_INPUT_PENDING;
        if (res.first_problem < focal.first_problem) focal.first_problem = res.first_problem;
        const double g[2][4] = {{fsr[0].s + fsr[0].c, fsi[0].s + fsi[0].c, fpr[0].s + fpr[0].c, fpi[0].s + fpi[0].c},
                                {fsr[1].s + fsr[1].c, fsi[1].s + fsi[1].c, fpr[1].s + fpr[1].c, fpi[1].s + fpi[1].c}};
        for (unsigned k = 0; k < 4; ++k) {
            focal.field[k] = g[0][k];
            focal.field2[k] = g[1][k];
        }
        for (unsigned j = 0; j < columns; ++j) {
            focal.s += weight * fma(g[j][0], g[j][0], g[j][1] * g[j][1]);
            focal.p += weight * fma(g[j][2], g[j][2], g[j][3] * g[j][3]);
        }
        for (unsigned k = 0; k < 4; ++k) focal.fam_inc[k] = env[k].s + env[k].c;
        if (!fin(g[0][0]) || !fin(g[0][1]) || !fin(g[0][2]) || !fin(g[0][3]) || !fin(g[1][0]) || !fin(g[1][1]) ||
            !fin(g[1][2]) || !fin(g[1][3]) || !fin(focal.s + focal.p))
            focal.flags |= FO_ARITH;
        if (focal.flags) focal_nan(&focal);
        *focal_out = focal;
    }
    return res;
}

/* Every direction of the input; focal results too when fc != NULL. */
void icpo_patch_optics(const pinput* in, const pfocal_cfg* fc, poptical* results, rb_focal* focal)
{
    for (uint32_t i = 0; i < in->direction_count; ++i)
        results[i] = optics_direction(in, i, fc, fc ? focal + i : NULL);
}

/* ---------------------------------------------------------------- patch build
 * Restates the reference's patch construction (PatchConstruction::make,
 * include/rainbow/patch_geometry.hpp:117-172; BilinearPatchGeometry :75-114 with its outward
 * rounded interval orientation test and the two-triangle solid angle; the layout of
 * include/rainbow/outgoing_patch.hpp:59-92) and its compaction in patch_id order
 * (device/patch_build.cu:13-77).  Binary32 with the reference's explicit fmaf and nextafterf,
 * no contraction: bit-identical to the reference's headers compiled on the host. */
typedef struct { float lo, hi; } piv;
typedef struct { piv x, y, z; } piv3;
typedef struct { float min_x, min_y, min_z, max_x, max_y, max_z; } paabb;

static piv iv_pt(float x) { piv r = {x, x}; return r; }
static piv iv_add(piv a, piv b) { piv r = {nextafterf(a.lo + b.lo, -INFINITY), nextafterf(a.hi + b.hi, INFINITY)}; return r; }
static piv iv_sub(piv a, piv b) { piv r = {nextafterf(a.lo - b.hi, -INFINITY), nextafterf(a.hi - b.lo, INFINITY)}; return r; }
static piv iv_mul(piv a, piv b)
{
    const float p0 = a.lo * b.lo, p1 = a.lo * b.hi, p2 = a.hi * b.lo, p3 = a.hi * b.hi;
    piv r = {nextafterf(fminf(fminf(p0, p1), fminf(p2, p3)), -INFINITY),
             nextafterf(fmaxf(fmaxf(p0, p1), fmaxf(p2, p3)), INFINITY)};
    return r;
}
static piv3 iv3_pt(pf3 p) { piv3 r = {iv_pt(p.x), iv_pt(p.y), iv_pt(p.z)}; return r; }
static piv3 iv3_sub(piv3 a, piv3 b) { piv3 r = {iv_sub(a.x, b.x), iv_sub(a.y, b.y), iv_sub(a.z, b.z)}; return r; }
static piv3 iv3_cross(piv3 a, piv3 b)
{
    piv3 r = {iv_sub(iv_mul(a.y, b.z), iv_mul(a.z, b.y)), iv_sub(iv_mul(a.z, b.x), iv_mul(a.x, b.z)),
              iv_sub(iv_mul(a.x, b.y), iv_mul(a.y, b.x))};
    return r;
}
static piv iv3_dot(piv3 a, piv3 b) { return iv_add(iv_add(iv_mul(a.x, b.x), iv_mul(a.y, b.y)), iv_mul(a.z, b.z)); }

static float pb_dop(float x, float y, float z, float w)
{
    const float zw = z * w;
    const float residual = fmaf(-z, w, zw);
    return fmaf(x, y, -zw) + residual;
}
static float pb_det(pf3 a, pf3 b, pf3 c)
{
    const pf3 u = f3_sub(b, a), v = f3_sub(c, a);
    return fmaf(a.x, pb_dop(u.y, v.z, u.z, v.y), fmaf(a.y, pb_dop(u.z, v.x, u.x, v.z), a.z * pb_dop(u.x, v.y, u.y, v.x)));
}
/* signed solid angle of the spherical triangle (Van Oosterom & Strackee) */
static float pb_triangle(pf3 a, pf3 b, pf3 c)
{
    const float la = sqrtf(f3_dot(a, a)), lb = sqrtf(f3_dot(b, b)), lc = sqrtf(f3_dot(c, c));
    const float den = fmaf(la, lb * lc, fmaf(f3_dot(a, b), lc, fmaf(f3_dot(b, c), la, f3_dot(c, a) * lb)));
    return 2.0f * atan2f(pb_det(a, b, c), den);
}
static pf3 f3_add(pf3 a, pf3 b) { pf3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
/* +1 / -1 when the corner Jacobians have one certified sign and all corners lie in the
 * hemisphere of their mean direction; 0 otherwise */
static int pb_orientation(const pf3* c)
{
    const piv3 p0 = iv3_pt(c[0]), p1 = iv3_pt(c[1]), p2 = iv3_pt(c[2]), p3 = iv3_pt(c[3]);
    const piv d0 = iv3_dot(p0, iv3_cross(iv3_sub(p1, p0), iv3_sub(p2, p0)));
    const piv d1 = iv3_dot(p1, iv3_cross(iv3_sub(p1, p0), iv3_sub(p3, p1)));
    const piv d2 = iv3_dot(p2, iv3_cross(iv3_sub(p3, p2), iv3_sub(p2, p0)));
    const piv d3 = iv3_dot(p3, iv3_cross(iv3_sub(p3, p2), iv3_sub(p3, p1)));
    const int positive = d0.lo > 0 && d1.lo > 0 && d2.lo > 0 && d3.lo > 0;
    const int negative = d0.hi < 0 && d1.hi < 0 && d2.hi < 0 && d3.hi < 0;
    if (!positive && !negative) return 0;
    const piv3 a = iv3_pt(f3_add(f3_add(c[0], c[1]), f3_add(c[2], c[3])));
    if (!(iv3_dot(a, p0).lo > 0 && iv3_dot(a, p1).lo > 0 && iv3_dot(a, p2).lo > 0 && iv3_dot(a, p3).lo > 0)) return 0;
    return positive ? 1 : -1;
}
static paabb pb_bounds(const pf3* c)
{
    pf3 lo = c[0], hi = c[0];
    for (unsigned i = 1; i < 4; ++i) {
        lo.x = fminf(lo.x, c[i].x); lo.y = fminf(lo.y, c[i].y); lo.z = fminf(lo.z, c[i].z);
        hi.x = fmaxf(hi.x, c[i].x); hi.y = fmaxf(hi.y, c[i].y); hi.z = fmaxf(hi.z, c[i].z);
    }
    const float pad = 0x1p-19f;
    paabb r = {nextafterf(lo.x - pad, -INFINITY), nextafterf(lo.y - pad, -INFINITY), nextafterf(lo.z - pad, -INFINITY),
               nextafterf(hi.x + pad, INFINITY), nextafterf(hi.y + pad, INFINITY), nextafterf(hi.z + pad, INFINITY)};
    return r;
}
static int pb_usable(const pvertex* v)
{
    const float n2 = f3_dot(v->direction, v->direction);
    return f3_fin(v->position) && f3_fin(v->direction) && f3_fin(v->basis) && fabsf(n2 - 1.0f) <= 0x1p-16f &&
           cyc_ok(v->cycles) && pfield_fin32(v->field);
}
typedef struct { uint32_t width, height, per_path, cells, cell_count; float area; } playout;
/* PatchBuildLayout::try_make */
int icpo_patch_layout(uint32_t width, uint32_t height, float half_extent, uint32_t* out /* 5 */, float* area)
{
    if (width < 2 || height < 2 || !(half_extent > 0.0f) || !(half_extent <= 0x1.fffffep127f)) return 0;
    const uint64_t vertices = (uint64_t)width * height, cells = (uint64_t)(width - 1) * (height - 1);
    if (vertices > 0xffffffffull / 4u || cells > 0xffffffffull / 4u) return 0;
    const float du = 2.0f * half_extent / (float)(width - 1), dv = 2.0f * half_extent / (float)(height - 1);
    const float a = du * dv;
    if (!(a > 0.0f && a <= 0x1.fffffep127f)) return 0;
    out[0] = width;
    out[1] = height;
    out[2] = (uint32_t)vertices;
    out[3] = (uint32_t)cells;
    out[4] = (uint32_t)(4 * cells);
    *area = a;
    return 1;
}
static void pb_make(const pvertex* vertices, const playout* L, uint32_t id, ppatch* patch, paabb* box)
{
    memset(patch, 0, sizeof *patch);
    memset(box, 0, sizeof *box);
    patch->patch_id = id;
    patch->area = L->area;
    patch->solid_angle = NAN;
    const uint32_t family = id / L->cells, cell = id % L->cells;
    const uint32_t ix = cell % (L->width - 1), iy = cell / (L->width - 1);
    const uint32_t first = family * L->per_path + iy * L->width + ix;
    patch->v[0] = first;
    patch->v[1] = first + 1;
    patch->v[2] = first + L->width;
    patch->v[3] = first + L->width + 1;
    unsigned valid = 0;
    int bad_vertex = 0, bad_geometry = 0;
    pf3 corners[4];
    memset(corners, 0, sizeof corners);
    for (unsigned i = 0; i < 4; ++i) {
        const pvertex* v = vertices + patch->v[i];
        if (v->status == 1u) {
            ++valid;
            bad_geometry |= !pb_usable(v);
            corners[i] = v->direction;
        } else if (v->status != 2u && v->status != 3u) /* neither a miss nor total internal reflection */
            bad_vertex = 1;
    }
    if (bad_vertex) patch->status = 6;
    else if (bad_geometry) patch->status = 7;
    else if (valid == 0) patch->status = 5;
    else if (valid < 4) patch->status = 4;
    else {
        *box = pb_bounds(corners);
        const int orientation = pb_orientation(corners);
        patch->status = 3; /* needs refinement unless certified regular */
        if (orientation != 0) {
            const float angle = pb_triangle(corners[0], corners[1], corners[3]) + pb_triangle(corners[0], corners[3], corners[2]);
            if (angle >= -0x1.fffffep127f && angle <= 0x1.fffffep127f && angle * (float)orientation > 0.0f) {
                patch->status = orientation > 0 ? 1u : 2u;
                patch->solid_angle = angle;
            }
        }
    }
}
/* Every cell's status (statuses[cell_count]), the patches with geometry (status 1..3) in
 * patch_id order with their boxes, and the status histogram; returns the patch count. */
uint32_t icpo_patch_build(const pvertex* vertices, uint32_t width, uint32_t height, float half_extent,
                          uint32_t* statuses, ppatch* patches, paabb* boxes, uint32_t* histogram /* 8 */)
{
    uint32_t lay[5];
    float area;
    if (!icpo_patch_layout(width, height, half_extent, lay, &area)) return 0xffffffffu;
    const playout L = {lay[0], lay[1], lay[2], lay[3], lay[4], area};
    uint32_t count = 0;
    for (unsigned k = 0; k < 8; ++k) histogram[k] = 0;
    for (uint32_t id = 0; id < L.cell_count; ++id) {
        ppatch p;
        paabb b;
        pb_make(vertices, &L, id, &p, &b);
        statuses[id] = p.status;
        ++histogram[p.status];
        if (p.status >= 1u && p.status <= 3u) {
            patches[count] = p;
            boxes[count] = b;
            ++count;
        }
    }
    return count;
}

/* ------------------------------------------------ ray / bilinear patch intersection
 * Restates BilinearPatchIntersector::intersect (include/rainbow/bilinear_patch_intersection.hpp
 * :58-314): the patch and the ray projected along the ray's dominant axis, the quadratic in u
 * with scaled coefficients, three Newton steps in (u, v), the acceptance tests, first in binary32
 * and, when that is not conclusive, again in binary64.  One generic body instantiated for both
 * types by the macro below; same operations and order as the reference's template. */
typedef struct { float u, v, t, residual; uint32_t flags; } pbhit;
typedef struct { pbhit hits[2]; uint32_t count, flags; } pbhits;
enum { BH_BOUNDARY = 1, BH_SINGULAR = 2, BH_FP64 = 4 };
enum { BQ_UNRESOLVED = 1, BQ_INVALID = 2, BQ_FP64 = 4 };

#define PB_SOLVER(T, SUF, FMA, SQRT, COPYSIGN, EPS, IS_FLOAT)                                                       \
    typedef struct { T x, y; } pb2##SUF;                                                                            \
    typedef struct { T x, y, z; } pb3##SUF;                                                                         \
    static T pb_abs_##SUF(T x) { return x < (T)0 ? -x : x; }                                                         \
    static T pb_max_##SUF(T a, T b) { return a > b ? a : b; }                                                        \
    static T pb_dop##SUF(T x, T y, T z, T w) { const T zw = z * w; return FMA(x, y, -zw) + FMA(-z, w, zw); }        \
    static pb2##SUF pb2_add##SUF(pb2##SUF a, pb2##SUF b) { pb2##SUF r = {a.x + b.x, a.y + b.y}; return r; }          \
    static pb2##SUF pb2_mul##SUF(pb2##SUF a, T s) { pb2##SUF r = {a.x * s, a.y * s}; return r; }                    \
    static T pb2_big##SUF(pb2##SUF a) { return pb_max_##SUF(pb_abs_##SUF(a.x), pb_abs_##SUF(a.y)); }                   \
    static T pb2_cross##SUF(pb2##SUF a, pb2##SUF b) { return pb_dop##SUF(a.x, b.y, a.y, b.x); }                     \
    static T pb3_c##SUF(pb3##SUF p, unsigned k) { return k == 0 ? p.x : (k == 1 ? p.y : p.z); }                    \
    static pb3##SUF pb3_sub##SUF(pb3##SUF a, pb3##SUF b) { pb3##SUF r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; } \
    static pb3##SUF pb3_add##SUF(pb3##SUF a, pb3##SUF b) { pb3##SUF r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; } \
    static pb3##SUF pb3_mul##SUF(pb3##SUF a, T s) { pb3##SUF r = {a.x * s, a.y * s, a.z * s}; return r; }           \
    static pb2##SUF pb_project##SUF(pb3##SUF p, pb3##SUF w, unsigned kz)                                            \
    {                                                                                                               \
        const unsigned kx = (kz + 1) % 3, ky = (kz + 2) % 3;                                                        \
        const T z = pb3_c##SUF(w, kz);                                                                              \
        pb2##SUF r = {pb_dop##SUF(z, pb3_c##SUF(p, kx), pb3_c##SUF(w, kx), pb3_c##SUF(p, kz)),                       \
                      pb_dop##SUF(z, pb3_c##SUF(p, ky), pb3_c##SUF(w, ky), pb3_c##SUF(p, kz))};                      \
        return r;                                                                                                   \
    }                                                                                                               \
    static int pb_solve##SUF(const pf3* corner, pf3 dir, pbhits* out)                                               \
    {                                                                                                               \
        int retry = 0;                                                                                              \
        memset(out, 0, sizeof *out);                                                                                \
        const pb3##SUF w = {(T)dir.x, (T)dir.y, (T)dir.z};                                                          \
        unsigned kz = 0;                                                                                            \
        if (pb_abs_##SUF(w.y) > pb_abs_##SUF(w.x)) kz = 1;                                                            \
        if (pb_abs_##SUF(w.z) > pb_abs_##SUF(pb3_c##SUF(w, kz))) kz = 2;                                              \
        const pb3##SUF p0 = {(T)corner[0].x, (T)corner[0].y, (T)corner[0].z};                                       \
        const pb3##SUF p1 = {(T)corner[1].x, (T)corner[1].y, (T)corner[1].z};                                       \
        const pb3##SUF p2 = {(T)corner[2].x, (T)corner[2].y, (T)corner[2].z};                                       \
        const pb3##SUF p3 = {(T)corner[3].x, (T)corner[3].y, (T)corner[3].z};                                       \
        const pb3##SUF eu = pb3_sub##SUF(p1, p0), ev = pb3_sub##SUF(p2, p0);                                        \
        const pb3##SUF tw = pb3_sub##SUF(pb3_sub##SUF(p3, p2), eu);                                                 \
        pb2##SUF a = pb_project##SUF(p0, w, kz), b = pb_project##SUF(eu, w, kz);                                    \
        pb2##SUF c = pb_project##SUF(ev, w, kz), d = pb_project##SUF(tw, w, kz);                                    \
        const T scale = pb_max_##SUF(pb_max_##SUF(pb2_big##SUF(a), pb2_big##SUF(b)),                                  \
                                    pb_max_##SUF(pb2_big##SUF(c), pb2_big##SUF(d)));                                 \
        if (!(scale > (T)0)) return 1;                                                                              \
        a = pb2_mul##SUF(a, (T)1 / scale); b = pb2_mul##SUF(b, (T)1 / scale);                                       \
        c = pb2_mul##SUF(c, (T)1 / scale); d = pb2_mul##SUF(d, (T)1 / scale);                                       \
        const T eps = EPS;                                                                                          \
        const pb2##SUF cs[4] = {a, pb2_add##SUF(a, b), pb2_add##SUF(a, c),                                          \
                                pb2_add##SUF(pb2_add##SUF(pb2_add##SUF(a, b), c), d)};                              \
        T xlo = cs[0].x, xhi = xlo, ylo = cs[0].y, yhi = ylo;                                                       \
        for (unsigned i = 1; i < 4; ++i) {                                                                          \
            xlo = xlo < cs[i].x ? xlo : cs[i].x;                                                                    \
            xhi = pb_max_##SUF(xhi, cs[i].x);                                                                        \
            ylo = ylo < cs[i].y ? ylo : cs[i].y;                                                                    \
            yhi = pb_max_##SUF(yhi, cs[i].y);                                                                        \
        }                                                                                                           \
        const T guard = (T)64 * eps;                                                                                \
        if (xlo > guard || xhi < -guard || ylo > guard || yhi < -guard) return 0;                                   \
        const T A = pb2_cross##SUF(b, d), B = pb2_cross##SUF(a, d) + pb2_cross##SUF(b, c), Cc = pb2_cross##SUF(a, c); \
        const T mag = pb_max_##SUF(pb_abs_##SUF(A), pb_max_##SUF(pb_abs_##SUF(B), pb_abs_##SUF(Cc)));                    \
        if (!(mag > (T)0)) return 1;                                                                                \
        const T qa = A / mag, qb = B / mag, qc = Cc / mag;                                                          \
        if (IS_FLOAT && A != (T)0 && pb_abs_##SUF(qa) < (T)64 * eps) return 1;                                       \
        T roots[2] = {0, 0};                                                                                        \
        unsigned nroot = 0;                                                                                         \
        int repeated = 0;                                                                                           \
        if (A == (T)0) {                                                                                            \
            if (B == (T)0) return pb_abs_##SUF(qc) <= guard;                                                         \
            roots[nroot++] = -qc / qb;                                                                              \
        } else {                                                                                                    \
            const T disc = pb_dop##SUF(qb, qb, (T)4 * qa, qc);                                                      \
            const T err = (T)64 * eps * (qb * qb + pb_abs_##SUF((T)4 * qa * qc));                                    \
            if (disc < (T)0) return disc >= -err;                                                                   \
            if (disc == (T)0) {                                                                                     \
                if (IS_FLOAT) return 1;                                                                             \
                roots[nroot++] = -qb / ((T)2 * qa);                                                                 \
                repeated = 1;                                                                                       \
            } else {                                                                                                \
                if (disc <= err) return 1;                                                                          \
                const T q = -(T)0.5 * (qb + COPYSIGN(SQRT(disc), qb));                                              \
                roots[0] = q / qa;                                                                                  \
                roots[1] = qc / q;                                                                                  \
                if (roots[1] < roots[0]) { const T tmp = roots[0]; roots[0] = roots[1]; roots[1] = tmp; }           \
                nroot = 2;                                                                                          \
            }                                                                                                       \
        }                                                                                                           \
        for (unsigned r = 0; r < nroot; ++r) {                                                                      \
            T u = roots[r];                                                                                         \
            if (!(u == u)) { retry = 1; continue; }                                                                 \
            if (u < -guard || u > (T)1 + guard) continue;                                                           \
            const pb2##SUF num = pb2_add##SUF(a, pb2_mul##SUF(b, u)), den = pb2_add##SUF(c, pb2_mul##SUF(d, u));    \
            if (pb2_big##SUF(den) <= guard) { retry = 1; continue; }                                                \
            T v = pb_abs_##SUF(den.x) >= pb_abs_##SUF(den.y) ? -num.x / den.x : -num.y / den.y;                       \
            if (!(v == v)) { retry = 1; continue; }                                                                 \
            if (v < -guard || v > (T)1 + guard) continue;                                                           \
            T cond = (T)1;                                                                                          \
            for (unsigned it = 0; it < 3; ++it) {                                                                   \
                const pb2##SUF fu = pb2_add##SUF(b, pb2_mul##SUF(d, v)), fv = pb2_add##SUF(c, pb2_mul##SUF(d, u));  \
                const T det = pb2_cross##SUF(fu, fv);                                                               \
                const pb2##SUF res = pb2_add##SUF(pb2_add##SUF(pb2_add##SUF(a, pb2_mul##SUF(b, u)),                 \
                                                               pb2_mul##SUF(c, v)), pb2_mul##SUF(d, u * v));        \
                if (pb_abs_##SUF(det) <= (T)64 * eps * pb2_big##SUF(fu) * pb2_big##SUF(fv)) {                        \
                    if (!repeated) retry = 1;                                                                       \
                    break;                                                                                          \
                }                                                                                                   \
                cond = pb_max_##SUF((T)1, pb_max_##SUF(pb2_big##SUF(fu), pb2_big##SUF(fv)) / pb_abs_##SUF(det));       \
                const T du = pb2_cross##SUF(res, fv) / det, dv = pb2_cross##SUF(fu, res) / det;                     \
                u -= du;                                                                                            \
                v -= dv;                                                                                            \
            }                                                                                                       \
            const T perr = (T)32 * eps * cond;                                                                      \
            if (IS_FLOAT && (perr > (T)2e-5 || u <= perr || u >= (T)1 - perr || v <= perr || v >= (T)1 - perr)) {   \
                retry = 1;                                                                                          \
                continue;                                                                                           \
            }                                                                                                       \
            if (perr > (T)1e-5 && !repeated) { retry = 1; continue; }                                               \
            if (u < -perr || u > (T)1 + perr || v < -perr || v > (T)1 + perr) continue;                             \
            const int boundary = u <= perr || u >= (T)1 - perr || v <= perr || v >= (T)1 - perr;                    \
            if (u < (T)0 || u > (T)1) u = u < (T)0 ? (T)0 : (T)1;                                                   \
            if (v < (T)0 || v > (T)1) v = v < (T)0 ? (T)0 : (T)1;                                                   \
            const pb2##SUF res = pb2_add##SUF(pb2_add##SUF(pb2_add##SUF(a, pb2_mul##SUF(b, u)), pb2_mul##SUF(c, v)), \
                                              pb2_mul##SUF(d, u * v));                                              \
            if (pb2_big##SUF(res) > (T)256 * eps) { retry = 1; continue; }                                          \
            const pb3##SUF lower = pb3_add##SUF(pb3_mul##SUF(p0, (T)1 - u), pb3_mul##SUF(p1, u));                   \
            const pb3##SUF upper = pb3_add##SUF(pb3_mul##SUF(p2, (T)1 - u), pb3_mul##SUF(p3, u));                   \
            const pb3##SUF point = pb3_add##SUF(pb3_mul##SUF(lower, (T)1 - v), pb3_mul##SUF(upper, v));             \
            const T t = pb3_c##SUF(point, kz) / pb3_c##SUF(w, kz);                                                  \
            if (!(t > (T)0)) {                                                                                      \
                if (pb_abs_##SUF(t) <= (T)64 * eps) retry = 1;                                                       \
                continue;                                                                                           \
            }                                                                                                       \
            pbhit hit = {(float)u, (float)v, (float)t, 0.0f, 0};                                                    \
            if (boundary) hit.flags |= BH_BOUNDARY;                                                                 \
            if (repeated) hit.flags |= BH_SINGULAR;                                                                 \
            if (!IS_FLOAT) hit.flags |= BH_FP64;                                                                    \
            const pf3 e3 = f3_sub(pb_eval(corner, hit.u, hit.v), f3_scale(dir, hit.t));                             \
            hit.residual = pb_max_f(pb_abs_f(e3.x), pb_max_f(pb_abs_f(e3.y), pb_abs_f(e3.z)));                             \
            if (!(hit.residual <= 0x1p-21f && hit.t < 4.0f)) { retry = 1; continue; }                               \
            if (out->count < 2) out->hits[out->count++] = hit;                                                      \
            else retry = 1;                                                                                         \
        }                                                                                                           \
        return retry;                                                                                               \
    }

/* |x| and max are the reference's x < 0 ? -x : x and a > b ? a : b, not fabsf / fmaxf (the sign
 * of a zero and the NaN rule differ); the float instances serve the residual. */
static float pb_abs_f(float x);
static float pb_max_f(float a, float b);
/* BilinearPatchGeometry::evaluate in binary32 */
static pf3 pb_eval(const pf3* c, float u, float v)
{
    const pf3 lower = f3_add(f3_scale(c[0], 1.0f - u), f3_scale(c[1], u));
    const pf3 upper = f3_add(f3_scale(c[2], 1.0f - u), f3_scale(c[3], u));
    return f3_add(f3_scale(lower, 1.0f - v), f3_scale(upper, v));
}
PB_SOLVER(float, f, fmaf, sqrtf, copysignf, 0x1p-23f, 1)
PB_SOLVER(double, d, fma, sqrt, copysign, 0x1p-52, 0)

void icpo_bilinear_intersect(const float* corners /* 12 */, const float* direction /* 3 */, void* out /* pbhits */)
{
    pbhits* r = (pbhits*)out;
    memset(r, 0, sizeof *r);
    const pf3 dir = {direction[0], direction[1], direction[2]};
    pf3 c[4];
    for (unsigned i = 0; i < 4; ++i) {
        c[i].x = corners[3 * i];
        c[i].y = corners[3 * i + 1];
        c[i].z = corners[3 * i + 2];
    }
    const float n2 = f3_dot(dir, dir);
    if (!f3_fin(dir) || !(n2 > 0.99f && n2 < 1.01f)) {
        r->flags = BQ_INVALID;
        return;
    }
    for (unsigned i = 0; i < 4; ++i)
        if (!f3_fin(c[i]) || !(f3_dot(c[i], c[i]) <= 4.0f)) {
            r->flags = BQ_INVALID;
            return;
        }
    if (pb_solvef(c, dir, r)) {
        const int unresolved = pb_solved(c, dir, r);
        r->flags |= BQ_FP64;
        if (unresolved) r->flags |= BQ_UNRESOLVED;
    }
    if (r->count == 2) {
        pbhit* a = &r->hits[0];
        pbhit* b = &r->hits[1];
        if (b->u < a->u || (b->u == a->u && b->v < a->v)) {
            const pbhit t = *a;
            *a = *b;
            *b = t;
        }
    }
}

/* --------------------------------------------------------------- all-hit patch query
 * Restates the reference's per-direction query (shaders/entry/patch_query.cu: raygen,
 * intersection and any-hit programs; PatchHitCollector, include/rainbow/patch_query_data.hpp
 * :43-128): every patch whose padded box the ray t d (0 <= t <= 4) meets is intersected, its
 * roots collected, then sorted by (patch_id, compact index, root), duplicates removed and the
 * summary counted.  The box test is a plain binary32 slab test (the reference leaves it to the
 * OptiX traversal); the oracle tests every patch, the device bins them by direction first. */
typedef struct { uint32_t compact, patch_id, root, flags; float u, v, t, residual; } pqhit;
enum { PQ_UNRESOLVED = 1, PQ_INVALID = 2, PQ_MISMATCH = 4, PQ_REFINE = 8, PQ_BOUNDARY = 16, PQ_FP64 = 32,
       PQ_DUPLICATE = 64, PQ_SINGULAR = 128, PQ_OVERFLOW = 256 };

int icpo_ray_box(const float* dir, const paabb* b)
{
    const float lo[3] = {b->min_x, b->min_y, b->min_z}, hi[3] = {b->max_x, b->max_y, b->max_z};
    float tnear = 0.0f, tfar = 4.0f;
    for (unsigned a = 0; a < 3; ++a) {
        if (dir[a] == 0.0f) {
            if (lo[a] > 0.0f || hi[a] < 0.0f) return 0;
            continue;
        }
        const float t1 = lo[a] / dir[a], t2 = hi[a] / dir[a];
        const float tmin = t1 < t2 ? t1 : t2, tmax = t1 < t2 ? t2 : t1;
        if (tmin > tnear) tnear = tmin;
        if (tmax < tfar) tfar = tmax;
    }
    return tnear <= tfar;
}
static int pq_less(const pqhit* a, const pqhit* b)
{
    if (a->patch_id != b->patch_id) return a->patch_id < b->patch_id;
    if (a->compact != b->compact) return a->compact < b->compact;
    return a->root < b->root;
}
/* One direction: hits into out[capacity] (pass 2) or only counted (out == NULL, pass 1). */
static void pq_direction(const pvertex* vertices, uint32_t vertex_count, const ppatch* patches, const paabb* boxes,
                         uint32_t patch_count, const float* dir, pqhit* out, uint32_t capacity, psummary* sm)
{
    uint32_t count = 0, flags = 0, first = 0xffffffffu;
    const float n2 = fmaf(dir[0], dir[0], fmaf(dir[1], dir[1], dir[2] * dir[2]));
    const int finite_dir = dir[0] >= -0x1.fffffep127f && dir[0] <= 0x1.fffffep127f && dir[1] >= -0x1.fffffep127f &&
                           dir[1] <= 0x1.fffffep127f && dir[2] >= -0x1.fffffep127f && dir[2] <= 0x1.fffffep127f;
    if (!finite_dir || !(n2 > 0.99f && n2 < 1.01f))
        flags |= PQ_INVALID;
    else
        for (uint32_t k = 0; k < patch_count; ++k) {
            if (!icpo_ray_box(dir, boxes + k)) continue;
            const ppatch* p = patches + k;
            float corners[12];
            int bad = 0;
            for (unsigned i = 0; i < 4 && !bad; ++i) {
                if (p->v[i] >= vertex_count) { bad = 1; break; }
                const pf3 c = vertices[p->v[i]].direction;
                corners[3 * i] = c.x; corners[3 * i + 1] = c.y; corners[3 * i + 2] = c.z;
            }
            if (bad) { flags |= PQ_INVALID; continue; }
            pbhits h;
            icpo_bilinear_intersect(corners, dir, &h);
            if ((h.flags & (BQ_UNRESOLVED | BQ_INVALID)) && p->patch_id < first) first = p->patch_id;
            if (h.flags & BQ_UNRESOLVED) flags |= PQ_UNRESOLVED;
            if (h.flags & BQ_INVALID) flags |= PQ_INVALID;
            if (h.flags & BQ_FP64) flags |= PQ_FP64;
            for (uint32_t r = 0; r < h.count; ++r) {
                if (out) {
                    if (count >= capacity) flags |= PQ_MISMATCH;
                    else {
                        pqhit x = {k, p->patch_id, r, h.hits[r].flags, h.hits[r].u, h.hits[r].v, h.hits[r].t,
                                   h.hits[r].residual};
                        out[count] = x;
                    }
                }
                ++count;
            }
        }
    memset(sm, 0, sizeof *sm);
    if (!out) { /* count pass */
        sm->candidates = count;
        sm->flags = flags;
        sm->first_problem = first;
        return;
    }
    sm->candidates = capacity;
    if (count != capacity) flags |= PQ_MISMATCH;
    sm->flags = flags;
    sm->first_problem = first;
    if (count > capacity) return;
    for (uint32_t i = 1; i < count; ++i) { /* insertion sort: stable, as the reference */
        const pqhit x = out[i];
        uint32_t j = i;
        while (j != 0 && pq_less(&x, out + j - 1)) { out[j] = out[j - 1]; --j; }
        out[j] = x;
    }
    uint32_t kept = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const pqhit h = out[i];
        if (kept != 0 && h.compact == out[kept - 1].compact && h.root == out[kept - 1].root) {
            sm->flags |= PQ_DUPLICATE;
            continue;
        }
        if (h.compact >= patch_count) { sm->flags |= PQ_INVALID; continue; }
        out[kept++] = h;
        const uint32_t st = patches[h.compact].status;
        if (st == 3u) { ++sm->refinement; sm->flags |= PQ_REFINE; }
        else if (st == 1u || st == 2u) ++sm->regular;
        else sm->flags |= PQ_INVALID;
        if (h.flags & BH_BOUNDARY) { ++sm->boundary; sm->flags |= PQ_BOUNDARY; }
        if (h.flags & BH_SINGULAR) sm->flags |= PQ_SINGULAR;
    }
    sm->hits = kept;
}
/* Both passes over all directions: offsets[n + 1], summaries[n]; hits written when
 * hits != NULL (capacity offsets[n]).  Returns the total candidate count. */
uint64_t icpo_patch_query(const pvertex* vertices, uint32_t vertex_count, const ppatch* patches, const paabb* boxes,
                          uint32_t patch_count, const float* directions, uint32_t n, uint64_t* offsets,
                          psummary* summaries, pqhit* hits)
{
    offsets[0] = 0;
    for (uint32_t i = 0; i < n; ++i) {
        pq_direction(vertices, vertex_count, patches, boxes, patch_count, directions + 3 * i, NULL, 0, summaries + i);
        offsets[i + 1] = offsets[i] + summaries[i].candidates;
    }
    if (hits)
        for (uint32_t i = 0; i < n; ++i)
            pq_direction(vertices, vertex_count, patches, boxes, patch_count, directions + 3 * i, hits + offsets[i],
                         (uint32_t)(offsets[i + 1] - offsets[i]), summaries + i);
    return offsets[n];
}
