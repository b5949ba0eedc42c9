"""Drop path on the CPU: the oracle restatement and the product's host inputs, pinned to the
reference's own outputs (tests/golden/drop_reference.npz, made by make_golden.py from the
reference's header-only drop tracer, src/projected_area.cpp and src/water_refractive_index.cpp)
and to closed-form sphere results.

Reference tests followed: tests/test_raindrop_cpu.cpp:11-30 (five radii, lattice traces against
independent intersectors), tests/raindrop_validation.hpp:134-199 (sphere deflection, Fresnel
powers), tests/test_water_optics_cpu.cpp, tests/test_projected_area_cpu.cpp:40-57.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle as oracle_mod

G = np.load(GOLDEN / "drop_reference.npz")


# ------------------------------------------------------------------ host inputs (product)
def _frame_from_reference(kf, ef):
    # apps/generate_phase.cpp:242-245: promote, normalise k, orthogonalise e0, e1 = k x e0
    k = np.array(kf, dtype=np.float64)
    k = k / math.sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2])
    e = np.array(ef, dtype=np.float64)
    d = e[0] * k[0] + e[1] * k[1] + e[2] * k[2]
    e = e - d * k
    e = e / math.sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2])
    e1 = np.array([k[1] * e[2] - k[2] * e[1], k[2] * e[0] - k[0] * e[2], k[0] * e[1] - k[1] * e[0]])
    return k, e, e1


def test_drop_frame_matches_reference(icp, oracle):
    for alpha, row in zip(G["frame_alpha"], G["frame"]):
        k, e0, e1 = _frame_from_reference(row[:3], row[3:])
        pk, pe0, pe1 = icp.drop_frame(float(alpha))
        assert np.array_equal(pk, k) and np.array_equal(pe0, e0) and np.array_equal(pe1, e1), alpha
        ok, oe0, oe1 = oracle.drop_frame(float(alpha))
        assert np.array_equal(ok, k) and np.array_equal(oe0, e0) and np.array_equal(oe1, e1), alpha


def test_drop_shape_matches_reference(icp):
    for r, row in zip(G["shape_radius"], G["shape"]):
        s = icp.RaindropShape.make(float(np.float32(r)))
        assert s.coefficients == list(row[:8]), r
        assert (s.inner_radius, s.outer_radius) == (row[8], row[9]), r
    sphere = icp.RaindropShape.make(2.0, sphere=True)
    assert sphere.coefficients == [0.0] * 8
    for bad in (0.0, -1.0, 3.0001, float("nan")):
        with pytest.raises(icp.InvalidArgument):
            icp.RaindropShape.make(bad)


def test_water_index_matches_reference(icp):
    # IAPWS-95 liquid density (all 56 residual terms, the reference's bisection) and R9-97 index:
    # bit for bit the reference's evaluate_water_optics on its golden grid
    for (lam, t, p), (n_ref, rho_ref) in zip(G["water_in"], G["water"]):
        w = icp.evaluate_water_optics(lam, t, p)
        assert w.refractive_index == n_ref, (lam, t, p)
        assert w.density_kg_m3 == rho_ref, (lam, t, p)
    for bad in ((150.0, 20.0, 101325.0), (700.0, -1.0, 101325.0), (700.0, 61.0, 101325.0), (700.0, 20.0, 1e9)):
        with pytest.raises(icp.InvalidArgument):
            icp.evaluate_water_optics(*bad)


@pytest.mark.skipif(not oracle_mod.ref_drop_available(), reason="reference drop harness not built")
def test_water_index_matches_reference_on_random_states(icp):
    # seeded states over the whole domain (200-1100 nm, 0-60 C, 50 kPa-100 MPa) through the
    # reference's own evaluate_water_optics compiled here
    rng = np.random.default_rng(20261204)
    ins = [(float(lam), float(t), float(p)) for lam, t, p in
           zip(rng.uniform(200, 1100, 300), rng.uniform(0, 60, 300), np.exp(rng.uniform(np.log(5e4), np.log(1e8), 300)))]
    ref = oracle_mod.ref_drop_lines("water_state", [f"{lam!r} {t!r} {p!r}" for lam, t, p in ins])
    for (lam, t, p), (n_ref, rho_ref, res_ref, width_ref) in zip(ins, ref):
        w = icp.evaluate_water_optics(lam, t, p)
        assert (w.refractive_index, w.density_kg_m3) == (n_ref, rho_ref), (lam, t, p)
        # the residual and bracket width metadata.json reports (rainbow::WaterOptics)
        assert (w.density_pressure_residual_pascal, w.density_bracket_width_kg_m3) == (res_ref, width_ref), (lam, t, p)


def test_projected_area_matches_reference(icp):
    for row, a_ref in zip(G["area_in"], G["area"]):
        a = icp.compute_projected_area(row[:8], row[8], row[9:12])
        assert abs(a / a_ref - 1) <= 1e-10, row
    assert icp.compute_projected_area([0.0] * 8, 0.4, (1, 0, 0)) == math.pi * 0.4 * 0.4
    with pytest.raises(icp.InvalidArgument):  # strongly nonconvex: rejected, no hull substitute
        icp.compute_projected_area([0, 0, 0.5, 0, 0, 0, 0, 0], 1.0, (1, 0, 0))


def test_diffraction_rows_match_independent_evaluation(icp):
    from scipy.special import j0, j1

    edges = icp.u_edges(180)
    for area, lam in ((7.07, 550.0), (0.01, 700.0), (1e-5, 400.0)):
        rows = icp.diffraction_rows(edges, area, lam)
        x = 2 * math.pi * math.sqrt(area / math.pi) / (lam * 1e-6)
        u = np.minimum(edges, 0.5)
        z = x * 2 * np.sqrt(u * (1 - u))
        enc = 1 - j0(z) ** 2 - j1(z) ** 2
        expect = area * np.diff(enc) / enc[-1]
        assert np.abs(rows - expect).max() <= 1e-12 * area
        assert abs(rows.sum() - area) <= 1e-12 * area
        assert np.all(rows[90:] == 0)


# ------------------------------------------------------------------ oracle vs reference tracer
@pytest.mark.parametrize("case", range(3))
def test_oracle_four_families_match_reference(oracle, case):
    """R, TT, TRT, TRRT from every lattice vertex of RaindropPathTracer (FP32 Jones) against the
    oracle's FP64 flux chain from the same origin: same statuses, directions within the binary32
    tracer's error, flux powers within 2e-4."""
    r, sphere, n, kx, ky, kz, grid = G["family_cases"][case]
    geom = G[f"families{case}_geom"].astype(np.float64)
    power = G[f"families{case}_power"]
    row = G["shape"][list(G["shape_radius"]).index(r)] if not sphere else np.zeros(10)
    geo = oracle.drop_geometry(row[:8], r)
    checked = 0
    for v in range(geom.shape[0]):
        o, w, e0 = geom[v, 0:3], geom[v, 3:6], geom[v, 6:9]
        w = w / np.linalg.norm(w)
        e0 = e0 - w * np.dot(w, e0)
        e0 /= np.linalg.norm(e0)
        info, ex = oracle.drop_trace_from(geo, o, w, e0, n, max_hits=3)
        fam = {int(e[4]): e for e in ex}
        for f in range(4):
            st = geom[v, 9 + 7 * f]
            if st == 2:  # Miss
                assert info[6] == 1, (v, f)
                continue
            if st == 3:  # total internal reflection: no transmitted exit
                assert f not in fam, (v, f)
                continue
            assert st == 1, (v, f, st)
            mine = fam[f]
            d_ref = geom[v, 10 + 7 * f:13 + 7 * f]
            assert np.abs(mine[:3] - d_ref).max() <= 5e-5, (v, f)
            assert abs(mine[3] - power[v, f]) <= 2e-4, (v, f)
            checked += 1
    assert checked > geom.shape[0]  # misses and TIR take the rest of the 4 x lattice slots


def test_oracle_sphere_deflection_and_fresnel(oracle):
    """Closed form for a sphere (raindrop_validation.hpp:134-199 generalised to every order):
    order p >= 1 leaves after p chords, deviated by D_p = 2(i - r) + (p - 1)(pi - 2r), with
    power 0.5 sum_{s,p} (1-R)^2 R^(p-1); the entry reflection carries 0.5 (Rs + Rp)."""
    n = 1.3330
    geo = oracle.drop_geometry(np.zeros(8), 1.0)
    k = np.array([1.0, 0.0, 0.0])
    e0 = np.array([0.0, 0.0, 1.0])
    rng = np.random.default_rng(7)
    for b in list(rng.uniform(0.01, 0.999, 60)) + [0.5, 0.861, 0.95]:
        phi = rng.uniform(0, 2 * math.pi)
        o = np.array([-3.0, b * math.cos(phi), b * math.sin(phi)])
        info, ex = oracle.drop_trace_from(geo, o, k, e0, n, max_hits=8, max_out=16)
        i = math.asin(b)
        r = math.asin(b / n)
        ci, ct = math.cos(i), math.cos(r)
        rs = ((ci - n * ct) / (ci + n * ct)) ** 2
        rp = ((n * ci - ct) / (n * ci + ct)) ** 2
        for e in ex:
            p = int(e[4])
            d = e[:3]
            if p == 0:
                dev = math.pi - 2 * i
                pw = 0.5 * (rs + rp)
            else:
                dev = 2 * (i - r) + (p - 1) * (math.pi - 2 * r)
                pw = 0.5 * ((1 - rs) ** 2 * rs ** (p - 1) + (1 - rp) ** 2 * rp ** (p - 1))
            cos_dev = math.cos(dev)
            assert abs(float(np.dot(d, k)) - cos_dev) <= 1e-12, (b, p)
            assert abs(e[3] - pw) <= 1e-13 + 1e-12 * pw, (b, p)
        assert info[0] in (0, 1, 2) and abs(info[2] + info[3] - 1) <= 1e-13


def test_oracle_drop_record_energy_and_area(oracle, icp):
    """escaped + residual = incident hit area; the hit fraction of the sampling disk estimates the
    CPU projected area (Monte Carlo, 5 sigma); the transparent limit puts every ray forward."""
    sh = icp.RaindropShape.make(1.5)
    geo = oracle.drop_geometry(sh.coefficients, 1.5)
    frame = np.array(icp.drop_frame(20.0))
    rec = oracle.drop_record(geo, frame, 1.3318, 36, 72, 20000, 99, max_hits=10)
    assert abs((rec.escaped_area + rec.unresolved_area) / rec.incident_area - 1) <= 1e-12
    assert rec.max_balance <= 1e-12
    area = icp.compute_projected_area(sh.coefficients, 1.5, frame[0])
    pr = area / geo.disk_area_mm2
    sigma = geo.disk_area_mm2 * math.sqrt(pr * (1 - pr) / 20000)
    assert abs(rec.incident_area - area) <= 5 * sigma
    assert rec.counts["rays"] == 20000 and rec.counts["missed"] > 0
    # a pure sphere sampled on its own disk: no misses; n = 1: straight through, all forward
    sph = oracle.drop_geometry(np.zeros(8), 0.3)
    t = oracle.drop_record(sph, frame, 1.0, 36, 72, 3000, 5, tail=0.0)
    assert t.counts["missed"] == 0
    assert abs(t.forward / t.incident_area - 1) <= 1e-12
    assert abs(t.incident_area - math.pi * 0.09) <= 1e-15


def test_oracle_intersections_are_surface_points(oracle, icp):
    sh = icp.RaindropShape.make(2.5)
    geo = oracle.drop_geometry(sh.coefficients, 2.5)
    rng = np.random.default_rng(3)
    c = np.array(sh.coefficients)

    def radius(mu):
        t = np.polynomial.chebyshev.chebval(mu, c)
        return 1 + t

    hits = 0
    for _ in range(300):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        o = -3 * d + 0.9 * np.cross(d, rng.normal(size=3))
        h = oracle.drop_intersect(geo, o, d, False)
        if not h[0]:
            continue
        hits += 1
        p = h[2:5]
        rr = np.linalg.norm(p)
        assert abs(rr - radius(-p[1] / rr)) <= 1e-13
        assert float(np.dot(h[5:8], d)) < 0
        inward = 0.7 * d - 0.3 * h[5:8]
        x = oracle.drop_intersect(geo, p, inward / np.linalg.norm(inward), True)
        q = x[2:5]
        assert abs(np.linalg.norm(q) - radius(-q[1] / np.linalg.norm(q))) <= 1e-13
    assert hits > 100
