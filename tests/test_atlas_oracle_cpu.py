"""Deterministic atlas composition, CPU: the library's orientation rule equals the reference's
bit for bit, and the oracle (oracle/atlas_oracle.py, written in the device kernel's operation
order and fixed-point accumulation) reproduces the reference's coupling weights, composed
masses and CDFs (tests/golden/atlas_reference.npz, from hex_atlas/python/atlas_math.py on a
traced reference atlas)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import atlas_oracle as AO

RULES = [
    {"quadrature": {"azimuth": 8, "tilt": 4, "spin": 3},
     "components": [{"kind": "horizontal_gaussian", "sigma_deg": 10, "fraction": 0.9},
                    {"kind": "isotropic", "fraction": 0.1}]},
    {"quadrature": {"azimuth": 3, "tilt": 5, "spin": 2},
     "components": [{"kind": "fixed", "fraction": 0.4,
                     "quaternion_wxyz": [0.9238795325112867, 0.0, 0.3826834323650898, 0.0]},
                    {"kind": "isotropic", "fraction": 0.6}]},
]


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN / "atlas_reference.npz")


@pytest.fixture(scope="module")
def atlas(gold):
    case = gold["nodes1_case"]
    T, P = int(case[5]), int(case[6])
    head = gold["nodes1_head"].reshape(T + 1, P + 1, 16)
    return {"R": case[0], "L": case[1], "T": T, "P": P, "area": head[:, :, 8], "residual": head[:, :, 10],
            "mass": gold["nodes1_mass"]}


def test_orientation_rule_matches_reference(gold):
    from ice_crystal_phase_b200 import atlas as A

    for ri, rule in enumerate(RULES):
        r, w, meta = A.orientation_rule(rule)
        assert np.array_equal(r, gold[f"rule{ri}_rotations"]) and np.array_equal(w, gold[f"rule{ri}_weights"])
        assert meta["randomness"] is False and meta["component_nodes"][-1] == math.prod(rule["quadrature"].values())
    assert np.array_equal(A.gaussian_tilt_nodes(4, 10), gold["rule0_tilts"])
    # the reference's own checks of the rule (hex_atlas/tests/test_compose.py:37-62)
    for sigma in (.1, 3, 10, 90):
        b = A.gaussian_tilt_nodes(16, sigma)
        s = math.radians(sigma)
        e = math.erf(math.pi / (2 * math.sqrt(2) * s))
        c = np.array([(1 + math.erf((x - math.pi / 2) / (math.sqrt(2) * s)) / e) / 2 for x in b])
        assert np.allclose(c, (np.arange(16) + .5) / 16, atol=6e-14, rtol=0)
        assert np.allclose(b + b[::-1], math.pi, atol=2e-15, rtol=0)
    assert np.array_equal(A.gaussian_tilt_nodes(4, 0), [math.pi / 2] * 4)
    for sigma in (-1, float("nan")):
        with pytest.raises(ValueError):
            A.gaussian_tilt_nodes(10, sigma)
    with pytest.raises(ValueError):
        A.orientation_rule({"quadrature": {"azimuth": 2, "tilt": 2, "spin": 2},
                            "components": [{"kind": "isotropic", "fraction": .5}]})


def _oracle_coupling(atlas, gold, ri, ki):
    """coupling_for_rule in the oracle: the vertical-incidence orbit average per component."""
    from ice_crystal_phase_b200 import atlas as A

    rule = RULES[ri]
    k = AO.unit3(ki)
    vertical = k[0] == 0.0 and k[2] == 0.0
    eligible = [c["kind"] in ("isotropic", "horizontal_gaussian") for c in rule["components"]]
    args = (atlas["area"], atlas["T"], atlas["P"], 32, atlas["R"], atlas["L"])
    if not vertical or not any(eligible):
        return AO.coupling(*args, gold[f"rule{ri}_rotations"], gold[f"rule{ri}_weights"], ki)
    w = np.zeros(((atlas["T"] + 1) * (atlas["P"] + 1), 2, 32))
    areas = []
    for comp, analytic in zip(rule["components"], eligible):
        quad = dict(rule["quadrature"])
        if analytic:
            quad["azimuth"] = 1
        r1, w1, _ = A.orientation_rule({"quadrature": quad, "components": [dict(comp, fraction=1.0)]})
        _, a = AO.coupling(*args, r1, w1, ki, fraction=comp["fraction"], orbit=analytic, out=w)
        areas.append(comp["fraction"] * a)
    return w, math.fsum(areas)


@pytest.mark.parametrize("ri", [0, 1])
@pytest.mark.parametrize("ii", range(5))
def test_oracle_coupling_and_compose_match_reference(gold, atlas, ri, ii):
    ki = tuple(gold["compose_incidents"][ii])
    key = f"compose{ri}_{ii}"
    want_w = gold[key + "_coupling"].reshape(-1, 2, 32)
    w, area = _oracle_coupling(atlas, gold, ri, ki)
    area_ref, residual_ref = gold[key + "_scalars"][:2]
    assert abs(area / area_ref - 1) < 1e-13
    # weights: same nonzero pattern, values to a few ulps of the largest weight of the row
    scale = np.abs(want_w).max()
    assert np.max(np.abs(w - want_w)) <= 1e-13 * scale
    # composition of the reference's own weights is bit-exact (same order, separate roundings)
    nodes = atlas["mass"].reshape(-1, 16, 32)
    mass = AO.compose(nodes, want_w)
    assert np.array_equal(mass, gold[key + "_mass"])
    # and of the oracle's weights within the weights' tolerance
    mass2 = AO.compose(nodes, w)
    assert np.max(np.abs(mass2 - mass)) <= 1e-12 * mass.max()
    residual = float(np.sum(np.sum(want_w, axis=(1, 2)) * atlas["residual"].reshape(-1)))
    assert residual == pytest.approx(residual_ref, rel=1e-12, abs=1e-30)
    # conservation: composed flux + residual = expected area (compose_atlas.py:171-173)
    assert abs((math.fsum(mass.flat) + residual) / area_ref - 1) < 2e-10
    a, b, rep = AO.make_cdf(mass, gold["compose_edges"])
    assert np.allclose(a, gold[key + "_phi"], rtol=0, atol=1e-15)
    assert np.allclose(b, gold[key + "_theta"], rtol=0, atol=1e-15)
    assert rep["g"] == pytest.approx(gold[key + "_scalars"][2], abs=1e-14)


def test_oracle_fold_covers_the_sphere():
    """Every direction folds into t in [0, pi/2], p in [0, pi/6] with q k(t,p) = direction
    (hex_atlas/tests/test_compose.py:24-30)."""
    for theta in np.linspace(0, math.pi, 21):
        for phi in np.linspace(0, 2 * math.pi, 43):
            k = [math.sin(theta) * math.cos(phi), math.cos(theta), math.sin(theta) * math.sin(phi)]
            b = AO.unit3(k)
            t, p, c, s, sy, sz, _ = AO.fold(b)
            assert 0 <= t <= math.pi / 2 and 0 <= p <= math.pi / 6
            kc = (math.sin(t) * math.cos(p), math.cos(t), math.sin(t) * math.sin(p))
            qk = (c * kc[0] + s * sz * kc[2], sy * kc[1], -s * kc[0] + c * sz * kc[2])
            assert np.allclose(qk, b, atol=2e-14)


def test_composed_record_meets_the_reader_contract(gold, tmp_path):
    """A record written with atlas.record_metadata around the reference's composed masses and the
    oracle's CDF passes the record reader's checks (python/rainbow_dataset/record.py:19-158)."""
    import json
    from types import SimpleNamespace

    from record_check import validate_record
    from ice_crystal_phase_b200 import atlas as A

    key = "compose0_1"
    mass = gold[key + "_mass"]
    edges = gold["compose_edges"]
    a, b, rep = AO.make_cdf(mass, edges)
    frame = gold[key + "_frame"]
    stub = SimpleNamespace(meta={"material": {"wavelength_nm": 550.0, "interior_index": 1.31, "exterior_index": 1.0},
                                 "geometry": {"shape": "regular_hexagonal_prism", "circumradius_mm": .05,
                                              "full_length_mm": .2}},
                           hashes={}, it=6, ip=3, nt=16, np=32)
    area, residual = gold[key + "_scalars"][:2]
    meta = A.record_metadata(stub, float(area), float(residual),
                             {"g_stored": rep["g"], "cdf_mass": rep["cdf_mass"], "l1_error": rep["l1"],
                              "lost_mass": 0.0, "maximum_cell_error": 0.0}, frame, "0" * 64, {"config": RULES[0]},
                             {"inclination_deg": 30.0}, {"method": "original_fixed_orientation_quadrature"}, "rainbow",
                             float(mass.sum()))
    d = tmp_path / "rec"
    d.mkdir()
    (d / "metadata.json").write_text(json.dumps(meta))
    np.save(d / "phi_cdf.npy", a)
    np.save(d / "theta_given_phi_cdf.npy", b)
    np.save(d / "u_edges.npy", edges)
    out = validate_record(d)
    assert out["metadata"]["incident_inclination_degrees"] == pytest.approx(30.0, abs=1e-12)


# ---------------------------------------------------------------- the reference's composition properties
def pattern_atlas():
    """The reference's synthetic atlas (hex_atlas/tests/test_compose.py:13-21): 6 x 3 incident
    intervals, 4 x 12 cells, every node the same normalised pattern times its projected area."""
    from ice_crystal_phase_b200 import atlas as A

    it, ip, nt, np_ = 6, 3, 4, 12
    area = np.zeros((it + 1, ip + 1))
    mass = np.zeros((it + 1, ip + 1, nt, np_))
    pattern = np.arange(1, nt * np_ + 1, dtype=float).reshape(nt, np_)
    pattern /= pattern.sum()
    for i in range(it + 1):
        for j in range(ip + 1):
            area[i, j] = A.projected_area(.1, .2, A.canonical_frame(i * math.pi / 2 / it, j * math.pi / 6 / ip)[:, 2])
            mass[i, j] = area[i, j] * pattern
    return dict(it=it, ip=ip, nt=nt, np=np_, area=area, mass=mass, residual=np.zeros_like(area), R=.1, L=.2)


def shift_cases():
    """Rotations that bring node (2, 1) to ki = (1, 0, 0) with its frame turned by a chosen number
    of phi cells, with and without a reflection (test_compose.py:76-94)."""
    from ice_crystal_phase_b200 import atlas as A

    f = A.canonical_frame(math.pi / 6, math.pi / 18)
    fw = np.column_stack(_frame_of([1.0, 0.0, 0.0]))
    for reflected in (False, True):
        q = np.diag([1., 1., -1.]) if reflected else np.eye(3)
        for shift in (0, 1, 2.3, -.7, 11.999):
            d = 2 * math.pi * shift / 12
            h = np.array([[math.cos(d), -math.sin(d), 0], [math.sin(d), math.cos(d), 0], [0, 0, 1.]])
            if reflected:
                h = h @ np.diag([1., -1., 1.])
            yield reflected, shift, fw @ h @ f.T @ q.T


def _frame_of(k):
    e0, e1, kk = AO.output_frame(k)
    return e0, e1, kk


def expected_shift(a, reflected, shift):
    original = a["mass"][2, 1]
    if reflected:
        original = original[:, ::-1]
    lower = math.floor(shift)
    fraction = shift - lower
    return (1 - fraction) * np.roll(original, lower, axis=1) + fraction * np.roll(original, lower + 1, axis=1)


def test_oracle_shift_and_reflection():
    a = pattern_atlas()
    for reflected, shift, r in shift_cases():
        w, expected = AO.coupling(a["area"], 6, 3, 12, .1, .2, np.array([r]), np.ones(1), [1, 0, 0])
        got = AO.compose(a["mass"].reshape(-1, 4, 12), w)
        assert np.allclose(got, expected_shift(a, reflected, shift), atol=3e-17, rtol=1e-12), (reflected, shift)
        assert got.sum() == pytest.approx(expected)


def test_oracle_area_weighted_mixture_and_residual():
    from ice_crystal_phase_b200 import atlas as A

    a = pattern_atlas()
    rot = np.array([np.eye(3), A._rz(np.array(math.pi / 2))])
    w, area = AO.coupling(a["area"], 6, 3, 12, .1, .2, rot, np.array([.25, .75]), [1, 0, 0])
    out = AO.compose(a["mass"].reshape(-1, 4, 12), w)
    exact = .25 * A.projected_area(.1, .2, [1, 0, 0]) + .75 * A.projected_area(.1, .2, [0, -1, 0])
    assert area == pytest.approx(exact) and out.sum() == pytest.approx(exact)
    # a retained tail is propagated, not renormalised away (test_compose.py:103-108)
    mass, residual = a["mass"] * .99, .01 * a["area"]
    r = A._ry(np.array(.213)) @ A._rz(np.array(.7))
    w, area = AO.coupling(a["area"], 6, 3, 12, .1, .2, np.array([r]), np.ones(1), [1, -.4, .3])
    m = AO.compose(mass.reshape(-1, 4, 12), w)
    tail = float(np.sum(w.sum(axis=(1, 2)) * residual.reshape(-1)))
    assert m.sum() / area == pytest.approx(.99) and tail / area == pytest.approx(.01)


def polar_rule(na=16):
    return {"quadrature": {"azimuth": na, "tilt": 4, "spin": 3},
            "components": [{"kind": "horizontal_gaussian", "sigma_deg": 10, "fraction": .9},
                           {"kind": "isotropic", "fraction": .1}]}


def oracle_vertical(a, rule, ki, mass):
    """The vertical-incidence orbit average through the oracle (per component: one azimuth node,
    row means), then the composition."""
    from ice_crystal_phase_b200 import atlas as A

    w = np.zeros(((a["it"] + 1) * (a["ip"] + 1), 2, a["np"]))
    areas = []
    for comp in rule["components"]:
        analytic = comp["kind"] in ("isotropic", "horizontal_gaussian")
        quad = dict(rule["quadrature"], azimuth=1) if analytic else rule["quadrature"]
        r1, w1, _ = A.orientation_rule({"quadrature": quad, "components": [dict(comp, fraction=1.0)]})
        _, ar = AO.coupling(a["area"], a["it"], a["ip"], a["np"], a["R"], a["L"], r1, w1, ki,
                            fraction=comp["fraction"], orbit=analytic, out=w)
        areas.append(comp["fraction"] * ar)
    return AO.compose(mass.reshape(-1, a["nt"], a["np"]), w), math.fsum(areas)


def test_oracle_poles_are_uniform_in_phi():
    """At exact vertical incidence the analytic azimuth average equals the phi mean of the discrete
    rule, row by row, at both poles; and it does not depend on the azimuth node count
    (hex_atlas/tests/test_polar_azimuth.py:34-69)."""
    from ice_crystal_phase_b200 import atlas as A

    a = pattern_atlas()
    mass = a["mass"] * .97
    for sign in (-1, 1):
        ki = [0, sign, 0]
        rot, w, _ = A.orientation_rule(polar_rule())
        wd, area_d = AO.coupling(a["area"], 6, 3, 12, .1, .2, rot, w, ki)
        old = AO.compose(mass.reshape(-1, 4, 12), wd)
        new, area = oracle_vertical(a, polar_rule(), ki, mass)
        assert np.allclose(new, np.repeat(old.mean(axis=1, keepdims=True), 12, axis=1), rtol=1e-12, atol=2e-17)
        assert area == pytest.approx(area_d, abs=1e-15)
        first, _ = oracle_vertical(a, polar_rule(1), ki, mass)
        for na in (2, 7, 23):
            assert np.array_equal(oracle_vertical(a, polar_rule(na), ki, mass)[0], first)


def test_oracle_atlas_nodes_match_reference_bit_for_bit(icp, gold):
    """The oracle's atlas node (C, the pinned prism tracer from given entries, per-ray Kahan
    columns reduced in ray order) equals the reference's trace_cpu on every node of both
    reference atlases, bit for bit."""
    from oracle import oracle as O

    for c in (0, 1):
        R, L, n, ne, _, T, P, nt, np_, S, hits, tail = gold[f"nodes{c}_case"]
        T, P, nt, np_, S = int(T), int(P), int(nt), int(np_), int(S)
        head, want = gold[f"nodes{c}_head"], gold[f"nodes{c}_mass"]
        for m in range((T + 1) * (P + 1)):
            i, j = divmod(m, P + 1)
            node = icp.atlas_incident_node(T, P, i, j)
            faces, pts, w = icp.atlas_area_rule(R, L, list(node.rule_ki), S)
            mass, st = O.atlas_node(R, L, n, list(node.ki), list(node.e0), list(node.e1), faces, pts, w, nt, np_,
                                    n_ext=ne, tail=tail, max_hits=int(hits))
            assert st[6] == -1 and st[2] == head[m, 12] and st[3] == head[m, 13]
            assert st[0] == head[m, 9] and st[1] == head[m, 10]
            assert np.array_equal(mass, want[i, j]), (c, i, j, np.abs(mass - want[i, j]).max())
