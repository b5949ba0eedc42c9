"""Deterministic atlas on the GPU, through the C ABI, against the reference's own atlas and
composition (tests/golden/atlas_reference.npz).  The file sorts after the record-path GPU
suites.

* atlas trace: every node of two reference atlases (the reference's own test setting and the
  composition atlas); cell masses to L1 2e-11 with the same occupied cells, the ray-ordered escaped /
  unresolved sums, determinism, the index-matched delta and the failure gate of
  hex_atlas/tests/atlas_tests.cpp:43-72.
* coupling: the reference's rotations through icp_atlas_coupling; the expected area, the
  weight of every node (summed over the two parities, which a fold that lands exactly on a
  mirror plane may exchange), and the composed masses.
* compose: the reference's own weights give the reference's masses bit for bit.
* end to end: precompute -> Atlas reader -> compose -> records, conservation and CDF audit.
"""
from __future__ import annotations

import json
import math
from types import SimpleNamespace

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

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


def _settings(A, case, **over):
    R, L, n, ne, _, T, P, nt, np_, S, hits, tail = case
    kw = dict(exterior_index=ne, max_internal_hits=int(hits), tail_tolerance=tail)
    kw.update(over)
    return A.settings(R, L, n, int(T), int(P), int(nt), int(np_), int(S), **kw)


@pytest.mark.parametrize("c", [0, 1])
def test_atlas_nodes_match_reference(ctx, icp, gold, c):
    from ice_crystal_phase_b200 import atlas as A

    case = gold[f"nodes{c}_case"]
    s = _settings(A, case)
    T, P = s.theta_intervals, s.phi_intervals
    head, want = gold[f"nodes{c}_head"], gold[f"nodes{c}_mass"]
    launches = icp.kernel_launches()
    for n in range((T + 1) * (P + 1)):
        i, j = divmod(n, P + 1)
        mass, rep = A.trace_node(ctx, s, i, j)
        ref = want[i, j]
        assert rep.rays == int(head[n, 12]) and rep.outputs == int(head[n, 13])
        assert rep.projected_area_mm2 == head[n, 8]
        assert rep.escaped_mm2 == pytest.approx(head[n, 9], rel=1e-14)
        assert rep.unresolved_mm2 == pytest.approx(head[n, 10], rel=1e-9, abs=1e-30)
        assert rep.first_rejected == -1 and rep.invalid_bins == 0
        assert np.all(mass >= 0) and np.array_equal(mass > 0, ref > 0)
        # L1 as the FP64 record-path tests (the reference's own CUDA/CPU atlas bar is 2e-9)
        assert np.abs(mass - ref).sum() / ref.sum() <= 2e-11
        assert abs(mass.sum() / rep.escaped_mm2 - 1) < 1e-12
    assert icp.kernel_launches() - launches == 2 * (T + 1) * (P + 1)


def test_atlas_trace_is_deterministic_and_index_matched(ctx, icp, gold):
    from ice_crystal_phase_b200 import atlas as A

    s = _settings(A, gold["nodes0_case"])
    a, _ = A.trace_node(ctx, s, 1, 1)
    b, _ = A.trace_node(ctx, s, 1, 1)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    # n = 1: every ray passes straight through into the forward cap (atlas_tests.cpp:50-55)
    s.interior_index = 1.0
    m, rep = A.trace_node(ctx, s, 1, 1)
    want = np.zeros_like(m)
    want[0, :] = rep.projected_area_mm2 / s.np
    assert np.max(np.abs(m - want)) < 1e-15


def test_atlas_trace_failure_gates(ctx, icp, gold):
    from ice_crystal_phase_b200 import atlas as A

    s = _settings(A, gold["nodes0_case"], max_internal_hits=1)
    with pytest.raises(icp.AuditError, match="Deterministic area ray rejected"):
        A.trace_node(ctx, s, 1, 1)
    for over in ({"subdivisions": 0}, {"tail_tolerance": 1e-9, "max_unresolved_fraction": 1e-10}):
        s = _settings(A, gold["nodes0_case"])
        for k, v in over.items():
            setattr(s, k, v)
        with pytest.raises(icp.InvalidArgument):
            A.trace_node(ctx, s, 0, 0)


def _atlas_stub(gold):
    case = gold["nodes1_case"]
    T, P, nt, np_ = (int(x) for x in case[5:9])
    head = gold["nodes1_head"].reshape(T + 1, P + 1, 16)
    return SimpleNamespace(it=T, ip=P, nt=nt, np=np_, radius=case[0], length=case[1], area=head[:, :, 8].copy(),
                           residual=head[:, :, 10].copy(), mass=gold["nodes1_mass"], nodes=(T + 1) * (P + 1),
                           edges=gold["compose_edges"])


@pytest.mark.parametrize("ri", [0, 1])
@pytest.mark.parametrize("ii", range(5))
def test_coupling_and_compose_match_reference(ctx, icp, gold, ri, ii):
    from ice_crystal_phase_b200 import atlas as A

    atlas = _atlas_stub(gold)
    comp = A.Composer(ctx, atlas)
    rot, w, meta = A.orientation_rule(RULES[ri])
    ki = gold["compose_incidents"][ii]
    key = f"compose{ri}_{ii}"
    wts, area, frame, info = comp.coupling_for_rule(rot, w, ki, meta)
    want = gold[key + "_coupling"].reshape(atlas.nodes, 2, atlas.np)
    assert area == pytest.approx(gold[key + "_scalars"][0], rel=1e-13)
    assert np.allclose(frame, gold[key + "_frame"], rtol=0, atol=1e-15)
    assert info["method"].startswith("analytic") == bool(gold[key + "_scalars"][4])
    per_node, per_node_ref = wts.sum(axis=(1, 2)), want.sum(axis=(1, 2))
    assert np.max(np.abs(per_node - per_node_ref)) <= 1e-12 * per_node_ref.max()
    mass, residual = comp.compose(atlas, wts)
    m = mass.download().reshape(atlas.nt, atlas.np)
    ref = gold[key + "_mass"]
    assert np.max(np.abs(m - ref)) <= 1e-10 * ref.max()
    assert residual == pytest.approx(gold[key + "_scalars"][1], rel=1e-9, abs=1e-30)
    # the reference's own weights: bit for bit
    comp.coupling.upload(want.reshape(-1))
    mass, _ = comp.compose(atlas, want)
    assert np.array_equal(mass.download().reshape(atlas.nt, atlas.np), ref)


def test_compose_larger_grid_matches_oracle(ctx, icp):
    """Sparse and dense weights over a grid wider than one thread strip (np = 2100 > 2048),
    against the oracle's ordered sum: bit for bit."""
    from oracle import atlas_oracle as AO

    rng = np.random.default_rng(7)
    nodes, nt, np_ = 3, 5, 2100
    mass = rng.random((nodes, nt, np_))
    w = np.zeros((nodes, 2, np_))
    w[0, 0, rng.choice(np_, 9, replace=False)] = rng.random(9)
    w[1, 1, :] = rng.random(np_) * 1e-3
    w[2, 0, 100:140] = rng.random(40)
    d_mass = icp.DeviceArray(ctx, mass.size).upload(mass.reshape(-1))
    d_w = icp.DeviceArray(ctx, w.size).upload(w.reshape(-1))
    out = icp.DeviceArray(ctx, nt * np_)
    icp.check(icp.LIB.icp_atlas_compose(ctx.handle, nodes, nt, np_, d_mass.ptr, d_w.ptr, out.ptr))
    assert np.array_equal(out.download().reshape(nt, np_), AO.compose(mass, w))


def test_precompute_and_compose_end_to_end(ctx, icp, tmp_path):
    from ice_crystal_phase_b200 import atlas as A

    s = A.settings(0.05, 0.2, 0.0, 2, 1, 16, 32, 2)
    out = A.precompute(ctx, tmp_path / "atlas_550", s, 550.0, log=lambda *_: None)
    atlas = A.Atlas(out)  # the reader's audits: frames, areas, mass vs escaped, residual
    assert atlas.meta["material"]["model"] == "ice_ih_warren_brandt_2008_real_only"
    assert atlas.meta["material"]["interior_index"] == icp.evaluate_ice_optics(550.0).n
    cfg = tmp_path / "cfg.json"
    cfg.write_text(json.dumps({"inclinations_deg": [0, 45, 90], "orientation": RULES[0]}))
    res = A.compose(ctx, [out], cfg, tmp_path / "phase", log=lambda *_: None)
    plan = json.loads((res / "batch_plan.json").read_text())
    assert plan["complete"] and len(plan["records"]) == 3
    for rec in plan["records"]:
        d = res / rec["path"]
        meta = json.loads((d / "metadata.json").read_text())
        phi = np.load(d / "phi_cdf.npy")
        theta = np.load(d / "theta_given_phi_cdf.npy")
        assert phi[0] == 0 and phi[-1] == 1 and np.all(np.diff(phi) >= 0)
        assert np.all(theta[:, 0] == 0) and np.all(theta[:, -1] == 1)
        assert meta["quality"]["cdf_l1_mass_error"] <= 1e-10
        assert abs(meta["transport_audit"]["balance_error"]) <= 2e-10
        assert -1 < meta["hg"]["g"] < 1
    vertical = json.loads((res / plan["records"][2]["path"] / "metadata.json").read_text())
    assert vertical["orientation"]["azimuth_integration"]["method"].startswith("analytic")
    assert math.isclose(vertical["incident_inclination_degrees"], 90.0)


def test_precompute_cli_matches_the_library(ctx, icp, tmp_path):
    """bin/ice_precompute_atlas writes the same atlas as atlas.precompute (deterministic
    histograms: equal bits), and the reader's audits accept it."""
    import subprocess

    from conftest import ROOT
    from ice_crystal_phase_b200 import atlas as A

    exe = ROOT / "ice_crystal_phase_b200" / "bin" / "ice_precompute_atlas"
    out = tmp_path / "cli"
    r = subprocess.run([str(exe), "--out", str(out), "--radius-mm", "0.05", "--length-mm", "0.2", "--wavelength-nm",
                        "550", "--incident-theta-intervals", "2", "--incident-phi-intervals", "1", "--theta", "16",
                        "--phi", "32", "--area-subdivisions", "2"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "atlas_complete nodes=6" in r.stdout
    lib = A.precompute(ctx, tmp_path / "lib", A.settings(0.05, 0.2, 0.0, 2, 1, 16, 32, 2), 550.0, log=lambda *_: None)
    a, b = A.Atlas(out), A.Atlas(lib)
    assert np.array_equal(np.asarray(a.mass).view(np.uint64), np.asarray(b.mass).view(np.uint64))
    assert np.array_equal(a.area, b.area) and np.array_equal(a.edges, b.edges)
    assert a.meta["material"]["interior_index"] == b.meta["material"]["interior_index"]


def test_spectral_runner_end_to_end(ctx, icp, tmp_path):
    """Three dispersive-ice atlases and twelve records (hex_atlas/tests/spectral_cli_test.py):
    the ice index per wavelength, different atlases per wavelength, the record contract, a
    repeat with --reuse that leaves the cached atlases untouched and gives equal bytes, and the
    refusal of a cache whose request changed."""
    import copy

    from record_check import validate_record
    from test_atlas_cpu import SPECTRAL_PLAN
    from ice_crystal_phase_b200 import atlas as A

    plan = tmp_path / "plan.json"
    plan.write_text(json.dumps(SPECTRAL_PLAN))
    root = tmp_path / "atlases"
    quiet = dict(log=lambda *_: None)
    A.spectrum(plan, root, tmp_path / "dataset", **quiet)
    arrays, times = [], []
    for w, n in zip(SPECTRAL_PLAN["wavelengths_nm"], [1.3157, 1.3110, 1.3080]):
        p = root / A.atlas_name(w)
        m = json.loads((p / "metadata.json").read_text())
        assert m["material"]["interior_index"] == n and m["material"]["automatic_ice_dispersion"] is True
        arrays.append(np.load(p / "mass_mm2.npy"))
        times.append((p / "mass_mm2.npy").stat().st_mtime_ns)
    assert not np.array_equal(arrays[0], arrays[1]) and not np.array_equal(arrays[1], arrays[2])
    index = json.loads((tmp_path / "dataset" / "batch_plan.json").read_text())
    assert index["complete"] and len(index["records"]) == 12
    for row in index["records"]:
        validate_record(tmp_path / "dataset" / row["path"])
    A.spectrum(plan, root, tmp_path / "repeat", reuse=True, **quiet)
    for w, t in zip(SPECTRAL_PLAN["wavelengths_nm"], times):
        assert (root / A.atlas_name(w) / "mass_mm2.npy").stat().st_mtime_ns == t
    for row in index["records"]:
        for f in ("phi_cdf.npy", "theta_given_phi_cdf.npy", "u_edges.npy"):
            assert (tmp_path / "repeat" / row["path"] / f).read_bytes() == (tmp_path / "dataset" / row["path"] / f).read_bytes()
    changed = copy.deepcopy(SPECTRAL_PLAN)
    changed["precompute"]["length_mm"] = .3
    plan.write_text(json.dumps(changed))
    with pytest.raises(ValueError):
        A.spectrum(plan, root, tmp_path / "reject", reuse=True, **quiet)
    assert not (tmp_path / "reject").exists()


def _pattern_stub():
    from test_atlas_oracle_cpu import pattern_atlas

    a = pattern_atlas()
    return SimpleNamespace(it=a["it"], ip=a["ip"], nt=a["nt"], np=a["np"], radius=a["R"], length=a["L"],
                           area=a["area"], residual=a["residual"], mass=a["mass"], nodes=(a["it"] + 1) * (a["ip"] + 1)), a


def test_device_coupling_shift_reflection_and_mixture(ctx, icp):
    """The reference's composition properties (hex_atlas/tests/test_compose.py:76-108) through
    icp_atlas_coupling and icp_atlas_compose."""
    from test_atlas_oracle_cpu import expected_shift, shift_cases
    from ice_crystal_phase_b200 import atlas as A

    stub, a = _pattern_stub()
    comp = A.Composer(ctx, stub)

    def run(rot, w, ki):
        comp.coupling.zero()
        area = comp.add_coupling(np.asarray(rot), np.asarray(w, float), np.asarray(ki, float), 1.0, False)
        wts = comp.coupling.download().reshape(stub.nodes, 2, stub.np)
        mass, _ = comp.compose(stub, wts)
        return mass.download().reshape(stub.nt, stub.np), area, wts

    for reflected, shift, r in shift_cases():
        got, area, _ = run(np.array([r]), [1.0], [1, 0, 0])
        assert np.allclose(got, expected_shift(a, reflected, shift), atol=3e-17, rtol=1e-12), (reflected, shift)
        assert got.sum() == pytest.approx(area)
    rot = np.array([np.eye(3), A._rz(np.array(math.pi / 2))])
    out, area, _ = run(rot, [.25, .75], [1, 0, 0])
    exact = .25 * A.projected_area(.1, .2, [1, 0, 0]) + .75 * A.projected_area(.1, .2, [0, -1, 0])
    assert area == pytest.approx(exact) and out.sum() == pytest.approx(exact)


def test_device_poles_are_uniform_in_phi(ctx, icp):
    """Vertical incidence: the analytic azimuth average equals the phi mean of the discrete rule
    and does not depend on the azimuth node count (hex_atlas/tests/test_polar_azimuth.py:34-69)."""
    from test_atlas_oracle_cpu import polar_rule
    from ice_crystal_phase_b200 import atlas as A

    stub, a = _pattern_stub()
    comp = A.Composer(ctx, stub)
    for sign in (-1, 1):
        ki = np.array([0.0, float(sign), 0.0])
        rot, w, meta = A.orientation_rule(polar_rule())
        comp.coupling.zero()
        comp.add_coupling(rot, w, ki, 1.0, False)
        wd = comp.coupling.download().reshape(stub.nodes, 2, stub.np)
        old = comp.compose(stub, wd)[0].download().reshape(stub.nt, stub.np)
        wts, area, _, info = comp.coupling_for_rule(rot, w, ki, meta)
        new = comp.compose(stub, wts)[0].download().reshape(stub.nt, stub.np)
        assert info["method"].startswith("analytic") and info["effective_pose_evaluations"] == 24
        assert np.allclose(new, np.repeat(old.mean(axis=1, keepdims=True), stub.np, axis=1), rtol=1e-12, atol=2e-17)
        first = None
        for na in (1, 2, 7, 23):
            r2, w2, m2 = A.orientation_rule(polar_rule(na))
            wts, _, _, _ = comp.coupling_for_rule(r2, w2, ki, m2)
            got = comp.compose(stub, wts)[0].download()
            if first is None:
                first = got
            assert np.array_equal(got, first)


def test_atlas_nodes_match_oracle_beyond_the_fixtures(ctx, icp):
    """Settings outside the fixtures (S = 3, the ice index at 400 nm, 20 x 40 cells, a longer
    column) against the oracle's atlas node, which equals the reference's trace_cpu bit for bit
    on the fixtures."""
    from oracle import oracle as O
    from ice_crystal_phase_b200 import atlas as A

    n = icp.evaluate_ice_optics(400.0).n
    s = A.settings(0.08, 0.5, n, 2, 1, 20, 40, 3)
    for m in range(6):
        i, j = divmod(m, 2)
        mass, rep = A.trace_node(ctx, s, i, j)
        node = icp.atlas_incident_node(2, 1, i, j)
        faces, pts, w = icp.atlas_area_rule(0.08, 0.5, list(node.rule_ki), 3)
        ref, st = O.atlas_node(0.08, 0.5, n, list(node.ki), list(node.e0), list(node.e1), faces, pts, w, 20, 40)
        assert rep.rays == st[2] and rep.outputs == st[3] and rep.first_rejected == -1 and st[6] == -1
        assert rep.escaped_mm2 == pytest.approx(st[0], rel=1e-14)
        assert np.array_equal(mass > 0, ref > 0)
        assert np.abs(mass - ref).sum() / ref.sum() <= 2e-11
