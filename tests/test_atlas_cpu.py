"""Deterministic atlas, host side (no GPU): the projected-area quadrature and the incident nodes
equal the reference's bit for bit (tests/golden/atlas_reference.npz, from hex_atlas/src/atlas.cpp
compiled by oracle/build_ref.sh); the quadrature keeps the properties the reference's own test
checks (hex_atlas/tests/atlas_tests.cpp:30-41); invalid input is rejected."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import GOLDEN


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN / "atlas_reference.npz")


def test_area_rule_matches_reference_bit_for_bit(icp, gold):
    off = gold["area_offsets"]
    for c, (R, L, kx, ky, kz, S) in enumerate(gold["area_cases"]):
        faces, pts, w = icp.atlas_area_rule(R, L, (kx, ky, kz), int(S))
        lo, hi = off[c], off[c + 1]
        assert np.array_equal(faces, gold["area_face"][lo:hi])
        assert np.array_equal(pts, gold["area_pos"][lo:hi])  # -0.0 and +0.0 compare equal; bits below
        assert np.array_equal(pts.view(np.uint64), gold["area_pos"][lo:hi].view(np.uint64))
        assert np.array_equal(w.view(np.uint64), gold["area_weight"][lo:hi].view(np.uint64))


def test_area_rule_properties(icp):
    """Every point strictly inside its face, the weights add up to the projected area, and the
    rule is deterministic (atlas_tests.cpp:30-41)."""
    R, L = 0.1, 0.7
    hl = 0.5 * L / R
    normals = np.array([[1, 0, 0], [.5, 0, math.sqrt(3) / 2], [-.5, 0, math.sqrt(3) / 2], [-1, 0, 0],
                        [-.5, 0, -math.sqrt(3) / 2], [.5, 0, -math.sqrt(3) / 2], [0, 1, 0], [0, -1, 0]])
    offsets = np.array([math.sqrt(3) / 2] * 6 + [hl] * 2)
    areas = np.array([R * L] * 6 + [3 * math.sqrt(3) / 2 * R * R] * 2)
    for k in ([1, 0, 0], [0, 1, 0], [1, 2, 3], [-1, -.001, -.9]):
        k = np.array(k, float) / np.linalg.norm(k)
        faces, pts, w = icp.atlas_area_rule(R, L, k, 3)
        assert np.all(w > 0)
        assert abs(w.sum() / float(areas @ np.maximum(0, -normals @ k)) - 1) < 5e-14
        gap = offsets[None, :] - pts @ normals.T
        own = gap[np.arange(len(faces)), faces]
        assert np.all(np.abs(own) <= 1e-12)
        others = gap.copy()
        others[np.arange(len(faces)), faces] = np.inf
        assert np.all(others > 1e-12)
        f2, p2, w2 = icp.atlas_area_rule(R, L, k, 3)
        assert np.array_equal(f2, faces) and np.array_equal(p2, pts) and np.array_equal(w2, w)
        # lit faces only; 6 points per cell, S^2 cells per side face and per cap sector
        lit = np.flatnonzero(-normals @ k > 0)
        assert set(faces.tolist()) <= set(lit.tolist())
        assert len(faces) == sum(6 * 9 * (1 if f < 6 else 6) for f in lit if areas[f] * -(normals[f] @ k) > 0)


def test_area_rule_rejects(icp):
    for args in [(0.0, 0.2, (1, 0, 0), 2), (0.1, -1.0, (1, 0, 0), 2), (0.1, 0.2, (1, 0, 0), 0),
                 (0.1, 0.2, (1, 0, 0), 1001), (0.1, 0.2, (0, 0, 0), 2), (0.1, 0.2, (math.nan, 0, 1), 2)]:
        with pytest.raises(icp.InvalidArgument):
            icp.atlas_area_rule(*args)


def test_incident_nodes_match_reference(icp, gold):
    for c in (0, 1):
        case = gold[f"nodes{c}_case"]
        T, P = int(case[5]), int(case[6])
        head = gold[f"nodes{c}_head"]
        for n in range((T + 1) * (P + 1)):
            i, j = divmod(n, P + 1)
            node = icp.atlas_incident_node(T, P, i, j)
            assert node.theta == head[n, 0] and node.phi == head[n, 1]
            assert list(node.ki) == list(head[n, 2:5])
            assert list(node.e0) == list(head[n, 5:8])
            e1 = np.cross(np.array(node.ki), np.array(node.e0))
            assert np.allclose(list(node.e1), e1, rtol=0, atol=1e-16)
    with pytest.raises(icp.InvalidArgument):
        icp.atlas_incident_node(3, 2, 4, 0)
    with pytest.raises(icp.InvalidArgument):
        icp.atlas_incident_node(0, 2, 0, 0)


def test_reference_atlas_nodes_are_consistent(gold):
    """The golden atlas itself: areas equal the analytic projected areas, masses close the
    escaped flux, and the node frames follow k(t,p), e0(t,p) (atlas.cpp:76-97)."""
    for c in (0, 1):
        case = gold[f"nodes{c}_case"]
        R, L, T, P = case[0], case[1], int(case[5]), int(case[6])
        head, mass = gold[f"nodes{c}_head"], gold[f"nodes{c}_mass"].reshape((T + 1) * (P + 1), -1)
        for n in range((T + 1) * (P + 1)):
            t, p = head[n, 0], head[n, 1]
            assert np.allclose(head[n, 2:5], [math.sin(t) * math.cos(p), math.cos(t), math.sin(t) * math.sin(p)],
                               atol=1e-15)
            assert abs(mass[n].sum() / head[n, 9] - 1) < 1e-12
            assert abs((head[n, 9] + head[n, 10]) / head[n, 8] - 1) < 1e-10


def _write_reference_atlas(gold, path, **spoil):
    """The golden reference atlas as a directory in the atlas contract."""
    import json

    case = gold["nodes1_case"]
    R, L, n, ne, nm, T, P, nt, np_, S, hits, tail = case
    T, P, nt, np_ = int(T), int(P), int(nt), int(np_)
    head = gold["nodes1_head"]
    path.mkdir()
    np.save(path / "mass_mm2.npy", gold["nodes1_mass"] * spoil.get("mass_scale", 1.0))
    np.save(path / "u_edges.npy", gold["compose_edges"])
    nodes = [{"i": k // (P + 1), "j": k % (P + 1), "theta": h[0], "phi": h[1], "ki": list(h[2:5]), "e0": list(h[5:8]),
              "projected_area_mm2": h[8], "escaped_mm2": h[9], "unresolved_mm2": h[10]} for k, h in enumerate(head)]
    meta = {"schema": "ice.single_particle_atlas.v1", "complete": True, "incident_theta_intervals": T,
            "incident_phi_intervals": P, "theta_count": nt, "phi_count": np_,
            "geometry": {"shape": "regular_hexagonal_prism", "circumradius_mm": R, "full_length_mm": L},
            "material": {"model": "constant", "wavelength_nm": nm, "interior_index": n, "exterior_index": ne},
            "symmetry": "D6h_O3_full_24_scalar_unpolarized",
            "incident_reconstruction": "bilinear_theta_phi_in_spherical_incident_frame",
            "transport": {"max_unresolved_fraction": 1e-10}, "nodes": nodes}
    meta.update(spoil.get("meta", {}))
    (path / "metadata.json").write_text(json.dumps(meta))
    return path


def test_atlas_reader_accepts_the_reference_atlas_and_rejects_damage(gold, tmp_path):
    from ice_crystal_phase_b200 import atlas as A

    a = A.Atlas(_write_reference_atlas(gold, tmp_path / "ok"))
    assert (a.it, a.ip, a.nt, a.np, a.nodes) == (6, 3, 16, 32, 28)
    assert np.array_equal(a.area.reshape(-1), gold["nodes1_head"][:, 8])
    for name, spoil in [("mass", {"mass_scale": 1.001}), ("schema", {"meta": {"schema": "other"}}),
                        ("incomplete", {"meta": {"complete": False}}),
                        ("symmetry", {"meta": {"symmetry": "none"}}), ("grid", {"meta": {"theta_count": 8}})]:
        with pytest.raises(ValueError):
            A.Atlas(_write_reference_atlas(gold, tmp_path / name, **spoil))
    part = tmp_path / "x.part"
    part.mkdir()
    with pytest.raises(ValueError):
        A.Atlas(part)


def test_incidents_and_cli_argument_checks(tmp_path):
    from ice_crystal_phase_b200 import atlas as A

    ks = A.incidents({"inclinations_deg": [0, 30, -90, 90]})
    assert np.array_equal(ks[2][0], [0.0, 1.0, 0.0]) and np.array_equal(ks[3][0], [0.0, -1.0, 0.0])
    assert np.allclose(ks[1][0], [math.cos(math.pi / 6), -0.5, 0.0], atol=1e-16)
    for bad in ({"inclinations_deg": [91]}, {"inclinations_deg": [0], "directions": [[1, 0, 0]]}, {},
                {"directions": [[0, 0, 0]]}):
        with pytest.raises(ValueError):
            A.incidents(bad)
    common = ["precompute", "--out", str(tmp_path / "a"), "--radius-mm", "0.1", "--length-mm", "0.2",
              "--wavelength-nm", "550", "--incident-theta-intervals", "2", "--incident-phi-intervals", "1",
              "--theta", "8", "--phi", "16", "--area-subdivisions", "1"]
    assert A.main(common + ["--ior", "1.31"]) == 2                       # ice material takes no --ior
    assert A.main(common + ["--material", "constant"]) == 2             # constant material needs --ior
    assert not (tmp_path / "a").exists() and not (tmp_path / "a.part").exists()


def test_precompute_cli_arguments(tmp_path):
    """The C++ drop-in of ice_precompute_atlas: the reference's option rules and exit code 2
    (hex_atlas/apps/precompute_atlas.cpp:44-98, 142-143), checked before any device is used."""
    import subprocess

    from conftest import ROOT

    exe = ROOT / "ice_crystal_phase_b200" / "bin" / "ice_precompute_atlas"

    def run(args, code):
        r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True)
        assert r.returncode == code, (r.returncode, r.stdout, r.stderr)
        return r

    assert "--material ice" in run(["--help"], 0).stdout
    base = ["--out", tmp_path / "a", "--radius-mm", "0.1", "--length-mm", "0.2", "--incident-theta-intervals", "2",
            "--incident-phi-intervals", "1", "--theta", "8", "--phi", "16", "--area-subdivisions", "1"]
    assert "--wavelength-nm is required" in run(base, 2).stderr
    assert "--ior requires explicit --material constant" in run(base + ["--wavelength-nm", "550", "--ior", "1.3"], 2).stderr
    assert "Constant material requires --ior" in run(base + ["--wavelength-nm", "550", "--material", "constant"], 2).stderr
    assert "200..1100 nm" in run(base + ["--wavelength-nm", "1200"], 2).stderr
    assert "Duplicate option" in run(base + ["--theta", "8"], 2).stderr
    assert "Unknown option" in run(base + ["--wavelength-nm", "550", "--bogus", "1"], 2).stderr
    assert "Invalid number" in run(base + ["--wavelength-nm", "5x0"], 2).stderr
    assert not (tmp_path / "a").exists() and not (tmp_path / "a.part").exists()


SPECTRAL_PLAN = {"wavelengths_nm": [450, 550, 650],
                 "precompute": {"radius_mm": .1, "length_mm": .2, "incident_theta_intervals": 3,
                                "incident_phi_intervals": 2, "theta": 12, "phi": 24, "area_subdivisions": 2,
                                "batch_rays": 8, "max_work_mib": 32},
                 "composition": {"inclinations_deg": [-90, 0, 35, 90], "orientation": {
                     "quadrature": {"azimuth": 4, "tilt": 4, "spin": 3},
                     "components": [{"kind": "horizontal_gaussian", "sigma_deg": 3, "fraction": .9},
                                    {"kind": "isotropic", "fraction": .1}]}}}


def test_spectral_plan_rules_and_dry_run(tmp_path, capsys):
    """The spectral runner's plan contract (hex_atlas/tools/run_spectrum.py:29-63) and its dry
    run, which creates nothing (hex_atlas/tests/spectral_cli_test.py:43-45)."""
    import copy
    import json

    from ice_crystal_phase_b200 import atlas as A

    path = tmp_path / "plan.json"
    path.write_text(json.dumps(SPECTRAL_PLAN))
    A.read_spectrum_plan(path)
    bad = []
    for mutate in (lambda p: p.pop("composition"), lambda p: p["precompute"].pop("batch_rays"),
                   lambda p: p["precompute"].update(theta=12.0), lambda p: p["precompute"].update(bogus=1),
                   lambda p: p.update(wavelengths_nm=[550, 450]), lambda p: p.update(wavelengths_nm=[150]),
                   lambda p: p.update(wavelengths_nm=[550, 550]),
                   lambda p: p["composition"].update(inclinations_deg=[0, 0]),
                   lambda p: p["composition"]["orientation"]["components"][0].update(fraction=.5)):
        q = copy.deepcopy(SPECTRAL_PLAN)
        mutate(q)
        bad.append(q)
    for k, q in enumerate(bad):
        p = tmp_path / f"bad{k}.json"
        p.write_text(json.dumps(q))
        with pytest.raises(ValueError):
            A.read_spectrum_plan(p)
    args = ["spectrum", "--plan", str(path), "--atlas-root", str(tmp_path / "atlases"), "--out", str(tmp_path / "dry"),
            "--dry-run"]
    assert A.main(args) == 0
    text = capsys.readouterr().out
    assert "DRY RUN: no files were created" in text and text.count("precompute --material ice") == 3
    assert "lambda_450_nm" in text
    assert not (tmp_path / "atlases").exists() and not (tmp_path / "dry").exists()
    p = tmp_path / "bad0.json"
    assert A.main(["spectrum", "--plan", str(p), "--atlas-root", str(tmp_path / "a"), "--out", str(tmp_path / "o")]) == 2
