"""Atlas orchestration on the CPU: precompute -> Atlas reader -> compose -> records, and the
spectral runner with its receipts and reuse, with the device steps (node trace, coupling,
composition, CDF) replaced by the oracle.  What runs for real is the library's host code:
directory and record contracts, plans, hashes, `.part` staging and the refusals."""
from __future__ import annotations

import json
import math
from types import SimpleNamespace

import numpy as np
import pytest

from oracle import atlas_oracle as AO
from oracle import oracle as O
from record_check import validate_record


class _Ctx:
    def __init__(self, *a):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


class _Dev:
    def __init__(self, *a, **k):
        pass

    def free(self):
        pass


def _trace_node(icp):
    def trace(ctx, s, i, j, mass=None):
        node = icp.atlas_incident_node(s.theta_intervals, s.phi_intervals, i, j)
        faces, pts, w = icp.atlas_area_rule(s.circumradius_mm, s.length_mm, list(node.rule_ki), s.subdivisions)
        m, st = O.atlas_node(s.circumradius_mm, s.length_mm, s.interior_index, list(node.ki), list(node.e0),
                             list(node.e1), faces, pts, w, s.nt, s.np, n_ext=s.exterior_index,
                             tail=s.tail_tolerance, max_hits=s.max_internal_hits)
        area = O.hex_projected_area(s.circumradius_mm, s.length_mm, list(node.ki))
        rep = SimpleNamespace(projected_area_mm2=area, escaped_mm2=st[0], unresolved_mm2=st[1],
                              histogram_relative_error=abs(m.sum() / st[0] - 1), rays=int(st[2]), outputs=int(st[3]),
                              max_balance_error=st[4], max_interface_balance_error=st[5])
        return m, rep
    return trace


def _composer(real):
    """The library's Composer with its device calls (coupling, composition) over the oracle; its own
    coupling_for_rule (vertical-incidence orbit average, rule check, area audit) runs unchanged."""

    class Composer(real):
        def __init__(self, ctx, first):
            self.first = first
            self.w = np.zeros((first.nodes, 2, first.np))
            self.coupling = SimpleNamespace(zero=lambda: self.w.fill(0.0), download=lambda: self.w.reshape(-1).copy())

        def add_coupling(self, rot, w, ki, fraction, orbit):
            a = self.first
            _, area = AO.coupling(a.area, a.it, a.ip, a.np, a.radius, a.length, np.asarray(rot), np.asarray(w),
                                  list(ki), fraction=fraction, orbit=orbit, out=self.w)
            return area

        def compose(self, atlas, wts):
            m = AO.compose(np.asarray(atlas.mass).reshape(atlas.nodes, atlas.nt, atlas.np), wts)
            residual = float(np.sum(np.sum(wts, axis=(1, 2)) * atlas.residual.reshape(-1)))
            return SimpleNamespace(download=lambda: m.reshape(-1).copy()), residual

    return Composer


def _cdf(ctx, mass, nt, np_):
    m = mass.download().reshape(nt, np_)
    a, b, rep = AO.make_cdf(m, O.u_edges(nt))
    return a, b, {"g_stored": rep["g"], "cdf_mass": rep["cdf_mass"], "l1_error": rep["l1"], "lost_mass": 0.0,
                  "maximum_cell_error": 0.0}


@pytest.fixture()
def A(icp, monkeypatch):
    from ice_crystal_phase_b200 import atlas as mod

    monkeypatch.setattr(mod, "trace_node", _trace_node(icp))
    monkeypatch.setattr(mod, "Composer", _composer(mod.Composer))
    monkeypatch.setattr(mod, "cdf", _cdf)
    monkeypatch.setattr(mod.icp, "DeviceArray", _Dev)
    monkeypatch.setattr(mod.icp, "Context", _Ctx)
    return mod


RULE = {"quadrature": {"azimuth": 4, "tilt": 4, "spin": 3},
        "components": [{"kind": "horizontal_gaussian", "sigma_deg": 10, "fraction": .75},
                       {"kind": "isotropic", "fraction": .25}]}


def test_precompute_compose_records(A, icp, tmp_path):
    """Two atlases, three inclinations, six records readable by the record reader; a repeat gives
    equal bytes; existing outputs are refused (hex_atlas/tests/cli_test.py:24-58)."""
    quiet = dict(log=lambda *_: None)
    paths = []
    for wave, n in ((550.0, 1.31), (650.0, 1.30)):
        s = A.settings(.1, .2, n, 3, 2, 12, 24, 2)
        paths.append(A.precompute(None, tmp_path / f"atlas{int(wave)}", s, wave, constant_index=True, **quiet))
    a = A.Atlas(paths[0])
    assert a.meta["material"]["model"] == "constant" and a.meta["total_rays"] > 0
    cfg = tmp_path / "compose.json"
    cfg.write_text(json.dumps({"inclinations_deg": [0, 35, 80], "orientation": RULE}))
    out = A.compose(None, paths, cfg, tmp_path / "dataset", **quiet)
    out2 = A.compose(None, paths, cfg, tmp_path / "repeat", **quiet)
    plan = json.loads((out / "batch_plan.json").read_text())
    assert plan["complete"] and len(plan["records"]) == 6
    gs = []
    for r in plan["records"]:
        d = out / r["path"]
        rec = validate_record(d)
        assert rec["metadata"]["orientation"]["randomness"] is False and rec["metadata"]["atlas"]["no_retracing"]
        assert abs(rec["metadata"]["transport_audit"]["balance_error"]) < 2e-10
        gs.append(rec["metadata"]["hg"]["g"])
        for f in ("phi_cdf.npy", "theta_given_phi_cdf.npy", "u_edges.npy"):
            assert (d / f).read_bytes() == (out2 / r["path"] / f).read_bytes()
        assert {p.name for p in d.iterdir()} == {"metadata.json", "phi_cdf.npy", "theta_given_phi_cdf.npy",
                                                 "u_edges.npy"}
    assert max(gs) - min(gs) > .01
    with pytest.raises(ValueError):
        A.compose(None, paths, cfg, out, **quiet)
    with pytest.raises(ValueError):
        A.precompute(None, paths[0], A.settings(.1, .2, 1.31, 3, 2, 12, 24, 2), 550.0, constant_index=True, **quiet)
    # an arbitrary direction needs the ensemble contract (compose_atlas.py:137-140)
    cfg.write_text(json.dumps({"directions": [[1, 0, 1]], "orientation": RULE}))
    with pytest.raises(ValueError, match="ensemble"):
        A.compose(None, paths[:1], cfg, tmp_path / "bad_contract", **quiet)
    assert not (tmp_path / "bad_contract").exists()
    A.compose(None, paths[:1], cfg, tmp_path / "ensemble", output_contract="ensemble", **quiet)


def test_spectral_runner_flow(A, icp, tmp_path):
    """Three dispersive-ice atlases, twelve records, a --reuse repeat that leaves the cached atlases
    untouched, the refusal of a changed request (hex_atlas/tests/spectral_cli_test.py)."""
    import copy

    from test_atlas_cpu import SPECTRAL_PLAN

    plan = tmp_path / "plan.json"
    plan.write_text(json.dumps(SPECTRAL_PLAN))
    root = tmp_path / "atlases"
    quiet = dict(log=lambda *_: None)
    A.spectrum(plan, root, tmp_path / "dataset", **quiet)
    times = []
    for w, n in zip(SPECTRAL_PLAN["wavelengths_nm"], [1.3157, 1.3110, 1.3080]):
        p = root / A.atlas_name(w)
        m = json.loads((p / "metadata.json").read_text())
        assert m["material"]["interior_index"] == n and m["material"]["wavelength_evaluated_nm"] == w
        assert (root / (A.atlas_name(w) + ".job.json")).exists() and (root / (A.atlas_name(w) + ".log")).exists()
        times.append((p / "mass_mm2.npy").stat().st_mtime_ns)
    index = json.loads((tmp_path / "dataset" / "batch_plan.json").read_text())
    assert index["complete"] and len(index["records"]) == 12
    for row in index["records"]:
        m = validate_record(tmp_path / "dataset" / row["path"])["metadata"]
        assert row["condition"][0] == m["wavelength_nm"]
    with pytest.raises(FileExistsError):
        A.spectrum(plan, root, tmp_path / "again", **quiet)      # cached atlases need --reuse
    A.spectrum(plan, root, tmp_path / "repeat", reuse=True, **quiet)
    for w, t in zip(SPECTRAL_PLAN["wavelengths_nm"], times):
        assert (root / A.atlas_name(w) / "mass_mm2.npy").stat().st_mtime_ns == t
    for row in index["records"]:
        for f in ("phi_cdf.npy", "theta_given_phi_cdf.npy"):
            assert (tmp_path / "repeat" / row["path"] / f).read_bytes() == \
                (tmp_path / "dataset" / row["path"] / f).read_bytes()
    changed = copy.deepcopy(SPECTRAL_PLAN)
    changed["precompute"]["length_mm"] = .3
    plan.write_text(json.dumps(changed))
    with pytest.raises(ValueError, match="differ"):
        A.spectrum(plan, root, tmp_path / "reject", reuse=True, **quiet)
    assert not (tmp_path / "reject").exists()
    assert math.isfinite(index["records"][0]["g"])
