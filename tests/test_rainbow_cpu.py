"""Table-II rainbow diffraction on the CPU (no GPU): the oracle pinned to the reference's
outputs (tests/golden/rainbow_reference.npz, made by the reference's own header), the
reference's diffraction unit tests restated over the oracle
(tests/test_wave_optics_cpu.cpp:63-133 of the reference), the host-side Table-II lookup of
the C ABI, the Python configuration mirror, and the ABI struct layouts."""
from __future__ import annotations

import ctypes as C
import math
import subprocess

import numpy as np
import pytest

import rainbow_cases as RC
from conftest import GOLDEN, ROOT

Z = np.load(GOLDEN / "rainbow_reference.npz")


def bits(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def same_results(a: np.ndarray, b: np.ndarray) -> bool:
    return all(np.array_equal(bits(a[k]), bits(b[k])) for k in ("intensity_s", "intensity_p", "sigma_rad", "blend")) \
        and np.array_equal(a["flags"], b["flags"]) and np.array_equal(a["transition_kind"], b["transition_kind"])


def case_inputs(name: str):
    spec = next(c for c in RC.CASES if c[0] == name)
    _, nt, np_, cfg, make, labels = spec
    f = make()
    assert RC.digest(f) == str(Z[f"{name}.digest"]), f"{name}: the grid differs from the one the reference saw"
    assert tuple(Z[f"{name}.shape"]) == (nt, np_) and np.array_equal(Z[f"{name}.config"], cfg)
    given = Z[f"{name}.edges"] if int(Z[f"{name}.given"]) else None
    return f, nt, np_, cfg, given


# ----------------------------------------------------------------- pinned to the reference
def test_table_sigma_matches_reference(oracle, icp):
    for r, ok, s in zip(Z["table_radius"], Z["table_ok"], Z["table_sigma"]):
        got = oracle.rainbow_table_sigma(float(r))
        assert (got is not None) == bool(ok), r
        if ok:
            assert np.float64(got).view(np.uint64) == np.float64(s).view(np.uint64), r
            assert icp.rainbow_table_sigma(float(r)) == got
        else:
            with pytest.raises(icp.InvalidArgument):
                icp.rainbow_table_sigma(float(r))


@pytest.mark.parametrize("name", [c[0] for c in RC.CASES])
def test_oracle_bit_identical_to_reference(oracle, name):
    f, nt, np_, cfg, given = case_inputs(name)
    edges = oracle.rainbow_detect(f, nt, np_, cfg) if given is None else given
    assert np.array_equal(edges, Z[f"{name}.edges"])
    out = oracle.rainbow_filter(f, edges, nt, np_, cfg)
    assert same_results(out, RC.expected(Z, name, f))
    sub = np.arange(0, nt * np_, 7)
    assert same_results(oracle.rainbow_filter_at(f, edges, nt, np_, cfg, sub), out[sub])


# ------------------------------------------------- the reference's unit tests, over the oracle
def test_table_ii_values():
    radii = [0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8, 0.9, 1.0]
    widths = [0.70, 0.45, 0.30, 0.25, 0.22, 0.20, 0.18, 0.17, 0.16, 0.15]
    from oracle import oracle as O
    assert [O.rainbow_table_sigma(r) for r in radii] == widths
    assert O.rainbow_table_sigma(1.01) is None and O.rainbow_table_sigma(0.01) is None
    assert abs(O.rainbow_table_sigma(0.35) - 0.275) <= 1e-7 * 1.275


def test_paper_labels_coverage_and_widths(oracle):
    f = RC.paper_grid()
    cfg = RC.PAPER_CONFIG
    e = oracle.rainbow_detect(f, 180, 72, cfg)
    assert (e & 1).astype(bool).sum() == 72 and (e & 2).astype(bool).sum() == 72
    out = oracle.rainbow_filter(f, e, 180, 72, cfg)
    assert not (out["flags"] & 60).any()  # every direction available
    filt = (out["flags"] & 1) != 0
    kinds = out["transition_kind"][filt]
    assert (kinds == 1).any() and (kinds == 2).any()
    assert ((out["blend"][filt] > 0) & (out["blend"][filt] < 1)).any()
    assert np.array_equal(out["sigma_rad"][filt], cfg[0] * np.where(kinds == 2, 2.0, 1.0))


def test_paper_stencil_equals_full_sphere_sum(oracle):
    """The cap window agrees with an independent all-grid convolution in extended precision."""
    f = RC.paper_grid()
    cfg = RC.PAPER_CONFIG
    e = oracle.rainbow_detect(f, 180, 72, cfg)
    dt, dp = np.longdouble(math.pi) / 180, 2 * np.longdouble(math.pi) / 72
    t = (np.arange(180, dtype=np.longdouble) + np.longdouble(0.5)) * dt
    for row in (126, 129, 137, 140):
        for col in (0, 1, 71):
            i = row * 72 + col
            out = oracle.rainbow_filter_at(f, e, 180, 72, cfg, [i])[0]
            assert out["flags"] & 1
            theta = t[row]
            dphi = (np.arange(72, dtype=np.longdouble) - col) * dp
            dot = np.cos(theta) * np.cos(t)[:, None] + np.sin(theta) * np.sin(t)[:, None] * np.cos(dphi)[None, :]
            d = np.arccos(np.clip(dot, -1, 1))
            keep = d <= cfg[1] * out["sigma_rad"] + 2.0 ** -44
            w = np.exp(np.longdouble(-0.5) * (d / out["sigma_rad"]) ** 2) * 2 * np.sin(t)[:, None] * np.sin(dt / 2) * dp
            w = np.where(keep, w, 0)
            for key in ("intensity_s", "intensity_p"):
                x = f[key].reshape(180, 72).astype(np.longdouble)
                want = f[key][i] + np.longdouble(out["blend"]) * ((w * x).sum() / w.sum() - f[key][i])
                assert abs(out[key] - float(want)) <= 2e-10 * (1 + abs(float(want)))


def test_constant_holes_unknown_and_zero(oracle):
    cfg = RC.PAPER_CONFIG
    paper = RC.paper_grid()
    e = oracle.rainbow_detect(paper, 180, 72, cfg)
    flat = RC.paper_grid()
    flat["intensity_s"], flat["intensity_p"] = 3.25, 0.125
    target = 137 * 72
    v = oracle.rainbow_filter_at(flat, e, 180, 72, cfg, [target])[0]
    assert abs(v["intensity_s"] - 3.25) <= 1e-14 * 4.25 and abs(v["intensity_p"] - 0.125) <= 1e-14 * 1.125
    flat["flags"][target + 1] = 2  # a pending neighbour is never filled in
    v = oracle.rainbow_filter_at(flat, e, 180, 72, cfg, [target])[0]
    assert v["flags"] & 8 and math.isnan(v["intensity_s"])
    flat["flags"][target + 1] = 0
    unknown = e.copy()
    unknown[target + 1] = 4
    v = oracle.rainbow_filter_at(flat, unknown, 180, 72, cfg, [target])[0]
    assert v["flags"] & 16 and math.isnan(v["intensity_p"])
    none = np.zeros_like(e)
    v = oracle.rainbow_filter_at(flat, none, 180, 72, cfg, [10 * 72])[0]
    assert v["flags"] == 0 and v["intensity_s"] == 3.25
    flat["intensity_s"], flat["intensity_p"] = 0, 0
    v = oracle.rainbow_filter_at(flat, none, 180, 72, cfg, [10 * 72])[0]
    assert v["flags"] == 0 and v["intensity_s"] == 0


def test_invalid_configs_and_coarse_kernel(oracle):
    nan = float("nan")
    assert not oracle.rainbow_config_ok(180, 72, (nan, 4, 0.25, 3))
    assert not oracle.rainbow_config_ok(1, 72, RC.PAPER_CONFIG)
    assert not oracle.rainbow_config_ok(180, 72, (0.5, 4, 0.25, 3))  # 2 sigma x support >= pi
    assert not oracle.rainbow_config_ok(180, 72, (0.01, 4, 1.0, 3))
    assert not oracle.rainbow_config_ok(180, 72, (0.01, 4, 0.25, 4))
    assert not oracle.rainbow_config_ok(32768, 2, RC.PAPER_CONFIG)
    f = RC.paper_grid()
    e = oracle.rainbow_detect(f, 180, 72, (nan, 4, 0.25, 3))
    assert (e == 4).all()
    out = oracle.rainbow_filter(f, e, 180, 72, (nan, 4, 0.25, 3))
    assert (out["flags"] == 32).all() and np.isnan(out["intensity_s"]).all()
    coarse = (0.15 * math.pi / 180, 4.0, 0.25, 3.0)
    e = oracle.rainbow_detect(f, 180, 72, coarse)
    v = oracle.rainbow_filter_at(f, e, 180, 72, coarse, [137 * 72])[0]
    assert v["flags"] & 1 and v["flags"] & 2


def test_distance_is_the_haversine(oracle):
    rng = np.random.default_rng(3)
    for _ in range(200):
        a, b, p = rng.uniform(0, math.pi), rng.uniform(0, math.pi), rng.uniform(-math.pi, math.pi)
        c = math.cos(a) * math.cos(b) + math.sin(a) * math.sin(b) * math.cos(p)
        assert abs(oracle.rainbow_distance(a, b, p) - math.acos(max(-1.0, min(1.0, c)))) < 1e-7


# ------------------------------------------------------------------- host side of the ABI
def test_diffraction_config_mirror(icp):
    c = icp.diffraction_config(0.55)
    assert c.primary_sigma_rad == icp.rainbow_table_sigma(0.55) * math.pi / 180.0
    assert (c.support_sigma, c.transition_contrast, c.inner_blend_sigma) == (4.0, 0.25, 3.0)
    assert icp.diffraction_config(1.5, primary_sigma_deg=0.3).primary_sigma_rad == 0.3 * math.pi / 180.0
    with pytest.raises(icp.InvalidArgument):
        icp.diffraction_config(1.5)
    with pytest.raises(icp.InvalidArgument):
        icp.diffraction_config(0.5, primary_sigma_deg=-1)


def test_numpy_records_match_the_c_structs(icp, oracle, tmp_path):
    assert icp.FOCAL_DTYPE == oracle.FOCAL_DTYPE == RC.FOCAL_DTYPE
    assert icp.DIFFRACTION_DTYPE == oracle.RESULT_DTYPE == RC.RESULT_DTYPE
    focal = ["field", "intensity_s", "intensity_p", "family_incoherent", "family_hits", "corrected_hits",
             "extra_quarter_turn_hits", "flags", "first_problem_patch_id", "field_second"]
    result = ["intensity_s", "intensity_p", "sigma_rad", "blend", "flags", "transition_kind"]
    lines = [f'printf("focal {k} %zu\\n", offsetof(icp_focal_sample, {k}));' for k in focal]
    lines += [f'printf("result {k} %zu\\n", offsetof(icp_diffraction_result, {k}));' for k in result]
    lines += ['printf("size focal %zu\\n", sizeof(icp_focal_sample));',
              'printf("size result %zu\\n", sizeof(icp_diffraction_result));',
              'printf("size config %zu\\n", sizeof(icp_diffraction_config));',
              'printf("size stats %zu\\n", sizeof(icp_diffraction_stats));']
    src = tmp_path / "layout.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "icp_b200.h"\nint main(void){\n' +
                   "\n".join(lines) + "\nreturn 0;}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = {tuple(line.split()[:2]): int(line.split()[2])
           for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines()}
    for k in focal:
        assert got[("focal", k)] == icp.FOCAL_DTYPE.fields[k][1], k
    for k in result:
        assert got[("result", k)] == icp.DIFFRACTION_DTYPE.fields[k][1], k
    assert got[("size", "focal")] == 144 and got[("size", "result")] == 40
    assert got[("size", "config")] == C.sizeof(icp.DiffractionConfig)
    assert got[("size", "stats")] == C.sizeof(icp.DiffractionStats)


def test_oracle_against_live_reference_when_present(oracle):
    """Fresh random grids through the reference's header (skipped where it is not built)."""
    if not oracle.ref_rainbow_available():
        pytest.skip("reference harness not built")
    rng = np.random.default_rng(8)
    for trial in range(6):
        nt, np_ = int(rng.integers(2, 70)), int(rng.integers(1, 90))
        f = RC.bow_grid(nt, np_, 100 + trial, invalid=0.01)
        sig = rng.uniform(0.3, 4) * math.pi / 180
        sup = rng.uniform(2, 8)
        cfg = (sig, sup, rng.uniform(0, 0.4), rng.uniform(0, sup))
        re, ro = oracle.ref_rainbow_grid(f, nt, np_, cfg)
        e = oracle.rainbow_detect(f, nt, np_, cfg)
        assert np.array_equal(e, re)
        assert same_results(oracle.rainbow_filter(f, e, nt, np_, cfg), ro)
