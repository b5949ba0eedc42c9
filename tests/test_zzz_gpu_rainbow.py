"""Table-II rainbow diffraction on the GPU, through the C ABI, against the reference's outputs
(tests/golden/rainbow_reference.npz) and the CPU oracle.

Tolerances are the reference's own for its CUDA kernels against its host build
(tests/wave_optics_test_cases.hpp:27-33 of the reference): flags and transition kinds exact,
sigma to 1e-11 and blend to 1e-9 relative, available intensities to 1e-9 relative,
unavailable ones NaN.  The last-ulp differences come from CUDA's libm (sin, asin, exp).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import rainbow_cases as RC
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

Z = np.load(GOLDEN / "rainbow_reference.npz")


def near(a, b, tol):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return np.isfinite(a) & np.isfinite(b) & (np.abs(a - b) <= tol * (1 + np.abs(b)))


def mismatches(got: np.ndarray, want: np.ndarray) -> list[str]:
    bad = []
    if not np.array_equal(got["flags"], want["flags"]):
        bad.append(f"flags at {np.flatnonzero(got['flags'] != want['flags'])[:8]}")
    if not np.array_equal(got["transition_kind"], want["transition_kind"]):
        bad.append("transition kind")
    if not (near(got["sigma_rad"], want["sigma_rad"], 1e-11) | (got["sigma_rad"] == want["sigma_rad"])).all():
        bad.append("sigma")
    if not (near(got["blend"], want["blend"], 1e-9) | (got["blend"] == want["blend"])).all():
        bad.append("blend")
    ok = (want["flags"] & 60) == 0
    for k in ("intensity_s", "intensity_p"):
        if not (near(got[k][ok], want[k][ok], 1e-9) | (got[k][ok] == want[k][ok])).all():
            bad.append(k)
        if not np.isnan(got[k][~ok]).all():
            bad.append(f"{k} unavailable not NaN")
    return bad


def counts(edges: np.ndarray, res: np.ndarray) -> dict:
    f = res["flags"]
    return {"primary_transitions": int(((edges & 1) != 0).sum()), "secondary_transitions": int(((edges & 2) != 0).sum()),
            "unknown_transitions": int(((edges & 4) != 0).sum()), "filtered_directions": int(((f & 1) != 0).sum()),
            "unavailable_directions": int(((f & 60) != 0).sum()), "underresolved_directions": int(((f & 2) != 0).sum())}


@pytest.mark.parametrize("name", [c[0] for c in RC.CASES])
def test_fixture_cases_match_reference(icp, ctx, name):
    spec = next(c for c in RC.CASES if c[0] == name)
    _, nt, np_, cfg, make, _ = spec
    f = make()
    assert RC.digest(f) == str(Z[f"{name}.digest"])
    given = Z[f"{name}.edges"] if int(Z[f"{name}.given"]) else None
    before = icp.kernel_launches()
    out = icp.rainbow_diffraction(ctx, f, nt, np_, icp.DiffractionConfig(*cfg), transitions=given)
    assert icp.kernel_launches() - before == 2
    assert np.array_equal(out.transitions, Z[f"{name}.edges"])
    want = RC.expected(Z, name, f)
    assert not mismatches(out.results, want), mismatches(out.results, want)
    dens = out.results["intensity_s"] + out.results["intensity_p"]
    assert np.array_equal(np.isnan(out.density), np.isnan(dens))
    assert np.array_equal(out.density[~np.isnan(dens)], dens[~np.isnan(dens)])
    want_counts = counts(out.transitions, out.results)
    if given is not None:  # the filter entry reports result counters only
        want_counts.update(primary_transitions=0, secondary_transitions=0, unknown_transitions=0)
    assert out.stats == want_counts


def test_separate_passes_equal_the_combined_call(icp, ctx):
    f = RC.bow_grid(120, 96, 21, invalid=0.003)
    cfg = icp.DiffractionConfig(1.1 * math.pi / 180, 4.0, 0.2, 3.0)
    both = icp.rainbow_diffraction(ctx, f, 120, 96, cfg)
    df = icp.DeviceArray(ctx, f.size, icp.FOCAL_DTYPE).upload(f)
    de = icp.DeviceArray(ctx, f.size, np.uint32)
    icp.check(icp.LIB.icp_rainbow_detect(ctx.handle, df.ptr, 120, 96, icp.C.byref(cfg), de.ptr))
    assert np.array_equal(de.download(), both.transitions)
    sep = icp.rainbow_diffraction(ctx, df, 120, 96, cfg, transitions=both.transitions)
    assert sep.results.tobytes() == both.results.tobytes()


def test_rejects_invalid_configuration(icp, ctx):
    f = RC.paper_grid()
    for cfg in ((float("nan"), 4, 0.25, 3), (0.5, 4, 0.25, 3), (0.01, 1.5, 0.25, 1), (0.01, 4, 0.25, 4)):
        with pytest.raises(icp.InvalidArgument):
            icp.rainbow_diffraction(ctx, f, 180, 72, icp.DiffractionConfig(*cfg))
    with pytest.raises(icp.InvalidArgument):
        icp.rainbow_diffraction(ctx, f[:72], 1, 72, icp.DiffractionConfig(*RC.PAPER_CONFIG))


def test_full_query_grid_against_oracle_and_properties(icp, ctx, oracle):
    """The 1800 x 3600 query grid of the drop records (0.1 degree cells): parity with the oracle
    at 3000 directions (those the pass changed and random ones), unflagged directions returned
    bit for bit, counters equal to the result arrays, and a constant preserved everywhere."""
    nt, np_ = 1800, 3600
    f = RC.bow_grid(nt, np_, 31, noise=0.2, invalid=2e-6)
    cfg = icp.diffraction_config(0.5)
    out = icp.rainbow_diffraction(ctx, f, nt, np_, cfg)
    assert out.stats == counts(out.transitions, out.results)
    assert out.stats["filtered_directions"] > 50000
    quiet = out.results["flags"] == 0
    assert (out.results["intensity_s"][quiet] == f["intensity_s"][quiet]).all()
    assert (out.results["sigma_rad"][quiet] == 0).all()
    rng = np.random.default_rng(4)
    changed = np.flatnonzero(~quiet)
    pick = np.unique(np.concatenate([rng.choice(changed, 2000, replace=False), rng.integers(0, nt * np_, 1000)]))
    cfg4 = (cfg.primary_sigma_rad, cfg.support_sigma, cfg.transition_contrast, cfg.inner_blend_sigma)
    edges = oracle.rainbow_detect(f, nt, np_, cfg4)
    assert np.array_equal(edges, out.transitions)
    want = oracle.rainbow_filter_at(f, edges, nt, np_, cfg4, pick)
    assert not mismatches(out.results[pick], want), mismatches(out.results[pick], want)
    flat = f.copy()
    flat["flags"] = 0
    flat["intensity_s"], flat["intensity_p"] = 2.5, 0.75
    const = icp.rainbow_diffraction(ctx, flat, nt, np_, cfg, transitions=out.transitions)
    filt = (const.results["flags"] & 1) != 0
    assert filt.sum() > 50000
    assert np.abs(const.results["intensity_s"][filt] - 2.5).max() <= 1e-14 * 3.5
    assert np.abs(const.results["intensity_p"][filt] - 0.75).max() <= 1e-14 * 1.75
