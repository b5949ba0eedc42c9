"""Per-direction optics of the drop's wave stages on the GPU, through the C ABI, against the
reference's outputs (tests/golden/optics_reference.npz) and the oracle.

Tolerances are the reference's own for its CUDA evaluator against its host build: flags,
query flags and every hit counter exact; fields to 8e-6 x (1 + sqrt(incoherent) + |x|),
intensities to 8e-6 relative (tests/patch_optics_test_cases.hpp:19-23, 227-243 of the
reference); focal flags, counters and family hits exact, focal values to 2e-6 relative
(tests/wave_optics_test_cases.hpp:10-25).  The differences come from CUDA's cosf / sinf /
atan2 in the last ulps.
"""
from __future__ import annotations

import numpy as np
import pytest

import optics_cases as OC
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

Z = np.load(GOLDEN / "optics_reference.npz")
COUNTERS = ("flags", "query_flags", "hit_count", "evaluated_hits", "rejected_hits", "first_problem_patch_id",
            "refinement_hits", "boundary_hits", "singular_hits", "folded_hits")


def near(a, b, tol, scale=1.0):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.isfinite(a) & np.isfinite(b) & (np.abs(a - b) <= tol * (scale + np.abs(b)))


def optics_mismatch(got, want) -> list[str]:
    bad = [k for k in COUNTERS if not np.array_equal(got[k], want[k])]
    ok = (want["flags"] & 31) == 0
    if not np.isnan(got["path_s"][~ok]).all():
        bad.append("unavailable not NaN")
    g, w = got[ok], want[ok]
    scale = 1.0 + np.sqrt(w["incoherent_s"] + w["incoherent_p"])
    for k in ("path_field", "path_field_second"):
        if not near(g[k], w[k], 8e-6, scale[:, None]).all():
            bad.append(k)
    for k in ("incoherent_s", "incoherent_p"):
        if not near(g[k], w[k], 8e-6).all():
            bad.append(k)
    for k in ("path_s", "path_p"):
        if not near(g[k], w[k], 8e-6, scale * scale).all():
            bad.append(k)
    return bad


def focal_mismatch(got, want) -> list[str]:
    bad = [k for k in ("flags", "corrected_hits", "extra_quarter_turn_hits", "first_problem_patch_id", "family_hits")
           if not np.array_equal(got[k], want[k])]
    ok = want["flags"] == 0
    if not np.isnan(got["intensity_s"][~ok]).all():
        bad.append("unavailable not NaN")
    for k in ("family_incoherent", "intensity_s", "intensity_p", "field", "field_second"):
        if not near(got[k][ok], want[k][ok], 2e-6).all():
            bad.append(k)
    return bad


def run(icp, ctx, c):
    return icp.patch_optics(ctx, c.vertices, c.patches, c.directions, c.offsets, c.summaries, c.hits, c.incident,
                            c.basis, second=c.second, polarization=c.polarization, focal=c.focal)


@pytest.mark.parametrize("name", [c[0] for c in OC.CASES])
def test_fixture_cases_match_reference(icp, ctx, name):
    c = dict(OC.CASES)[name]()
    assert OC.digest(c) == str(Z[f"{name}.digest"])
    before = icp.kernel_launches()
    out, focal = run(icp, ctx, c)
    assert icp.kernel_launches() - before == 1
    bad = optics_mismatch(out, Z[f"{name}.optical"])
    assert not bad, bad
    if c.focal:
        bad = focal_mismatch(focal, Z[f"{name}.focal"])
        assert not bad, bad


def test_large_lattice_against_oracle(icp, ctx, oracle):
    """A 129 x 129 lattice (66 564 vertices, 65 536 patches) queried in 20 000 directions."""
    c = OC.lattice_case(77, width=129, height=129, directions=20000)
    out, focal = run(icp, ctx, c)
    want, wfocal = oracle.patch_optics(c)
    assert not optics_mismatch(out, want)
    assert not focal_mismatch(focal, wfocal)
    assert (out["flags"] == 0).sum() > 5000


def test_focal_feeds_the_diffraction_pass(icp, ctx, oracle):
    """The focal stage's output is the diffraction pass's input, unchanged (one query grid)."""
    c = OC.lattice_case(9, directions=12 * 24, faults=False)
    _, focal = run(icp, ctx, c)
    cfg = icp.DiffractionConfig(3.0 * np.pi / 180, 4.0, 0.25, 3.0)
    d = icp.rainbow_diffraction(ctx, focal, 12, 24, cfg)
    edges = oracle.rainbow_detect(focal, 12, 24, (cfg.primary_sigma_rad, 4.0, 0.25, 3.0))
    assert np.array_equal(d.transitions, edges)


@pytest.mark.parametrize("name", [c[0] for c in OC.PATCH_CASES])
def test_patch_build_matches_reference(icp, ctx, name):
    """Statuses, order, corner indices, areas and boxes exact; the solid angle to 4 ulps
    (CUDA's atan2f)."""
    v, (w, h, e) = dict(OC.PATCH_CASES)[name]()
    before = icp.kernel_launches()
    got = icp.patch_build(ctx, v, w, h, e)
    assert icp.kernel_launches() - before == 3
    want = Z[f"patch.{name}.patches"]
    assert np.array_equal(got.statuses.astype(np.uint8), Z[f"patch.{name}.status"])
    assert got.histogram == [int(x) for x in Z[f"patch.{name}.histogram"]]
    assert len(got.patches) == len(want)
    for k in ("vertex_indices", "patch_id", "status", "incident_area_drop2"):
        assert np.array_equal(got.patches[k], want[k]), k
    a, b = got.patches["signed_solid_angle_sr"], want["signed_solid_angle_sr"]
    reg = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), reg)
    assert (np.abs(a[reg] - b[reg]) <= 4 * np.spacing(np.abs(b[reg]).astype(np.float32))).all()
    assert got.aabbs.tobytes() == Z[f"patch.{name}.aabbs"].tobytes()


def test_patch_build_large_lattice_against_oracle(icp, ctx, oracle):
    """A 257 x 257 lattice (262 144 cells, 1024 blocks: a multi-chunk block-count scan)."""
    v, (w, h, e) = OC.patch_lattice(41, width=257, height=257)
    got = icp.patch_build(ctx, v, w, h, e)
    st, pa, bx, hist = oracle.patch_build(v, w, h, e)
    assert np.array_equal(got.statuses, st) and got.histogram == [int(x) for x in hist]
    assert np.array_equal(got.patches["patch_id"], pa["patch_id"]) and got.aabbs.tobytes() == bx.tobytes()


def _query_case(seed, width, height, nt, np_):
    import ice_crystal_phase_b200 as icp
    v, (w, h, e) = OC.patch_lattice(seed, width=width, height=height)
    dirs = icp.query_directions(nt, np_, np.float32(OC._K20), np.float32((0, 0, 1)))
    return v, (w, h, e), dirs


@pytest.mark.parametrize("seed,width,height,nt,np_", [(21, 9, 8, 36, 72), (24, 33, 5, 60, 120), (41, 65, 65, 90, 180)])
def test_patch_query_bit_identical_to_oracle(icp, ctx, oracle, seed, width, height, nt, np_):
    """The binned device query equals the brute-force oracle (every patch box tested) bit for
    bit: offsets, summaries and hits."""
    v, (w, h, e), dirs = _query_case(seed, width, height, nt, np_)
    st, pa, bx, hist = oracle.patch_build(v, w, h, e)
    got = icp.patch_query(ctx, v, pa, bx, dirs)
    off, sm, hits = oracle.patch_query(v, pa, bx, dirs)
    assert np.array_equal(got.offsets, off)
    assert got.summaries.tobytes() == sm.tobytes()
    assert got.hits.tobytes() == hits.tobytes()
    assert len(hits) > 0


def test_device_chain_lattice_to_diffraction(icp, ctx, oracle):
    """Patch build, query, optics and diffraction chained on the device from one lattice,
    against the same chain in the oracle."""
    v, (w, h, e) = OC.patch_lattice(22, width=17, height=13, faults=False)
    k, e0 = np.float32(OC._K20), np.float32((0, 0, 1))
    nt, np_ = 45, 90
    dirs = icp.query_directions(nt, np_, k, e0)
    pb = icp.patch_build(ctx, v, w, h, e)
    q = icp.patch_query(ctx, v, pb.patches, pb.aabbs, dirs)
    out, focal = icp.patch_optics(ctx, v, pb.patches, dirs, q.offsets, q.summaries, q.hits, k, e0,
                                  focal=(w, h, e, (0, 0, 0, 0)))
    st, pa, bx, hist = oracle.patch_build(v, w, h, e)
    off, sm, hits = oracle.patch_query(v, pa, bx, dirs)
    assert q.hits.tobytes() == hits.tobytes()
    case = OC.OpticsInput(v, pa, dirs, off, sm, hits, None, k, e0, 0, (w, h, e, (0, 0, 0, 0)))
    want, wfocal = oracle.patch_optics(case)
    assert not optics_mismatch(out, want)
    assert not focal_mismatch(focal, wfocal)
    cfg = icp.DiffractionConfig(2.0 * np.pi / 180, 4.0, 0.25, 3.0)
    d = icp.rainbow_diffraction(ctx, focal, nt, np_, cfg)
    assert np.array_equal(d.transitions, oracle.rainbow_detect(wfocal, nt, np_, (cfg.primary_sigma_rad, 4.0, 0.25, 3.0)))


def test_stage_density_and_audit(icp, ctx):
    """Densities and the CDF input audit of every stage against the predicates of the
    reference's density() and phase_check_density, on a faulty case (incomplete directions)."""
    c = OC.lattice_case(1)
    out, focal = run(icp, ctx, c)
    n = c.count
    cfg = icp.DiffractionConfig(3.0 * np.pi / 180, 4.0, 0.25, 3.0)
    d = icp.rainbow_diffraction(ctx, focal, 10, n // 10, cfg) if n % 10 == 0 else None
    complete = ((out["flags"] & 255) == 0) & (out["rejected_hits"] == 0) & (out["evaluated_hits"] == out["hit_count"])
    for stage in ("incoherent", "path", "focal") + (("diffraction",) if d else ()):
        dens, rep = icp.stage_density(ctx, stage, out, focal, d.results if d else None)
        got = dens.download()
        if stage == "incoherent":
            want, inc, under = out["incoherent_s"] + out["incoherent_p"], ~complete, np.zeros(n, bool)
        elif stage == "path":
            want, inc, under = out["path_s"] + out["path_p"], ~complete, np.zeros(n, bool)
        elif stage == "focal":
            want, inc, under = focal["intensity_s"] + focal["intensity_p"], ~complete | (focal["flags"] != 0), np.zeros(n, bool)
        else:
            r = d.results
            want = r["intensity_s"] + r["intensity_p"]
            inc = ~complete | (focal["flags"] != 0) | ((r["flags"] & 60) != 0)
            under = (r["flags"] & 2) != 0
        assert np.array_equal(np.isnan(got), np.isnan(want)) and np.array_equal(got[~np.isnan(want)], want[~np.isnan(want)])
        bad = ~np.isfinite(want) | (want < 0)
        assert rep["invalid_values"] == bad.sum() and rep["incomplete"] == inc.sum() and rep["underresolved"] == under.sum()
        assert rep["maximum"] == (want[~bad].max() if (~bad).any() else 0.0)
        probs = np.flatnonzero(bad | inc | under)
        assert rep["first_problem"] == (probs[0] if probs.size else 2 ** 64 - 1)
    with pytest.raises(icp.AuditError):
        icp.stage_record(ctx, "path", 10, n // 10, out)


def test_reference_lattice_device_chain(icp, ctx, oracle):
    """The reference's own lattice trace of a 0.5 mm sphere through the whole device chain --
    patch build, query, optics with the focal stage, Table-II diffraction, stage densities --
    against the oracle chain."""
    import test_optics_cpu as T
    c = T.oracle_chain(oracle, icp)
    v, second, (w, h, e), k, e0 = T.reference_lattice()
    pb = icp.patch_build(ctx, v, w, h, e)
    assert list(pb.histogram) == [int(x) for x in c["hist"]]
    assert np.array_equal(pb.patches["patch_id"], c["patches"]["patch_id"]) and pb.aabbs.tobytes() == c["boxes"].tobytes()
    q = icp.patch_query(ctx, v, c["patches"], c["boxes"], c["dirs"])
    assert q.hits.tobytes() == c["hits"].tobytes() and q.summaries.tobytes() == c["summaries"].tobytes()
    out, focal = icp.patch_optics(ctx, v, c["patches"], c["dirs"], q.offsets, q.summaries, q.hits, k, e0,
                                  second=second, focal=(w, h, e, (0, 0, 0, 0)))
    assert not optics_mismatch(out, c["out"])
    assert not focal_mismatch(focal, c["focal"])
    cfg = icp.diffraction_config(0.5)
    d = icp.rainbow_diffraction(ctx, focal, 90, 180, cfg)
    c4 = (cfg.primary_sigma_rad, cfg.support_sigma, cfg.transition_contrast, cfg.inner_blend_sigma)
    assert np.array_equal(d.transitions, oracle.rainbow_detect(c["focal"], 90, 180, c4))
    for stage in ("incoherent", "path", "focal", "diffraction"):
        _, rep = icp.stage_density(ctx, stage, out, focal, d.results)
        assert rep["incomplete"] > 0  # the caustic's refinement-pending directions
