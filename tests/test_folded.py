"""Folded patches of the drop's wave stages against the REFERENCE (tests/golden/folded_reference.npz,
written by tests/golden/make_folded_fixtures.py with FoldedPatchBuilder::prepare and
PatchOpticalEvaluator::evaluate_direction over a FoldedPatchView, compiled from the reference's
sources, on the reference's own lattices of three drops).

On the GPU the whole chain runs on the device -- lattice trace, patch build, query directions,
all-hit query -- and must hand the optics an input byte-identical to the reference's chain (its
SHA-256); the folded records must then equal the reference's bit for bit (binary64 quadrature,
no transcendental functions; the focal quarter turns use atan2 and must agree exactly), every
direction's counters and flags exactly, and the fields and intensities of the directions with
refinement hits within the tolerances of the other optics tests (CUDA's cosf / sinf / atan2).
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

import optics_cases as OC
from conftest import GOLDEN

Z = np.load(GOLDEN / "folded_reference.npz")
NAMES = [k[:-len(".args")] for k in Z.files if k.endswith(".args")]
OPTICAL_COUNTERS = ("hit_count", "evaluated_hits", "rejected_hits", "refinement_hits", "boundary_hits",
                    "singular_hits", "flags", "query_flags", "first_problem_patch_id", "folded_hits")
FOCAL_COUNTERS = ("family_hits", "corrected_hits", "extra_quarter_turn_hits", "flags", "first_problem_patch_id")


def counters_digest(optical, focal) -> str:
    h = hashlib.sha256()
    for k in OPTICAL_COUNTERS:
        h.update(np.ascontiguousarray(optical[k]).tobytes())
    for k in FOCAL_COUNTERS:
        h.update(np.ascontiguousarray(focal[k]).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("name", NAMES)
def test_fixture_records_are_indexed_in_compact_order(icp, name):
    rec, idx = Z[f"{name}.records"], Z[f"{name}.record_indices"]
    assert rec.dtype.itemsize == icp.FOLDED_DTYPE.itemsize == 320
    assert np.all(np.diff(rec["compact_index"].astype(np.int64)) > 0)
    assert np.array_equal(idx[rec["compact_index"]], np.arange(len(rec)))
    assert int((idx != 0xFFFFFFFF).sum()) == len(rec)
    ready = rec["flags"] == 0
    assert ready.any() and (rec["branch_count"][ready] >= 2).all()
    # the branches partition the parameter square: area fractions sum to one within 8 x tolerance
    area = np.array([rec["branches"]["area_fraction"][i, :rec["branch_count"][i]].sum() for i in np.flatnonzero(ready)])
    assert np.all(np.abs(area - 1) <= 8e-8)


def _near(a, b, tol, scale=1.0):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.isfinite(a) & np.isfinite(b) & (np.abs(a - b) <= tol * (scale + np.abs(b)))


def _device_chain(icp, ctx, name):
    a = str(Z[f"{name}.args"]).split()
    nt, np_ = (int(x) for x in Z[f"{name}.query"])
    coef = [float(x) for x in a[8:16]] if len(a) > 8 else None
    wavelength = float(a[7]) if len(a) > 7 else 700.0
    cfg = icp.raindrop_config(float(a[0]), wavelength, float(a[2]), tuple(float(x) for x in a[3:6]), int(a[6]),
                              sphere=a[1] == "1", coefficients=coef)
    lat = icp.lattice_trace(ctx, cfg)
    w, h, e = cfg.grid_width, cfg.grid_height, cfg.grid_half_extent
    v = lat.vertices.download()
    second = lat.second.download().reshape(-1, 4)
    pb = icp.patch_build(ctx, lat.vertices, w, h, e)
    k = np.array([cfg.incident_direction.x, cfg.incident_direction.y, cfg.incident_direction.z], np.float32)
    e0 = np.array([cfg.incident_basis_x.x, cfg.incident_basis_x.y, cfg.incident_basis_x.z], np.float32)
    dirs = icp.query_directions(nt, np_, k, e0)
    q = icp.patch_query(ctx, v, pb.patches, pb.aabbs, dirs)
    return OC.OpticsInput(v, pb.patches, dirs, q.offsets, q.summaries, q.hits, second, k, e0, 1,
                          (w, h, float(np.float32(e)), (0, 0, 0, 0)))


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_device_chain_folded_optics_match_reference(icp, name):
    with icp.Context(0) as ctx:
        c = _device_chain(icp, ctx, name)
        assert OC.digest(c) == str(Z[f"{name}.digest"]), "the device chain's optics input differs"
        out, focal, folded = icp.patch_optics(ctx, c.vertices, c.patches, c.directions, c.offsets, c.summaries,
                                              c.hits, c.incident, c.basis, second=c.second, focal=c.focal,
                                              folded=True)
    want = Z[f"{name}.records"]
    assert folded.records.tobytes() == want.tobytes()
    assert np.array_equal(folded.indices, Z[f"{name}.record_indices"])
    st = folded.stats
    assert (st.candidates, st.prepared, st.unresolved) == (len(want), int((want["flags"] == 0).sum()),
                                                           int((want["flags"] != 0).sum()))
    ready = want[want["flags"] == 0]
    assert st.branch_count == int(ready["branch_count"].sum())
    assert st.largest_estimated_relative_error == float(ready["largest_estimated_relative_error"].max())
    assert counters_digest(out, focal) == str(Z[f"{name}.counters_sha256"])
    r = Z[f"{name}.refined"]
    got, ref = out[r], Z[f"{name}.optical"]
    assert (ref["folded_hits"] > 0).any() and np.array_equal(got["folded_hits"], ref["folded_hits"])
    ok = (ref["flags"] & 31) == 0
    scale = 1.0 + np.sqrt(ref["incoherent_s"] + ref["incoherent_p"])
    for k in ("path_field", "path_field_second"):
        assert _near(got[k][ok], ref[k][ok], 8e-6, scale[ok][:, None]).all(), k
    for k in ("incoherent_s", "incoherent_p"):
        assert _near(got[k][ok], ref[k][ok], 8e-6).all(), k
    for k in ("path_s", "path_p"):
        assert _near(got[k][ok], ref[k][ok], 8e-6, (scale * scale)[ok]).all(), k
    fg, fr = focal[r], Z[f"{name}.focal"]
    fok = fr["flags"] == 0
    for k in ("family_incoherent", "intensity_s", "intensity_p", "field", "field_second"):
        assert _near(fg[k][fok], fr[k][fok], 2e-6).all(), k


@pytest.mark.gpu
def test_folded_records_off_leaves_refinement_pending(icp):
    """Without records a refinement hit stays pending (icp_patch_optics), as the reference's
    evaluate_patch_optics does; with records the same directions complete."""
    name = NAMES[0]
    with icp.Context(0) as ctx:
        c = _device_chain(icp, ctx, name)
        plain, _ = icp.patch_optics(ctx, c.vertices, c.patches, c.directions, c.offsets, c.summaries, c.hits,
                                    c.incident, c.basis, second=c.second, focal=c.focal)
    r = Z[f"{name}.refined"]
    assert ((plain["flags"][r] & 32) != 0).all()
    assert ((Z[f"{name}.optical"]["flags"] & 32) == 0).all()


@pytest.mark.gpu
def test_folded_prepare_capacity_and_config(icp):
    name = NAMES[0]
    with icp.Context(0) as ctx:
        c = _device_chain(icp, ctx, name)
        dv = icp.DeviceArray(ctx, len(c.vertices), icp.VERTEX_DTYPE).upload(c.vertices)
        dp = icp.DeviceArray(ctx, len(c.patches), icp.PATCH_DTYPE).upload(c.patches)
        di = icp.DeviceArray(ctx, len(c.patches), np.uint32)
        n = icp.C.c_uint32(0)
        k = (icp.C.c_float * 3)(*map(float, c.incident))
        rc = icp.LIB.icp_folded_prepare(ctx.handle, dv.ptr, len(c.vertices), dp.ptr, len(c.patches), k, None, None,
                                        di.ptr, None, 0, icp.C.byref(n), None)
        assert rc == icp.ICP_ERR_CAPACITY and n.value == len(Z[f"{name}.records"])
        bad = icp.FoldedConfig(1e-2, 2048, 20)
        with pytest.raises(icp.InvalidArgument):
            icp.folded_prepare(ctx, dv, dp, len(c.patches), c.incident, config=bad)
