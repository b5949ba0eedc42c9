"""Per-direction optics of the drop's wave stages on the CPU (no GPU): the oracle pinned bit
for bit to the reference's evaluator (tests/golden/optics_reference.npz, made by the
reference's own headers through oracle/ref_optics_harness.cpp), properties the reference's
optics tests state (tests/test_patch_optics_cpu.cpp, tests/test_wave_optics_cpu.cpp of the
reference), and the ABI record layouts."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

import optics_cases as OC
from conftest import GOLDEN, ROOT

Z = np.load(GOLDEN / "optics_reference.npz")


@pytest.mark.parametrize("name", [c[0] for c in OC.CASES])
def test_oracle_bit_identical_to_reference(oracle, name):
    c = dict(OC.CASES)[name]()
    assert OC.digest(c) == str(Z[f"{name}.digest"]), f"{name}: the input differs from the one the reference saw"
    out, focal = oracle.patch_optics(c)
    assert out.tobytes() == Z[f"{name}.optical"].tobytes()
    if c.focal:
        assert focal.tobytes() == Z[f"{name}.focal"].tobytes()


def test_fixtures_cover_every_outcome():
    flags = np.concatenate([Z[f"{n}.optical"]["flags"] for n, _ in OC.CASES])
    for bit in (1, 2, 4, 8, 32, 64, 128):  # query, input, frame, phase errors; the three pending kinds
        assert (flags & bit).any(), bit
    assert (flags == 0).sum() > 300
    focal = np.concatenate([Z[f"{n}.focal"]["flags"] for n, _ in OC.CASES if f"{n}.focal" in Z.files])
    for bit in (1, 2, 8):
        assert (focal & bit).any(), bit
    ok = Z["unpolarized_focal.focal"][Z["unpolarized_focal.focal"]["flags"] == 0]
    assert (ok["extra_quarter_turn_hits"] > 0).any() and (ok["family_hits"].sum(axis=0) > 0).all()


def test_unavailable_values_are_nan_and_focal_matches_path_counts(oracle):
    c = OC.lattice_case(1)
    out, focal = oracle.patch_optics(c)
    err = (out["flags"] & 31) != 0
    assert np.isnan(out["path_s"][err]).all() and np.isfinite(out["path_s"][~err]).all()
    good = focal["flags"] == 0
    assert np.isnan(focal["intensity_s"][~good]).all()
    # a valid focal direction counts every evaluated hit once, across the four families
    assert (focal["corrected_hits"][good] == out["evaluated_hits"][good]).all()
    assert (focal["family_hits"][good].sum(axis=1) == out["evaluated_hits"][good]).all()
    # quarter turns change phases only: the focal incoherent envelope is the path stage's
    inc = out["incoherent_s"][good] + out["incoherent_p"][good]
    assert np.allclose(focal["family_incoherent"][good].sum(axis=1), inc, rtol=1e-12, atol=0)


def test_single_hit_intensity_is_the_jacobian_weighted_field(oracle):
    """One regular hit: incoherent = (area / solid angle) x |interpolated field|^2 and the
    coherent path intensity equals it up to the binary32 phasor's modulus (cosf / sinf)."""
    c = OC.lattice_case(5, directions=60, faults=False)
    out, _ = oracle.patch_optics(c)
    one = np.flatnonzero((out["flags"] == 0) & (out["evaluated_hits"] == 1))
    assert one.size > 5
    for i in one:
        assert out["path_s"][i] == pytest.approx(out["incoherent_s"][i], rel=3e-7)
        assert out["path_p"][i] == pytest.approx(out["incoherent_p"][i], rel=3e-7)


def test_live_reference_on_fresh_lattices(oracle):
    if not oracle.ref_optics_available():
        pytest.skip("reference harness not built")
    for seed in (101, 102, 103):
        c = OC.lattice_case(seed, width=5 + seed % 4, height=6, directions=80, dual=seed % 2 == 1)
        ro, rf = oracle.ref_patch_optics(OC.serialize(c), c.count, True)
        oo, of = oracle.patch_optics(c)
        assert oo.tobytes() == ro.tobytes() and of.tobytes() == rf.tobytes()


def test_records_match_the_c_structs(icp, tmp_path):
    assert icp.VERTEX_DTYPE == OC.VERTEX_DTYPE and icp.PATCH_DTYPE == OC.PATCH_DTYPE
    assert icp.HIT_DTYPE == OC.HIT_DTYPE and icp.SUMMARY_DTYPE == OC.SUMMARY_DTYPE
    assert icp.OPTICAL_DTYPE == OC.OPTICAL_DTYPE
    fields = {"icp_outgoing_vertex": ("position_drop", "direction_drop", "basis_x", "field", "optical_cycles",
                                      "status", "diagnostics"),
              "icp_optical_result": ("path_field", "incoherent_s", "incoherent_p", "path_s", "path_p", "hit_count",
                                     "flags", "first_problem_patch_id", "folded_hits", "path_field_second"),
              "icp_query_hit": ("compact_index", "patch_id", "root_index", "flags", "u", "v", "t", "residual")}
    lines = [f'printf("{s} {f} %zu\\n", offsetof({s}, {f}));' for s, fs in fields.items() for f in fs]
    lines += [f'printf("{s} size %zu\\n", sizeof({s}));' for s in
              ("icp_outgoing_vertex", "icp_outgoing_patch", "icp_query_hit", "icp_query_summary", "icp_optical_result",
               "icp_focal_config", "icp_optics_input")]
    src = tmp_path / "layout.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "icp_b200.h"\nint main(void){\n' +
                   "\n".join(lines) + "\nreturn 0;}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = {tuple(x.split()[:2]): int(x.split()[2])
           for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines()}
    vmap = {"position_drop": "position", "direction_drop": "direction", "optical_cycles": "turns"}
    for f in fields["icp_outgoing_vertex"]:
        assert got[("icp_outgoing_vertex", f)] == icp.VERTEX_DTYPE.fields[vmap.get(f, f)][1], f
    for f in fields["icp_optical_result"]:
        assert got[("icp_optical_result", f)] == icp.OPTICAL_DTYPE.fields[f][1], f
    for f in fields["icp_query_hit"]:
        assert got[("icp_query_hit", f)] == icp.HIT_DTYPE.fields[f][1], f
    assert [got[(s, "size")] for s in ("icp_outgoing_vertex", "icp_outgoing_patch", "icp_query_hit",
                                       "icp_query_summary", "icp_optical_result", "icp_focal_config")] == \
        [68, 32, 32, 32, 136, 32]
    assert got[("icp_optics_input", "size")] == icp.C.sizeof(icp.OpticsInput)


# ------------------------------------------------------------------------ patch build
@pytest.mark.parametrize("name", [c[0] for c in OC.PATCH_CASES])
def test_patch_build_oracle_bit_identical_to_reference(oracle, name):
    import hashlib
    v, (w, h, e) = dict(OC.PATCH_CASES)[name]()
    blob = OC.serialize_lattice(v, (w, h, e))
    assert hashlib.sha256(blob).hexdigest() == str(Z[f"patch.{name}.digest"])
    st, pa, bx, hist = oracle.patch_build(v, w, h, e)
    assert np.array_equal(st, Z[f"patch.{name}.status"]) and np.array_equal(hist, Z[f"patch.{name}.histogram"])
    assert pa.tobytes() == Z[f"patch.{name}.patches"].tobytes() and bx.tobytes() == Z[f"patch.{name}.aabbs"].tobytes()


def test_patch_build_covers_every_status_and_orders_by_id():
    hist = sum(Z[f"patch.{n}.histogram"].astype(np.int64) for n, _ in OC.PATCH_CASES)
    assert (hist[1:] > 0).all()  # regular +/-, refinement, missing, none, invalid vertex / geometry
    for n, _ in OC.PATCH_CASES:
        p = Z[f"patch.{n}.patches"]
        assert (np.diff(p["patch_id"].astype(np.int64)) > 0).all()
        reg = np.isin(p["status"], (1, 2))
        assert np.isfinite(p["signed_solid_angle_sr"][reg]).all() and np.isnan(p["signed_solid_angle_sr"][~reg]).all()
        assert (np.sign(p["signed_solid_angle_sr"][reg]) == np.where(p["status"][reg] == 1, 1, -1)).all()


def test_patch_build_live_reference(oracle):
    if not oracle.ref_optics_available() or not (oracle.REF_DIR / "ref_patch_harness").exists():
        pytest.skip("reference harness not built")
    for seed in (31, 32):
        v, (w, h, e) = OC.patch_lattice(seed, width=6 + seed % 5, height=7)
        cells = 4 * (w - 1) * (h - 1)
        ref = oracle.ref_patch_build(OC.serialize_lattice(v, (w, h, e)), cells)
        got = oracle.patch_build(v, w, h, e)
        assert all(a.tobytes() == b.tobytes() for a, b in zip(got, ref))


# ----------------------------------------------------------------- patch query
def test_intersection_oracle_bit_identical_to_reference(oracle):
    import hashlib
    corners, dirs = OC.intersection_pairs()
    assert hashlib.sha256(corners.tobytes() + dirs.tobytes()).hexdigest() == str(Z["intersect.digest"])
    got = oracle.bilinear_intersect(corners, dirs)
    want = Z["intersect.hits"]
    assert got.tobytes() == want.tobytes()
    assert set(np.unique(want["count"])) == {0, 1, 2} and (want["flags"] & 2).any() and (want["flags"] & 4).any()


@pytest.mark.parametrize("grid", OC.DIRECTION_GRIDS, ids=lambda g: f"{g[0]}x{g[1]}")
def test_query_directions_bit_identical_to_reference(icp, grid):
    nt, np_, axis, e0 = grid
    got = icp.query_directions(nt, np_, np.float32(axis), np.float32(e0))
    assert got.tobytes() == Z[f"directions.{nt}x{np_}"].tobytes()


def test_query_directions_reject_a_bad_frame(icp):
    with pytest.raises(icp.InvalidArgument):
        icp.query_directions(4, 4, (0.0, 0.0, 1.0), (0.0, 0.1, 1.0))
    with pytest.raises(icp.InvalidArgument):
        icp.query_directions(0, 4, (0.0, 0.0, 1.0), (1.0, 0.0, 0.0))


def test_oracle_query_is_sorted_and_consistent(oracle, icp):
    v, (w, h, e) = OC.patch_lattice(21)
    st, pa, bx, hist = oracle.patch_build(v, w, h, e)
    dirs = icp.query_directions(36, 72, np.float32(OC._K20), np.float32((0, 0, 1)))
    off, sm, hits = oracle.patch_query(v, pa, bx, dirs)
    assert off[-1] == len(hits) and (sm["candidate_count"] == np.diff(off)).all()
    for i in np.flatnonzero(sm["hit_count"]):
        hs = hits[off[i]:off[i] + sm["hit_count"][i]]
        key = list(zip(hs["patch_id"], hs["compact_index"], hs["root_index"]))
        assert key == sorted(set(key))
        assert (hs["residual"] <= 2.0 ** -21).all() and (hs["t"] > 0).all() and (hs["t"] < 4).all()
        # every hit point lies on its patch: the bilinear point along the query direction
        for hit in hs:
            c = v["direction"][pa["vertex_indices"][hit["compact_index"]]].astype(np.float64)
            u, t = float(hit["u"]), float(hit["v"])
            p = ((1 - u) * c[0] + u * c[1]) * (1 - t) + ((1 - u) * c[2] + u * c[3]) * t
            assert np.allclose(p / np.linalg.norm(p), dirs[i], atol=1e-5)
    assert (sm["regular_hits"] + sm["refinement_hits"] == sm["hit_count"]).all()


def test_oracle_chain_lattice_to_diffraction(oracle, icp):
    """Lattice -> patches -> query -> optics (focal) -> Table-II diffraction, on the CPU."""
    import rainbow_cases  # noqa: F401  (the focal record layout)
    v, (w, h, e) = OC.patch_lattice(22, width=17, height=13, faults=False)
    st, pa, bx, hist = oracle.patch_build(v, w, h, e)
    k, e0 = np.float32(OC._K20), np.float32((0, 0, 1))
    nt, np_ = 45, 90
    dirs = icp.query_directions(nt, np_, k, e0)
    off, sm, hits = oracle.patch_query(v, pa, bx, dirs)
    case = OC.OpticsInput(v, pa, dirs, off, sm, hits, None, k, e0, 0, (w, h, e, (0, 0, 0, 0)))
    out, focal = oracle.patch_optics(case)
    lit = sm["hit_count"] > 0
    assert lit.sum() > 50 and (out["evaluated_hits"][lit] > 0).any()
    assert np.isfinite(out["incoherent_s"][out["flags"] == 0]).all()
    cfg = (2.0 * np.pi / 180, 4.0, 0.25, 3.0)
    edges = oracle.rainbow_detect(focal, nt, np_, cfg)
    res = oracle.rainbow_filter(focal, edges, nt, np_, cfg)
    assert len(res) == nt * np_


def test_density_gate_mirrors_the_reference(icp):
    ok = {"maximum": 2.0, "invalid_values": 0, "incomplete": 0, "underresolved": 0, "first_problem": 2 ** 64 - 1}
    icp.density_gate(ok)
    for bad in ({"invalid_values": 1}, {"incomplete": 3}, {"maximum": 0.0}, {"underresolved": 1}):
        with pytest.raises(icp.AuditError):
            icp.density_gate({**ok, **bad})
    icp.density_gate({**ok, "underresolved": 5}, allow_underresolved=True)
    assert icp.C.sizeof(icp.DensityReport) == 40 and icp.WAVE_STAGES["diffraction"] == 4


# ------------------------------------------------- the reference's own drop lattice
def reference_lattice():
    z = np.load(GOLDEN / "drop_lattice_reference.npz")
    w, h = (int(x) for x in z["shape"])
    f = z["frame"]
    return z["vertices"], z["second"], (w, h, float(f[0])), np.float32(f[1:4]), np.float32(f[4:7])


def oracle_chain(oracle, icp, nt=90, np_=180):
    v, second, (w, h, e), k, e0 = reference_lattice()
    st, pa, bx, hist = oracle.patch_build(v, w, h, e)
    dirs = icp.query_directions(nt, np_, k, e0)
    off, sm, hits = oracle.patch_query(v, pa, bx, dirs)
    case = OC.OpticsInput(v, pa, dirs, off, sm, hits, second, k, e0, 1, (w, h, e, (0, 0, 0, 0)))
    out, focal = oracle.patch_optics(case)
    return dict(v=v, second=second, layout=(w, h, e), k=k, e0=e0, patches=pa, boxes=bx, hist=hist, dirs=dirs,
                offsets=off, summaries=sm, hits=hits, out=out, focal=focal)


def test_reference_lattice_chain_on_the_cpu(oracle, icp):
    """The reference's unpolarized lattice trace of a 0.5 mm sphere through the oracle chain:
    every query direction of the 90 x 180 grid sees patches, all but the caustic's are complete,
    and the four families appear in the focal stage."""
    c = oracle_chain(oracle, icp)
    sm, out, focal = c["summaries"], c["out"], c["focal"]
    assert (sm["hit_count"] > 0).all()
    complete = ((out["flags"] & 255) == 0) & (out["rejected_hits"] == 0) & (out["evaluated_hits"] == out["hit_count"])
    assert complete.sum() > 0.99 * len(out)
    incomplete = np.flatnonzero(~complete)
    assert incomplete.size > 0 and (out["flags"][incomplete] & 32).all()  # refinement-pending: the folds
    assert (focal["family_hits"][complete].sum(axis=0) > 0).all()
    assert np.isfinite(out["path_s"][complete]).all() and (out["incoherent_s"][complete] > 0).all()
