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
