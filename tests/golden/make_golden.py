"""Regenerates the golden fixtures in tests/golden/ from the REFERENCE implementation.

Runs the reference's own CPU code, compiled from its sources by oracle/build_ref.sh into
oracle/_ref/ (ice_generate_phase_cpu and the ref_*_harness drivers), imports the reference's
Python atlas composition (hex_atlas/python/atlas_math.py),
and stores its outputs as small .npz files.  Needs the reference checkout (the first argument, else
$ICP_REFERENCE_ROOT, else /root/reference);
the fixtures are committed so that tests never need it.

    python tests/golden/make_golden.py [REFERENCE_ROOT]
"""
from __future__ import annotations

import json
import math
import subprocess
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REF = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(os.environ.get("ICP_REFERENCE_ROOT", "/root/reference"))
REF_BIN = ROOT / "oracle" / "_ref"

# The reference's CLI test plan (hex_phase/configs/two_orientations.csv), reproduced as data:
# identity and an active +90 degree rotation about +z; 1024 and 2048 rays.
TWO_ORIENTATIONS = ("qw,qx,qy,qz,weight,samples,seed\n"
                    "1,0,0,0,0.5,1024,12345\n"
                    "0.7071067811865475244,0,0,0.7071067811865475244,0.5,2048,54321\n")
# Hex column: circumradius 0.05 mm, length 0.2 mm, n = 1.31, ki = (cos30, -sin30, 0).
COLUMN_PLAN = "qw,qx,qy,qz,weight,samples,seed\n1,0,0,0,1,20000,12345\n"


def run(cmd):
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode:
        raise SystemExit(f"{cmd[0]} failed: {r.stderr}")
    return r


def masses(td: Path, R, L, ki, n, nt, np_, plan: str, max_hits=1024, tail=1e-12, batch=4096):
    csv = td / "plan.csv"
    csv.write_text(plan)
    out = td / "m.bin"
    run([REF_BIN / "ref_hex_harness", "masses", repr(R), repr(L), *map(repr, ki), repr(n), "1", nt, np_, max_hits,
         repr(tail), csv, batch, out])
    raw = out.read_bytes()
    k = nt * np_
    return (np.frombuffer(raw[:8 * k], "<f8").copy(), np.frombuffer(raw[8 * k:8 * k + 72], "<f8").copy(),
            np.frombuffer(raw[8 * k + 72:], "<u8").copy())


def lines(mode: str, rows: list[str]) -> np.ndarray:
    r = subprocess.run([str(REF_BIN / "ref_drop_harness"), mode], input="\n".join(rows) + "\n", capture_output=True,
                       text=True, check=True)
    return np.array([[float(x) for x in line.split()] for line in r.stdout.splitlines()])


# Four-family configurations: radius, sphere, interior index, incident direction, lattice size.
FAMILY_CASES = [(0.4, 0, 1.3314, (1.0, -0.3, 0.1), 21), (1.5, 0, 1.3314, (0.9396926, -0.3420201, 0.0), 21),
                (3.0, 0, 1.3435, (1.0, -0.3, 0.1), 21)]


def drop_fixtures(td: Path) -> None:
    alphas = np.array([0.0, 20.0, -35.5, 45.0, 89.0, 120.0])
    frame = lines("frame", [repr(float(a)) for a in alphas])
    radii = np.array([0.05, 0.4, 0.41, 0.7, 1.0, 1.5, 1.73, 2.0, 2.5, 2.9, 3.0])
    shape = lines("shape", [f"{r} 0" for r in radii])
    water_in = np.array([[l, t, p] for l in (400.0, 550.0, 700.0, 1000.0) for t in (0.0, 20.0, 45.0, 60.0)
                         for p in (5e4, 101325.0, 1e7, 1e8)])
    water = lines("water", [f"{float(l)!r} {float(t)!r} {float(p)!r}" for l, t, p in water_in])
    ks = np.array([[1.0, 0.0, 0.0], [0.9396926164627075, -0.3420201539993286, 0.0], [0.0, 1.0, 0.0],
                   [0.3, -0.8, 0.52]])
    area_in = []
    for c in shape[[3, 5, 8, 10], :8]:
        for k in ks:
            area_in.append([*c, 1.5, *k])
    area_in.append([0, -0.08, -0.02, 0.005, 0, 0, 0, 0, 1.5, *ks[1]])
    area_in = np.array(area_in)
    area = lines("area", [" ".join(repr(float(x)) for x in row) for row in area_in])[:, 0]
    fam = {}
    for i, (r, sph, n, k, g) in enumerate(FAMILY_CASES):
        out = td / "f.bin"
        run([REF_BIN / "ref_drop_harness", "families", repr(r), sph, repr(n), *map(repr, k), g, out])
        a = np.fromfile(out, "<f8").reshape(-1, 41)
        power = a[:, [16, 24, 32, 40]]
        geom = np.delete(a, [16, 24, 32, 40], axis=1).astype(np.float32)  # binary32 values of the tracer
        fam[f"families{i}_geom"] = geom
        fam[f"families{i}_power"] = power
    np.savez_compressed(HERE / "drop_reference.npz", frame_alpha=alphas, frame=frame, shape_radius=radii,
                        shape=shape, water_in=water_in, water=water, area_in=area_in, area=area,
                        family_cases=np.array([[r, s, n, *k, g] for r, s, n, k, g in FAMILY_CASES]), **fam)


def ice_fixtures() -> None:
    """Ice Ih index (hex_atlas/src/ice_optics.cpp) at every table wavelength in range, the
    geometric midpoints, 400 seeded random wavelengths and the domain edges, exact."""
    knots = [199, 201, 201.9, 210, 250, 300, 350, 390, 400] + list(range(410, 1101, 10))
    wl = [float(k) for k in knots] + [math.sqrt(a * b) for a, b in zip(knots, knots[1:])]
    wl += [float(x) for x in np.random.default_rng(2008).uniform(200.0, 1100.0, 400)]
    wl += [200.0, 1100.0, 199.99999, 1100.00001, 0.0, -5.0, math.inf, math.nan, 555.5, 1099.9999999]
    r = subprocess.run([str(REF_BIN / "ref_ice_harness")], input="\n".join(repr(x) for x in wl) + "\n",
                       capture_output=True, text=True, check=True)
    status, vals = [], []
    for line in r.stdout.splitlines():
        f = line.split()
        if f[0] == "ok":
            status.append(0)
            vals.append([float.fromhex(x) for x in f[1:]])
        else:
            status.append(1 if f[0] == "invalid" else 2)
            vals.append([math.nan] * 5)
    assert len(status) == len(wl)
    np.savez_compressed(HERE / "ice_wb2008.npz", wavelength_nm=np.array(wl), status=np.array(status),
                        values=np.array(vals))


# Area quadratures: circumradius, length, incident direction, subdivisions.
ATLAS_AREA_CASES = [(0.1, 0.7, (1.0, 0.0, 0.0), 3), (0.1, 0.7, (0.0, 1.0, 0.0), 3), (0.1, 0.7, (1.0, 2.0, 3.0), 3),
                    (0.1, 0.7, (-1.0, -0.001, -0.9), 3), (0.05, 0.2, (0.8660254037844387, -0.5, 0.0), 2),
                    (0.1, 0.2, (0.3, 0.2, -0.9), 5), (0.1, 0.2, (0.0, 0.0, 1.0), 1)]
# Atlases: R, L, n_int, n_ext, nm, theta intervals, phi intervals, nt, np, S, max hits, tail.  The
# first is the reference's own atlas test setting (hex_atlas/tests/atlas_tests.cpp:12-16); the
# second is the atlas the composition fixtures are built on.
ATLAS_NODE_CASES = [(0.1, 0.2, 1.31, 1.0, 550.0, 3, 2, 12, 24, 2, 2048, 1e-12),
                    (0.05, 0.2, 1.31, 1.0, 550.0, 6, 3, 16, 32, 2, 2048, 1e-12)]
# Orientation models of the composition fixtures (the reference's own model kinds).
ATLAS_RULES = [
    {"quadrature": {"azimuth": 8, "tilt": 4, "spin": 3},
     "components": [{"kind": "horizontal_gaussian", "sigma_deg": 10, "fraction": 0.9},
                    {"kind": "isotropic", "fraction": 0.1}]},
    {"quadrature": {"azimuth": 3, "tilt": 5, "spin": 2},
     "components": [{"kind": "fixed", "fraction": 0.4,
                     "quaternion_wxyz": [0.9238795325112867, 0.0, 0.3826834323650898, 0.0]},
                    {"kind": "isotropic", "fraction": 0.6}]},
]
ATLAS_INCIDENTS = [(1.0, 0.0, 0.0), (0.8660254037844387, -0.5, 0.0), (0.0, -1.0, 0.0), (1.0, -0.4, 0.3),
                   (0.7071067811865476, 0.7071067811865476, 0.0)]


def atlas_fixtures(td: Path) -> None:
    """Deterministic atlas: the reference's area rule and traced nodes (hex_atlas/src/atlas.cpp),
    then its orientation composition (hex_atlas/python/atlas_math.py, imported from the
    reference checkout) on the second atlas."""
    out: dict[str, np.ndarray] = {}
    faces, pos, wts, off = [], [], [], [0]
    for R, L, k, S in ATLAS_AREA_CASES:
        r = subprocess.run([str(REF_BIN / "ref_atlas_harness"), "area", repr(R), repr(L), *map(repr, k), str(S)],
                           capture_output=True, text=True, check=True)
        rows = [line.split() for line in r.stdout.splitlines()]
        assert rows and rows[0][0] != "error", r.stdout
        faces += [int(x[0]) for x in rows]
        pos += [[float.fromhex(v) for v in x[1:4]] for x in rows]
        wts += [float.fromhex(x[4]) for x in rows]
        off.append(len(faces))
    out.update(area_cases=np.array([[R, L, *k, S] for R, L, k, S in ATLAS_AREA_CASES]), area_offsets=np.array(off),
               area_face=np.array(faces, np.uint32), area_pos=np.array(pos), area_weight=np.array(wts))
    atlases = []
    for c, case in enumerate(ATLAS_NODE_CASES):
        R, L, n, ne, nm, T, P, nt, np_, S, hits, tail = case
        f = td / "atlas.bin"
        run([REF_BIN / "ref_atlas_harness", "nodes", repr(R), repr(L), repr(n), repr(ne), repr(nm), T, P, nt, np_, S,
             hits, repr(tail), f])
        raw = np.fromfile(f, "<f8").reshape((T + 1) * (P + 1), 16 + nt * np_)
        out[f"nodes{c}_case"] = np.array(case, dtype=np.float64)
        out[f"nodes{c}_head"] = raw[:, :16]
        out[f"nodes{c}_mass"] = raw[:, 16:].reshape(T + 1, P + 1, nt, np_)
        atlases.append((case, raw))
    # composition on the second atlas, through the reference's own Python operator
    sys.path.insert(0, str(REF / "hex_atlas" / "python"))
    import atlas_math as am  # noqa: E402  (reference module, test-fixture generation only)
    from types import SimpleNamespace
    (R, L, _, _, _, T, P, nt, np_, _, _, _), raw = atlases[1]
    head = raw[:, :16].reshape(T + 1, P + 1, 16)
    edges = u_edges_ref(nt)
    atlas = SimpleNamespace(it=T, ip=P, nt=nt, np=np_, area=head[:, :, 8].copy(), residual=head[:, :, 10].copy(),
                            mass=raw[:, 16:].reshape(T + 1, P + 1, nt, np_), radius=R, length=L, edges=edges)
    for ri, rule in enumerate(ATLAS_RULES):
        rot, w, meta = am.orientation_rule(rule)
        out[f"rule{ri}_rotations"], out[f"rule{ri}_weights"] = rot, w
        out[f"rule{ri}_tilts"] = am.gaussian_tilt_nodes(rule["quadrature"]["tilt"], 10) if ri == 0 else np.zeros(0)
        for ki_index, ki in enumerate(ATLAS_INCIDENTS):
            c, area, frame, info = am.coupling_for_rule(atlas, rot, w, ki, meta)
            mass, residual = am.compose_mass(atlas, c)
            a, b, rep = am.make_cdf(mass, edges)
            key = f"compose{ri}_{ki_index}"
            out[key + "_coupling"] = c
            out[key + "_scalars"] = np.array([area, residual, rep["g"], rep["cdf_l1_mass_error"],
                                              float(info["method"].startswith("analytic"))])
            out[key + "_frame"] = frame
            out[key + "_mass"] = mass
            out[key + "_phi"] = a
            out[key + "_theta"] = b
    out["compose_incidents"] = np.array(ATLAS_INCIDENTS)
    out["compose_edges"] = edges
    np.savez_compressed(HERE / "atlas_reference.npz", **out)


def u_edges_ref(nt: int) -> np.ndarray:
    """u edges of the atlas grid as the reference's precompute stores them (make_phase_u_edges)."""
    r = subprocess.run([str(REF_BIN / "ref_atlas_harness"), "edges", str(nt)], capture_output=True, text=True,
                       check=True)
    return np.array([float.fromhex(x) for x in r.stdout.split()])


def compare_fixtures(td: Path) -> None:
    """The reference's record-vs-record metric (tools/phase_analysis.py compare_tables) on two
    records of one 64 x 128 grid: the TV judge of the learned surrogate's records."""
    sys.path.insert(0, str(REF / "tools"))
    sys.path.insert(0, str(REF / "python"))
    sys.path.insert(0, str(ROOT))
    import phase_analysis as pa  # noqa: E402  (reference module, test-fixture generation only)
    from oracle import atlas_oracle as AO

    nt, np_ = 64, 128
    edges = u_edges_ref(nt)
    rng = np.random.default_rng(44)
    base = rng.gamma(0.5, size=(nt, np_)) * np.diff(edges)[:, None]
    base[:, 7] = 0.0
    other = base * np.exp(0.05 * rng.normal(size=base.shape))
    other[3, :] *= 1.3
    out = {}
    for name, mass in (("a", base), ("b", other)):
        phi, theta, rep = AO.make_cdf(mass, edges)
        d = td / f"rec_{name}"
        d.mkdir()
        np.save(d / "phi_cdf.npy", phi)
        np.save(d / "theta_given_phi_cdf.npy", theta)
        np.save(d / "u_edges.npy", edges)
        q = np.diff(phi)[:, None] * np.diff(theta, axis=1)
        mu = 1.0 - (edges[:-1] + edges[1:])
        g = float(np.sum(q * mu[None, :], dtype=np.longdouble) / np.sum(q, dtype=np.longdouble))
        meta = {"schema": "rainbow.phase_cdf.numpy.v2", "complete": True, "dtype": "<f8", "order": "C",
                "theta_count": nt, "phi_count": np_, "density_measure": "solid_angle_sr",
                "cell_model": "constant_density_per_spherical_cell",
                "coordinates": "u=(1-cos(theta))/2; v=(phi+pi)/(2*pi)", "cdf_axis_order": ["phi_cell", "theta_edge"],
                "normalization": "integral_p_domega_equals_one", "input_polarization": "unpolarized",
                "direction_convention": "physical_propagation", "theta_zero": "forward", "theta_pi": "backward",
                "coordinate_contract_id": "rainbow.phase_cdf.coordinates.v1",
                "sampling_frame_map": "local_column_to_particle_column",
                "sampling_frame_columns": [[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]],
                "hg": {"g": g, "method": "first_moment_of_saved_cell_pdf", "target": "saved_cdf",
                       "cosine_convention": "dot(incident_propagation,outgoing_propagation)"}}
        (d / "metadata.json").write_text(json.dumps(meta))
        out[f"phi_{name}"], out[f"theta_{name}"] = phi, theta
    r = pa.compare_tables(pa.load_table(td / "rec_a"), pa.load_table(td / "rec_b"))
    out["metrics"] = np.array([r["tv"], r["l1"], r["theta_marginal_tv"], r["hellinger"], r["jensen_shannon_nats"],
                               r["g_a"], r["g_b"]])
    out["edges"] = edges
    np.savez_compressed(HERE / "compare_reference.npz", **out)


RAINBOW_RADII = ["0.1", "0.2", "0.3", "0.4", "0.5", "0.6", "0.7", "0.8", "0.9", "1.0", "1.01", "0.01", "0.35", "0.15",
                 "0.55", "0.95", "0.0999999", "0.1000001", "0.9999999", "1.0000001", "0.123456", "0.7777", "0.25",
                 "0.45", "nan", "-0.5"]


def rainbow_fixtures(td: Path) -> None:
    """The reference's Table-II lookup on float32 radii and its detect + filter on the grids of
    tests/rainbow_cases.py (every output field, bit for bit; the labels handed to the filter;
    the SHA-256 of each input grid)."""
    sys.path.insert(0, str(ROOT / "tests"))
    import rainbow_cases as RC  # noqa: E402
    r = subprocess.run([str(REF_BIN / "ref_rainbow_harness"), "table"], input="\n".join(RAINBOW_RADII) + "\n",
                       capture_output=True, text=True, check=True)
    rows = [line.split() for line in r.stdout.splitlines()]
    out = {"table_radius": np.array([np.float32(float(x)) for x in RAINBOW_RADII], dtype=np.float32),
           "table_ok": np.array([int(a) for a, _ in rows], dtype=np.uint8),
           "table_sigma": np.array([float.fromhex(b) for _, b in rows])}
    n = len(RAINBOW_RADII)
    assert len(rows) == n
    for name, nt, np_, cfg, make, spec in RC.CASES:
        f = make()
        src, dst = td / "rb.in", td / "rb.out"
        given = RC.labels_for(spec, lambda g: _ref_grid(src, dst, f if g is None else g, nt, np_, cfg, None)[0])
        edges, res = _ref_grid(src, dst, f, nt, np_, cfg, given)
        out[f"{name}.digest"] = np.array(RC.digest(f))
        out[f"{name}.shape"] = np.array([nt, np_], dtype=np.uint32)
        out[f"{name}.config"] = np.array(cfg, dtype=np.float64)
        out[f"{name}.given"] = np.array(0 if given is None else 1, dtype=np.uint8)
        out[f"{name}.edges"] = edges
        # a direction without flags is returned unchanged (input intensities, zero width and
        # blend, no kind): only the flagged ones are stored in full
        changed = np.flatnonzero(res["flags"])
        out[f"{name}.flags"] = res["flags"].copy()
        out[f"{name}.changed"] = changed.astype(np.uint32)
        for k in ("intensity_s", "intensity_p", "sigma_rad", "blend", "transition_kind"):
            out[f"{name}.{k}"] = res[k][changed].copy()
        quiet = res["flags"] == 0
        assert (res["transition_kind"][quiet] == 0).all() and (res["sigma_rad"][quiet] == 0).all()
        assert (res["blend"][quiet] == 0).all()
        assert (res["intensity_s"][quiet] == f["intensity_s"][quiet]).all()
        assert (res["intensity_p"][quiet] == f["intensity_p"][quiet]).all()
    np.savez_compressed(HERE / "rainbow_reference.npz", **out)


def _ref_grid(src: Path, dst: Path, f, nt, np_, cfg, edges):
    import rainbow_cases as RC  # noqa: E402
    with open(src, "wb") as fh:
        fh.write(np.array([nt, np_], dtype="<u4").tobytes() + np.asarray(cfg, dtype="<f8").tobytes())
        fh.write(np.array([0 if edges is None else 1, 0], dtype="<u4").tobytes())
        fh.write(np.ascontiguousarray(f, dtype=RC.FOCAL_DTYPE).tobytes())
        if edges is not None:
            fh.write(np.ascontiguousarray(edges, dtype="<u4").tobytes())
    run([REF_BIN / "ref_rainbow_harness", "grid", src, dst])
    raw = dst.read_bytes()
    n = nt * np_
    return np.frombuffer(raw[:4 * n], "<u4").copy(), np.frombuffer(raw[4 * n:], RC.RESULT_DTYPE).copy()


def optics_fixtures(td: Path) -> None:
    """The reference's per-direction optics (PatchOpticalEvaluator::evaluate_direction, with and
    without the focal stage) and patch construction (PatchConstruction::make, patch_id order) on
    the inputs of tests/optics_cases.py, with each input's SHA-256."""
    sys.path.insert(0, str(ROOT / "tests"))
    import optics_cases as OC  # noqa: E402
    out = {}
    for name, make in OC.CASES:
        c = make()
        blob = OC.serialize(c)
        src, dst = td / "op.in", td / "op.out"
        src.write_bytes(blob)
        run([REF_BIN / "ref_optics_harness", src, dst])
        raw = dst.read_bytes()
        n = c.count
        out[f"{name}.digest"] = np.array(OC.digest(c))
        out[f"{name}.optical"] = np.frombuffer(raw[:136 * n], dtype=OC.OPTICAL_DTYPE).copy()
        if c.focal:
            sys.path.insert(0, str(ROOT / "tests"))
            import rainbow_cases as RC  # noqa: E402
            out[f"{name}.focal"] = np.frombuffer(raw[136 * n:], dtype=RC.FOCAL_DTYPE).copy()
    for name, make in OC.PATCH_CASES:
        v, (w, h, e) = make()
        src, dst = td / "pa.in", td / "pa.out"
        src.write_bytes(OC.serialize_lattice(v, (w, h, e)))
        run([REF_BIN / "ref_patch_harness", src, dst])
        raw = dst.read_bytes()
        cells = 4 * (w - 1) * (h - 1)
        n = int(np.frombuffer(raw[4 * cells:4 * cells + 4], "<u4")[0])
        off = 4 * cells + 36
        out[f"patch.{name}.digest"] = np.array(hashlib_hex(OC.serialize_lattice(v, (w, h, e))))
        out[f"patch.{name}.status"] = np.frombuffer(raw[:4 * cells], "<u4").astype(np.uint8)
        out[f"patch.{name}.histogram"] = np.frombuffer(raw[4 * cells + 4:off], "<u4").copy()
        out[f"patch.{name}.patches"] = np.frombuffer(raw[off:off + 32 * n], OC.PATCH_DTYPE).copy()
        out[f"patch.{name}.aabbs"] = np.frombuffer(raw[off + 32 * n:off + 56 * n], OC.AABB_DTYPE).copy()
    # ray / bilinear patch intersections and the query direction grid
    corners, dirs = OC.intersection_pairs()
    src, dst = td / "is.in", td / "is.out"
    src.write_bytes(np.array([len(corners)], "<u4").tobytes() +
                    np.hstack([corners.reshape(-1, 12), dirs]).astype("<f4").tobytes())
    run([REF_BIN / "ref_query_harness", "intersect", src, dst])
    out["intersect.digest"] = np.array(hashlib_hex(corners.tobytes() + dirs.tobytes()))
    out["intersect.hits"] = np.frombuffer(dst.read_bytes(), dtype=OC.BILINEAR_HITS_DTYPE).copy()
    for nt, np_, axis, e0 in OC.DIRECTION_GRIDS:
        run([REF_BIN / "ref_query_harness", "directions", nt, np_, *map(repr, axis), *map(repr, e0), dst])
        out[f"directions.{nt}x{np_}"] = np.frombuffer(dst.read_bytes(), "<f4").reshape(-1, 3).copy()
    np.savez_compressed(HERE / "optics_reference.npz", **out)
    # the reference's own unpolarized lattice trace of a 0.5 mm sphere (25 x 25 vertices, four
    # families), the real input of the device chain from patch build to the stage densities
    lat = td / "lattice.bin"
    run([REF_BIN / "ref_drop_harness", "vertices", "0.5", "1", "1.3317", "0.9396926", "-0.3420201", "0", "25", lat])
    raw = lat.read_bytes()
    w, h = np.frombuffer(raw[:8], "<u4")
    n = 4 * int(w) * int(h)
    np.savez_compressed(HERE / "drop_lattice_reference.npz", shape=np.array([w, h], dtype=np.uint32),
                        frame=np.frombuffer(raw[8:36], "<f4").copy(),
                        vertices=np.frombuffer(raw[36:36 + 68 * n], OC.VERTEX_DTYPE).copy(),
                        second=np.frombuffer(raw[36 + 68 * n:], "<f4").reshape(-1, 4).copy())


def hashlib_hex(blob: bytes) -> str:
    import hashlib
    return hashlib.sha256(blob).hexdigest()


def main() -> None:
    subprocess.run([str(ROOT / "oracle" / "build_ref.sh"), str(REF)], check=True)
    with tempfile.TemporaryDirectory() as t:
        td = Path(t)
        # 1. the reference CLI test record (phase_cli_test.py:242-246) + its masses
        csv = td / "two.csv"
        csv.write_text(TWO_ORIENTATIONS)
        out = td / "rec"
        run([REF_BIN / "ice_generate_phase_cpu", "--orientations", csv, "--radius-mm", "0.1", "--length-mm", "0.2",
             "--ki", "1", "-0.4", "0.3", "--ior", "1.31", "--wavelength-nm", "550", "--theta", "72", "--phi", "144",
             "--cdf-theta", "36", "--cdf-phi", "72", "--out", out, "--batch-size", "512"])
        meta = json.loads((out / "metadata.json").read_text())
        m, d, u = masses(td, 0.1, 0.2, (1.0, -0.4, 0.3), 1.31, 72, 144, TWO_ORIENTATIONS, batch=512)
        np.savez_compressed(
            HERE / "hex_two_orientations.npz", masses=m, stats=d, counts=u,
            phi=np.load(out / "phi_cdf.npy"), theta=np.load(out / "theta_given_phi_cdf.npy"),
            u=np.load(out / "u_edges.npy"),
            meta=np.array([meta["hg"]["g"], meta["quality"]["cdf_l1_mass_error"],
                           meta["storage_processing"]["coarsening_tv"], meta["transport_audit"]["escaped_mm2"],
                           meta["transport_audit"]["unresolved_mm2"], meta["geometry"]["projected_area_mm2"],
                           meta["histogram"]["mass_mm2"], meta["histogram"]["g_rays"]]),
            sampling_frame_columns=np.array(meta["sampling_frame_columns"]))
        # 2. the hex column (circumradius 0.05 mm, length 0.2 mm) at 512x1024, 20k rays, 12 hits (sparse: the masses are a few hundred deltas)
        ki = (0.8660254037844387, -0.5, 0.0)
        m, d, u = masses(td, 0.05, 0.2, ki, 1.31, 512, 1024, COLUMN_PLAN, max_hits=12)
        nz = np.flatnonzero(m)
        np.savez_compressed(HERE / "hex_column_20k.npz", index=nz, value=m[nz], stats=d, counts=u)
        # 3. per-ray reference audits and exits for 48 rays of the hex column node
        out = td / "t.bin"
        run([REF_BIN / "ref_hex_harness", "trace", "0.05", "0.2", *map(repr, ki), "1.31", "1", 12345, 20000, 1024,
             repr(1e-12), 100, 48, out])
        raw = np.frombuffer(out.read_bytes(), "<f8")
        info = raw[:48 * 6].reshape(48, 6)
        exits = raw[48 * 6:].reshape(-1, 4)
        np.savez_compressed(HERE / "hex_rays.npz", info=info, exits=exits)
        # 4. drops: host inputs and the four-family path tracer
        drop_fixtures(td)
        # 5. ice Ih index of the prism records
        ice_fixtures()
        # 6. deterministic atlas: area rule, traced nodes, orientation composition
        atlas_fixtures(td)
        # 7. the reference's record-vs-record metric
        compare_fixtures(td)
        # 8. Table-II rainbow diffraction
        rainbow_fixtures(td)
        # 9. per-direction optics of the drop's wave stages
        optics_fixtures(td)
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
