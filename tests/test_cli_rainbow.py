"""The rainbow_generate drop-in CLI: the reference's option contract (apps/generate_phase.cpp:
84-223, messages and exit code 1) on the CPU, and the record contract (metadata schema,
PhaseRecord validation, .part staging, overwrite refusal) on the GPU, with the FP64 record
checked against the oracle's."""
from __future__ import annotations

import hashlib
import json
import math
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from record_check import validate_record

EXE = ROOT / "ice_crystal_phase_b200" / "bin" / "rainbow_generate"


def run(args, code=0):
    r = subprocess.run([str(EXE), *map(str, args)], capture_output=True, text=True)
    assert r.returncode == code, (r.returncode, r.stdout, r.stderr)
    return r


@pytest.mark.parametrize("args,message", [
    ([], "--out is required."),
    (["--out", "X"], "--wavelength-nm is required; there is no implicit wavelength."),
    (["--out", "X", "--wavelength-nm", "700", "--wavelength-nm", "600"], "Duplicate --wavelength-nm."),
    (["--out", "X", "--wavelength-nm", "700", "--ior", "1.33"], "Do not specify --ior for water."),
    (["--out", "X", "--wavelength-nm", "700", "--material", "constant"], "Constant material requires a finite positive --ior."),
    (["--out", "X", "--wavelength-nm", "700", "--material", "constant", "--ior", "1.33", "--temperature-c", "5"],
     "Temperature/pressure do not define a constant-index material."),
    (["--out", "X", "--wavelength-nm", "700", "--material", "ice"], "Material must be water or constant."),
    (["--out", "X", "--wavelength-nm", "700", "--radius-mm", "3.5", "--stage", "path"], "radius_mm must be in (0,3]"),
    (["--out", "X", "--wavelength-nm", "700", "--radius-mm", "1.5"], "Table II covers radius 0.1..1.0 mm only."),
    (["--out", "X", "--wavelength-nm", "700", "--radius-mm", "0.05", "--stage", "focal"],
     "Table II covers radius 0.1..1.0 mm only."),
    (["--out", "X", "--wavelength-nm", "150"], "IAPWS R9-97: wavelength/state outside supported range."),
    (["--out", "X", "--wavelength-nm", "700", "--temperature-c", "70"], "Water material supports liquid branch"),
    (["--out", "X", "--wavelength-nm", "300"], "wavelength_nm must be in [380,830]"),
    (["--out", "X", "--wavelength-nm", "1000"], "wavelength_nm must be in [380,830]"),
    (["--out", "X", "--wavelength-nm", "700", "--material", "constant", "--ior", "2.5"], "interior_index must be in [1,2]"),
    (["--out", "X", "--wavelength-nm", "700", "--query-theta", "90", "--cdf-theta", "60"],
     "CDF dimensions must divide the query dimensions without upsampling."),
    (["--out", "X", "--wavelength-nm", "700", "--max-coarsening-tv", "2"], "Coarsening TV limit must lie in [0,1]."),
    (["--out", "X", "--wavelength-nm", "700", "--grid", "1"], "Invalid grid dimensions"),
    (["--out", "X", "--wavelength-nm", "700", "--grid", "0"], "Invalid positive integer option."),
    (["--out", "X", "--wavelength-nm", "abc"], "Invalid numeric option."),
    (["--out", "X", "--wavelength-nm", "700", "--storage-gaussian-sigma-deg", "1"], "Global storage blur has been removed"),
    (["--out", "X", "--wavelength-nm", "700", "--diffraction-sigma-deg", "1"], "Manual diffraction width is not supported"),
    (["--out", "X", "--wavelength-nm", "700", "--focal-offsets", "0,1,2"], "Expected four focal offsets."),
    (["--out", "X", "--wavelength-nm", "700", "--focal-offsets", "0,1,2,4"], "Focal offsets must be 0..3."),
    (["--out", "X", "--wavelength-nm", "700", "--rays", "1000"], "apply to the ray model (--stage incoherent --optics rays)"),
    (["--out", "X", "--wavelength-nm", "700", "--stage", "path", "--optics", "rays"],
     "--optics rays applies to --stage incoherent only"),
    (["--out", "X", "--wavelength-nm", "700", "--stage", "incoherent", "--optics", "lattice", "--seed", "3"],
     "apply to the ray model"),
    (["--out", "X", "--wavelength-nm", "700", "--optics", "mesh"], "--optics must be lattice or rays."),
    (["--out", "X", "--wavelength-nm", "700", "--stage", "bogus"], "Unknown stage."),
    (["--out", "X", "--wavelength-nm", "700", "--device", "-1"], "Invalid device ordinal."),
    (["--out", "X", "--wavelength-nm", "700", "--bogus", "1"], "Unknown option: --bogus"),
    (["--out", "X", "--wavelength-nm", "700", "--shape-coefficients", "0,0,0.5"], "nonconvex"),
    (["--out", "X", "--wavelength-nm", "700", "--sphere", "--shape-coefficients", "0,-0.01"],
     "--sphere and --shape-coefficients are exclusive."),
    (["--out"], "Missing option value."),
])
def test_option_errors_exit_1(tmp_path, args, message):
    args = [str(tmp_path / a) if a == "X" else a for a in args]
    r = run(args, code=1)
    assert r.stderr.startswith("rainbow_generate: ") and message in r.stderr, r.stderr
    assert not any(tmp_path.iterdir())


def test_help_and_existing_outputs(tmp_path):
    assert "rainbow_generate --out DIRECTORY" in run(["--help"]).stdout
    (tmp_path / "done").mkdir()
    assert "Output already exists." in run(["--out", tmp_path / "done", "--wavelength-nm", "700"], 1).stderr
    (tmp_path / "half.part").mkdir()
    assert "Previous .part directory exists" in run(["--out", tmp_path / "half", "--wavelength-nm", "700"], 1).stderr


@pytest.mark.gpu
def test_record_contract(tmp_path, icp):
    out = tmp_path / "drop"
    r = run(["--out", out, "--wavelength-nm", "700", "--radius-mm", "1.5", "--query-theta", "180", "--query-phi",
             "360", "--cdf-theta", "90", "--cdf-phi", "180", "--stage", "incoherent", "--rays", "2000000"])
    assert "Saved NumPy CDF dataset" in r.stdout
    assert {p.name for p in out.iterdir()} == {"metadata.json", "phi_cdf.npy", "theta_given_phi_cdf.npy", "u_edges.npy"}
    rec = validate_record(out)
    m, mass, u = rec["metadata"], rec["cell_probability"], rec["u"]
    assert rec["phi"].shape == (181,) and rec["theta"].shape == (180, 91)
    assert abs(mass.sum() - 1) < 1e-12
    assert abs(np.sum(mass * (1 - u[:-1] - u[1:])[None, :]) - m["hg"]["g"]) < 1e-12
    shape = icp.RaindropShape.make(1.5)
    assert m["shape_coefficients"] == shape.coefficients and m["shape_source"] == "Sadeghi2012_TableI"
    k, e0, e1 = icp.drop_frame(20.0)
    assert m["sampling_frame_columns"] == [[e0[i], e1[i], k[i]] for i in range(3)]
    assert m["geometry"]["projected_area_mm2"] == icp.compute_projected_area(shape.coefficients, 1.5, k)
    water = icp.evaluate_water_optics(700.0)
    assert m["material"]["interior_index_evaluated_fp64"] == water.refractive_index
    assert m["interior_index"] == float(np.float32(water.refractive_index))
    t = m["transport_audit"]
    assert abs((t["escaped_mm2"] + t["unresolved_mm2"]) / t["incident_mm2"] - 1) < 1e-12
    assert m["stage"] == "incoherent" and m["diffraction_policy"]["computed"] is False
    assert m["sampling"]["rays"] == 2000000 and m["sampling"]["missed_rays"] > 0
    # the sampled hit area estimates the CPU projected area
    area, disk = m["geometry"]["projected_area_mm2"], m["geometry"]["sampled_disk_area_mm2"]
    p = area / disk
    assert abs(t["incident_mm2"] - area) <= 5 * disk * math.sqrt(p * (1 - p) / 2e6)
    # the primary bow: the mass peaks near 138 degrees of scattering (u ~ 0.87)
    rows = mass.sum(axis=0)
    theta_deg = np.degrees(np.arccos(1 - (u[:-1] + u[1:])))
    back = (theta_deg > 120) & (theta_deg < 160)
    assert 134 < theta_deg[back][np.argmax(rows[back])] < 142
    # a published record is not overwritten
    digest = {f.name: hashlib.sha256(f.read_bytes()).hexdigest() for f in out.iterdir()}
    assert "Output already exists." in run(["--out", out, "--wavelength-nm", "700", "--stage", "incoherent"], 1).stderr
    assert digest == {f.name: hashlib.sha256(f.read_bytes()).hexdigest() for f in out.iterdir()}


@pytest.mark.gpu
def test_fp64_record_matches_oracle(tmp_path, icp, oracle):
    """Four reference families only (3 internal hits): the FP64 record equals the oracle's CDF."""
    out = tmp_path / "fp64"
    run(["--out", out, "--wavelength-nm", "650", "--radius-mm", "1.0", "--inclination-deg", "35", "--query-theta", "72",
         "--query-phi", "144", "--cdf-theta", "36", "--cdf-phi", "72", "--stage", "incoherent", "--rays", "30000",
         "--seed", "5",
         "--trace-precision", "fp64", "--max-internal-hits", "3", "--max-unresolved-fraction", "0.5"])
    rec = validate_record(out)
    m = rec["metadata"]
    geo = oracle.drop_geometry(m["shape_coefficients"], m["radius_mm"])
    orc = oracle.drop_record(geo, np.array(icp.drop_frame(35.0)), m["interior_index"], 72, 144, 30000, 5, max_hits=3)
    cdf = oracle.build_cdf(orc.masses, 72, 144, 36, 72)
    ref = np.diff(cdf.phi)[:, None] * np.diff(cdf.theta, axis=1)
    assert np.abs(rec["cell_probability"] - ref).sum() <= 2e-10
    assert abs(m["hg"]["g"] - cdf.report["g_stored"]) <= 2e-11
    assert abs(m["transport_audit"]["unresolved_mm2"] / orc.unresolved_area - 1) <= 1e-10


@pytest.mark.gpu
def test_extensions(tmp_path):
    out = tmp_path / "baseline_shape"
    run(["--out", out, "--wavelength-nm", "550", "--radius-mm", "0.5", "--shape-coefficients", "0,-0.08,-0.02,0.005",
         "--stage", "incoherent", "--diffraction", "analytic", "--query-theta", "90", "--query-phi", "180", "--rays",
         "200000"])
    m = validate_record(out)["metadata"]
    assert m["shape_coefficients"] == [0, -0.08, -0.02, 0.005, 0, 0, 0, 0]
    assert m["shape_source"] == "command_line"
    d = m["diffraction_policy"]
    assert d["computed"] is True and abs(d["power_mm2"] / m["transport_audit"]["incident_mm2"] - 1) < 1e-12
    sphere = tmp_path / "sphere"
    run(["--out", sphere, "--wavelength-nm", "550", "--radius-mm", "2.0", "--sphere", "--query-theta", "90",
         "--query-phi", "180", "--stage", "incoherent", "--rays", "100000", "--material", "constant", "--ior", "1.333"])
    m = validate_record(sphere)["metadata"]
    assert m["sampling"]["missed_rays"] == 0 and m["geometry"]["projected_area_method"] == "analytic_sphere"
    assert m["material"]["model"] == "constant"


# ------------------------------------------------------------ the lattice (patch) model stages
def _stage(tmp_path, stage, extra=()):
    out = tmp_path / stage
    # the 0.5 mm drop's Table-II width (0.22 deg) needs cells below 0.11 deg to be resolved; at
    # this grid the diffraction stage is accepted only with --allow-underresolved, as in the
    # reference (its defaults, 360 x 720 and 1.0 mm, are underresolved as well)
    allow = ["--allow-underresolved"] if stage == "diffraction" else []
    r = run(["--out", out, "--wavelength-nm", "650", "--radius-mm", "0.5", "--grid", "129", "--query-theta", "180",
             "--query-phi", "360", "--cdf-theta", "90", "--cdf-phi", "180", "--stage", stage, *allow, *extra])
    assert "Saved NumPy CDF dataset" in r.stdout
    return validate_record(out)


@pytest.mark.gpu
@pytest.mark.parametrize("stage", ["diffraction", "focal", "path"])
def test_lattice_stage_records(tmp_path, icp, stage):
    """rainbow_generate --stage path | focal | diffraction: the reference's patch model on the
    device -- lattice trace, patches, query, folded records, optics, Table II, stored CDF --
    written in the record contract the reference's reader accepts."""
    rec = _stage(tmp_path, stage)
    m, mass, u = rec["metadata"], rec["cell_probability"], rec["u"]
    assert m["stage"] == stage and m["incident_grid"] == [129, 129]
    assert abs(mass.sum() - 1) < 1e-12
    assert m["diffraction_policy"]["computed"] is (stage != "path")
    assert m["diffraction_policy"]["selected_output_includes_diffraction"] is (stage == "diffraction")
    assert m["quality"]["incomplete_directions"] == 0 and m["quality"]["invalid_values"] == 0
    assert m["patches"]["pending_directions"] == 0 and m["patches"]["error_directions"] == 0
    assert m["patches"]["folded_candidates"] == m["patches"]["folded_prepared"] > 0
    assert m["patches"]["folded_evaluated_hits"] > 0
    assert m["material"]["density_model"] == "IAPWS R6-95(2018) liquid pressure EOS inversion"
    cfg = icp.raindrop_config(0.5, 650.0, m["interior_index"], (np.cos(np.radians(20.0)), -np.sin(np.radians(20.0)), 0.0),
                              129)
    assert m["incident_grid_half_extent"] == float(np.float32(cfg.grid_half_extent))
    # the primary bow near 138 degrees
    rows = mass.sum(axis=0)
    theta_deg = np.degrees(np.arccos(1 - (u[:-1] + u[1:])))
    back = (theta_deg > 120) & (theta_deg < 160)
    assert 134 < theta_deg[back][np.argmax(rows[back])] < 144


@pytest.mark.gpu
def test_lattice_incoherent_matches_ray_model(tmp_path):
    """--stage incoherent with the reference's patch model and with the ray model describe the same
    geometric optics: over the families both carry (R .. TRRT dominate the mass), their stored
    phase functions agree in g to 1e-2 and in total variation to 0.15."""
    lat = _stage(tmp_path, "incoherent", ["--optics", "lattice"])
    out = tmp_path / "rays"
    run(["--out", out, "--wavelength-nm", "650", "--radius-mm", "0.5", "--query-theta", "180", "--query-phi", "360",
         "--cdf-theta", "90", "--cdf-phi", "180", "--stage", "incoherent", "--rays", "4000000",
         "--max-internal-hits", "3", "--max-unresolved-fraction", "0.2"])
    ray = validate_record(out)
    assert abs(lat["metadata"]["hg"]["g"] - ray["metadata"]["hg"]["g"]) < 1e-2
    assert 0.5 * np.abs(lat["cell_probability"] - ray["cell_probability"]).sum() < 0.15


@pytest.mark.gpu
def test_lattice_diffraction_underresolved_gate(tmp_path):
    """A query grid too coarse for the Table-II width leaves directions underresolved: the
    reference's CDF input gate rejects the record unless --allow-underresolved is given."""
    args = ["--wavelength-nm", "650", "--radius-mm", "0.5", "--grid", "129", "--query-theta", "180", "--query-phi",
            "360", "--cdf-theta", "90", "--cdf-phi", "180"]
    r = run(["--out", tmp_path / "rejected", *args], code=1)
    assert "CDF input rejected" in r.stderr and "underresolved=" in r.stderr
    assert not (tmp_path / "rejected").exists() and not (tmp_path / "rejected.part").exists()
    run(["--out", tmp_path / "allowed", *args, "--allow-underresolved"])
    m = validate_record(tmp_path / "allowed")["metadata"]
    assert m["quality"]["underresolved_directions"] > 0 and m["quality"]["allow_underresolved"] is True
