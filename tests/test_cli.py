"""The ice_generate_phase drop-in CLI, exercised like the reference's own CLI test
(hex_phase/tests/phase_cli_test.py:34-110) and compared with the reference's record."""
from __future__ import annotations

import hashlib
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, TWO_ORIENTATIONS
from record_check import validate_record

EXE = ROOT / "ice_crystal_phase_b200" / "bin" / "ice_generate_phase"
COMMON = ["--radius-mm", "0.1", "--length-mm", "0.2", "--ki", "1", "-0.4", "0.3", "--ior", "1.31",
          "--wavelength-nm", "550", "--theta", "72", "--phi", "144", "--cdf-theta", "36", "--cdf-phi", "72"]


def run(args, code=0):
    r = subprocess.run([str(EXE), *map(str, args)], capture_output=True, text=True)
    assert r.returncode == code, (r.returncode, r.stdout, r.stderr)
    return r


@pytest.fixture()
def plan(tmp_path):
    p = tmp_path / "orientations.csv"
    p.write_text(TWO_ORIENTATIONS)
    return p


def test_parse_errors_exit_1(tmp_path, plan):
    assert "ice_generate_phase --out DIR" in run(["--help"]).stdout
    r = run(["--orientations", plan, *COMMON], code=1)
    assert "Required option: --out" in r.stderr
    run(["--out", tmp_path / "a", "--out", tmp_path / "b"], code=1)
    run(["--orientations", plan, *COMMON, "--out", tmp_path / "c", "--bogus", "1"], code=1)
    run(["--orientations", plan, *COMMON, "--out", tmp_path / "d", "--cdf-theta", "25"], code=1)
    run(["--orientations", plan, *COMMON, "--out", tmp_path / "e", "--trace-precision", "fp16"], code=1)
    assert not any(tmp_path.glob("*.part"))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_reference_cli_contract(tmp_path, plan, precision):
    out = tmp_path / "reference"
    run(["--orientations", plan, *COMMON, "--out", out, "--batch-size", "512", "--trace-precision", precision])
    assert {p.name for p in out.iterdir()} == {"metadata.json", "phi_cdf.npy", "theta_given_phi_cdf.npy", "u_edges.npy"}
    rec = validate_record(out)
    m, mass, u = rec["metadata"], rec["cell_probability"], rec["u"]
    assert rec["phi"].shape == (73,) and rec["theta"].shape == (72, 37) and u.shape == (37,)
    assert m["orientation"]["csv_sha256"] == hashlib.sha256(plan.read_bytes()).hexdigest()
    assert m["histogram"]["relative_mass_audit_error"] < 1e-10
    assert m["sampling"]["planned_rays"] == 3072
    assert abs(mass.sum() - 1) < 1e-12
    expected_g = np.sum(mass * (1 - u[:-1] - u[1:])[None, :])
    assert abs(expected_g - m["hg"]["g"]) < 1e-12
    area, esc, unres = (m["geometry"]["projected_area_mm2"], m["transport_audit"]["escaped_mm2"],
                        m["transport_audit"]["unresolved_mm2"])
    assert abs((esc + unres) / area - 1) < 1e-12
    assert m["diffraction_policy"]["computed"] is False and m["storage_processing"]["gaussian_sigma_degrees"] == 0
    # against the reference's own record for the same inputs and seeds
    g = np.load(GOLDEN / "hex_two_orientations.npz")
    ref = np.diff(g["phi"])[:, None] * np.diff(g["theta"], axis=1)
    assert np.array_equal(u, g["u"])
    if precision == "fp64":
        assert np.abs(mass - ref).sum() <= 2e-10
        assert abs(m["hg"]["g"] - g["meta"][0]) <= 2e-11
        assert area == g["meta"][5]
    else:
        assert 0.5 * np.abs(mass - ref).sum() <= 1e-3
        assert abs(m["hg"]["g"] - g["meta"][0]) <= 1e-4
    # chunking must not alter the sample ids
    other = tmp_path / "other"
    run(["--orientations", plan, *COMMON, "--out", other, "--batch-size", "31", "--trace-precision", precision])
    assert np.abs(validate_record(other)["cell_probability"] - mass).sum() < 1e-10
    # a published record is not overwritten
    digest = {f.name: hashlib.sha256(f.read_bytes()).hexdigest() for f in out.iterdir()}
    run(["--orientations", plan, *COMMON, "--out", out], code=1)
    assert digest == {f.name: hashlib.sha256(f.read_bytes()).hexdigest() for f in out.iterdir()}


@pytest.mark.gpu
@pytest.mark.parametrize("name,options", [("limited", ["--max-internal-hits", "1"]),
                                          ("large_tail", ["--tail-tolerance", "0.001"]),
                                          ("coarsening", ["--max-coarsening-tv", "0"]),
                                          ("capacity", ["--max-output-records", "1"])])
def test_failures_exit_2_and_keep_part(tmp_path, plan, name, options):
    failed = tmp_path / name
    run(["--orientations", plan, *COMMON, "--out", failed, *options], code=2)
    assert not failed.exists()
    part = tmp_path / (name + ".part")
    assert json.loads((part / "failure.json").read_text())["complete"] is False
    assert not (part / "metadata.json").exists()
    with pytest.raises((ValueError, OSError)):
        validate_record(part)


@pytest.mark.gpu
def test_transparent_limit(tmp_path, plan):
    args = list(COMMON)
    args[args.index("--ior") + 1] = "1"
    out = tmp_path / "transparent"
    run(["--orientations", plan, *args, "--out", out, "--tail-tolerance", "0"])
    rec = validate_record(out)
    pm = rec["cell_probability"]
    assert np.abs(pm[:, 0] - 1 / 72).max() < 1e-13
    assert np.abs(pm[:, 1:]).max() == 0
    assert abs(rec["metadata"]["hg"]["g"] - (1 - rec["u"][1])) < 1e-12


@pytest.mark.gpu
def test_npy_bytes_match_reference_writer(tmp_path, plan):
    # the NPY header layout of the reference writer (src/npy_writer.cpp:31-47)
    out = tmp_path / "rec"
    run(["--orientations", plan, *COMMON, "--out", out, "--trace-precision", "fp64"])
    raw = (out / "u_edges.npy").read_bytes()
    assert raw[:8] == b"\x93NUMPY\x01\x00"
    hlen = raw[8] | raw[9] << 8
    assert (10 + hlen) % 64 == 0 and raw[10:10 + hlen].startswith(b"{'descr': '<f8', 'fortran_order': False, 'shape': (37, ), }")
