"""The batched condition-grid dataset tool (ice_crystal_phase_b200.dataset), held to the reference
orchestrator's contract (tools/generate_phase_dataset.py): config validation messages, dry run,
the lock, the signed plan, .part -> rename per record, receipts verified on --resume, refusal
to adopt foreign directories or tampered records.  The CPU tests drive the orchestration with a
fake generator; the GPU test runs the batched library."""
from __future__ import annotations

import copy
import json
import math
import types

import numpy as np
import pytest

from record_check import validate_record

CONFIG = {
    "output_root": "out", "generator": "build/rainbow_generate", "radius_mm": 1.0, "force_sphere": False,
    "temperature_c": 20, "pressure_pa": 101325,
    "wavelengths": {"start_nm": 500, "stop_nm": 600, "step_nm": 100},
    "inclinations": {"min_degrees": -30, "max_degrees": 30, "count": 2, "placement": "linear_angle_cell_centers"},
    "solver": {"grid": 129, "query_theta": 72, "query_phi": 144, "cdf_theta": 36, "cdf_phi": 72,
               "stage": "incoherent", "device": 0, "focal_offsets": [0, 0, 0, 0], "allow_underresolved": False,
               "maximum_coarsening_tv": 1, "cdf_max_l1": 1e-10, "cdf_max_lost_mass": 1e-12},
    "reserve_gib": 0,
    "b200": {"rays": 200000, "batch_records": 3, "precision": "fp64"},
}


def _write(tmp_path, cfg):
    p = tmp_path / "config.json"
    p.write_text(json.dumps(cfg))
    return p


@pytest.fixture()
def ds():
    from ice_crystal_phase_b200 import dataset

    return dataset


@pytest.mark.parametrize("mutate,message", [
    (lambda c: c.pop("reserve_gib"), "Unexpected/missing config keys"),
    (lambda c: c["wavelengths"].update(step_nm=33), "integer number of steps"),
    (lambda c: c["wavelengths"].update(start_nm=300), "Require 380 <= start"),
    (lambda c: c["inclinations"].update(min_degrees=0, max_degrees=180), "Canonical inclination domain"),
    (lambda c: c["inclinations"].update(placement="edges"), "linear_angle_cell_centers"),
    (lambda c: c["solver"].update(cdf_theta=50), "CDF grids must divide query grids"),
    (lambda c: c["solver"].update(stage="bogus"), "Unknown stage"),
    (lambda c: c.update(radius_mm=4), "outside"),
    (lambda c: c["solver"].update(allow_underresolved=1), "Expected JSON true or false"),
    (lambda c: c["b200"].update(precision="fp16"), "b200.precision"),
    (lambda c: c["b200"].update(unknown=1), "b200 accepts only"),
])
def test_config_rejections(ds, mutate, message):
    cfg = copy.deepcopy(CONFIG)
    mutate(cfg)
    with pytest.raises(ValueError, match=message):
        ds.normalized_config(cfg)


def test_config_grid_and_defaults(ds):
    c = ds.normalized_config(copy.deepcopy(CONFIG))
    assert c["wavelength_nm"] == ["500", "600"]
    assert c["inclination_degrees"] == ["-15.0", "15.0"]
    cfg = copy.deepcopy(CONFIG)
    cfg.pop("b200")
    d = ds.normalized_config(cfg)["b200"]
    assert d["rays"] == 10_000_000 and d["precision"] == "fp32" and d["max_internal_hits"] == 1024
    seeds = {ds.condition_seed(12345, i, l) for i in range(50) for l in range(50)}
    assert len(seeds) == 2500


def test_dry_run_writes_nothing(ds, tmp_path, capsys):
    cfg = copy.deepcopy(CONFIG)
    cfg["output_root"] = str(tmp_path / "out")
    assert ds.run(["--config", str(_write(tmp_path, cfg))]) == 0
    assert "DRY RUN" in capsys.readouterr().out
    assert not (tmp_path / "out").exists()


def test_npy_writer_format(ds, tmp_path):
    a = np.arange(3 * 5, dtype=float).reshape(3, 5) / 7
    ds.write_npy(tmp_path / "a.npy", a)
    raw = (tmp_path / "a.npy").read_bytes()
    assert raw.startswith(b"\x93NUMPY\x01\x00")
    header_len = int.from_bytes(raw[8:10], "little")
    assert (10 + header_len) % 64 == 0
    assert b"'shape': (3, 5, ), }" in raw[:10 + header_len]
    assert np.array_equal(np.load(tmp_path / "a.npy"), a)
    assert ds.npy_size(tmp_path / "a.npy", (3, 5)) == len(raw)
    with pytest.raises(ValueError):
        ds.npy_size(tmp_path / "a.npy", (5, 3))


class FakeBackend:
    """Uniform records with plausible reports, for the orchestration logic on the CPU."""

    def __init__(self, icp):
        self.icp, self.calls = icp, []

    def library_sha256(self):
        return "0" * 64

    class _Ctx:
        def __enter__(self):
            return self

        def __exit__(self, *a):
            return False

    def context(self, device):
        return self._Ctx()

    def generate(self, ctx, c, todo):
        icp = self.icp
        self.calls.append(list(todo))
        s = c["solver"]
        nt, np_ = s["cdf_theta"], s["cdf_phi"]
        out = []
        for ii, ll in todo:
            lam = float(np.float32(float(c["wavelength_nm"][ll])))
            water = icp.evaluate_water_optics(lam, c["temperature_c"], c["pressure_pa"])
            spec = icp.DropSpec(icp.RaindropShape.make(1.0).coefficients, float(np.float32(c["radius_mm"])),
                                float(np.float32(water.refractive_index)), c["b200"]["rays"], seed=ii * 10 + ll,
                                inclination_deg=float(c["inclination_degrees"][ii]), wavelength_nm=lam)
            rep = icp.DropReport()
            k, e0, e1 = icp.drop_frame(spec.inclination_deg)
            for r in range(3):
                rep.ki[r], rep.e0[r], rep.e1[r] = k[r], e0[r], e1[r]
            rep.projected_area_mm2 = rep.sampled_area_mm2 = math.pi
            rep.incident_area_mm2 = rep.escaped_area_mm2 = rep.histogram_mass_mm2 = math.pi
            rep.cdf.g_stored = 0.0
            phi = np.linspace(0, 1, np_ + 1)
            theta = np.tile(icp.u_edges(nt), (np_, 1))
            out.append((spec, water, phi, theta, icp.u_edges(nt), rep))
        return out


def test_orchestration_lock_plan_receipts_resume(ds, icp, tmp_path):
    cfg = copy.deepcopy(CONFIG)
    root = tmp_path / "out"
    cfg["output_root"] = str(root)
    path = _write(tmp_path, cfg)
    fake = FakeBackend(icp)
    assert ds.run(["--config", str(path), "--execute", "--limit", "3"], backend=fake) == 0
    assert fake.calls == [[(0, 0), (0, 1), (1, 0)]]
    assert json.loads((root / "progress.json").read_text())["completed"] == 3
    rec = validate_record(root / "records/i0000/w0001")
    assert rec["metadata"]["generator_version"] == ds.GENERATOR_VERSION
    # a second writer without --resume is refused; a resume completes the plan
    with pytest.raises(FileExistsError):
        ds.run(["--config", str(path), "--execute"], backend=fake)
    assert ds.run(["--config", str(path), "--execute", "--resume"], backend=fake) == 0
    assert fake.calls[-1] == [(1, 1)]
    progress = json.loads((root / "progress.json").read_text())
    assert progress["complete"] is True and progress["completed"] == 4
    assert sorted(p.name for p in (root / "receipts").iterdir()) == [
        "i0000_w0000.json", "i0000_w0001.json", "i0001_w0000.json", "i0001_w0001.json"]
    # a tampered record fails its receipt on resume
    meta = root / "records/i0001/w0000/metadata.json"
    m = json.loads(meta.read_text())
    m["hg"]["g"] = 0.5
    meta.write_text(json.dumps(m))
    with pytest.raises(ValueError, match="Resume receipt/content mismatch"):
        ds.run(["--config", str(path), "--execute", "--resume"], backend=fake)
    # a changed configuration cannot resume the plan
    cfg2 = copy.deepcopy(cfg)
    cfg2["b200"]["rays"] = 300000
    with pytest.raises(ValueError, match="configuration/binaries differ"):
        ds.run(["--config", str(_write(tmp_path, cfg2)), "--execute", "--resume"], backend=fake)


def test_orchestration_refusals(ds, icp, tmp_path):
    cfg = copy.deepcopy(CONFIG)
    root = tmp_path / "out"
    cfg["output_root"] = str(root)
    path = _write(tmp_path, cfg)
    root.mkdir()
    (root / "foreign.txt").write_text("x")
    with pytest.raises(ValueError, match="nonempty directory"):
        ds.run(["--config", str(path), "--execute"], backend=FakeBackend(icp))
    (root / "foreign.txt").unlink()
    (root / ".batch.lock").write_text("pid=1\n")
    with pytest.raises(RuntimeError, match="Batch lock exists"):
        ds.run(["--config", str(path), "--execute"], backend=FakeBackend(icp))
    (root / ".batch.lock").unlink()
    assert ds.run(["--config", str(path), "--execute", "--limit", "1"], backend=FakeBackend(icp)) == 0
    (root / "records/i0000/w0001.part").mkdir(parents=True)
    with pytest.raises(ValueError, match="Incomplete .part exists"):
        ds.run(["--config", str(path), "--execute", "--resume"], backend=FakeBackend(icp))
    assert not (root / ".batch.lock").exists()


def test_io_failure_mid_record_stops_the_run(ds, icp, tmp_path, monkeypatch):
    """Host-side fault injection: the disk fails while the third record's arrays are written (an
    OSError from the NPY writer, as a full disk raises).  The run stops at that record with the
    error, keeps its <record>.part for inspection (never reused), writes no receipt for it, keeps
    the two completed records and their receipts, and releases the batch lock; a resume then
    refuses until the .part is moved away by hand, and completes the plan after that."""
    import shutil

    cfg = copy.deepcopy(CONFIG)
    root = tmp_path / "out"
    cfg["output_root"] = str(root)
    path = _write(tmp_path, cfg)
    real = ds.write_npy
    calls = {"n": 0}

    def failing(p, a):
        calls["n"] += 1
        if calls["n"] == 8:  # second array of the third record
            raise OSError(28, "No space left on device (injected)")
        return real(p, a)

    monkeypatch.setattr(ds, "write_npy", failing)
    with pytest.raises(OSError, match="injected"):
        ds.run(["--config", str(path), "--execute"], backend=FakeBackend(icp))
    monkeypatch.setattr(ds, "write_npy", real)
    assert not (root / ".batch.lock").exists()
    assert sorted(p.name for p in (root / "receipts").iterdir()) == ["i0000_w0000.json", "i0000_w0001.json"]
    part = root / "records/i0001/w0000.part"
    assert part.is_dir() and not (root / "records/i0001/w0000").exists()
    validate_record(root / "records/i0000/w0001")
    with pytest.raises(ValueError, match="Incomplete .part exists"):
        ds.run(["--config", str(path), "--execute", "--resume"], backend=FakeBackend(icp))
    shutil.move(str(part), str(tmp_path / "inspected.part"))
    fake = FakeBackend(icp)
    assert ds.run(["--config", str(path), "--execute", "--resume"], backend=fake) == 0
    assert fake.calls == [[(1, 0), (1, 1)]]
    assert json.loads((root / "progress.json").read_text())["complete"] is True


def test_device_allocation_failure_stops_the_run(ds, icp, tmp_path):
    """Host-side fault injection: the device library fails a batch with its device error (an
    allocation that cudaMalloc refused).  The run ends with that error before writing any record
    of the batch, the lock is released, and a resume from the same plan completes every record."""
    cfg = copy.deepcopy(CONFIG)
    root = tmp_path / "out"
    cfg["output_root"] = str(root)
    path = _write(tmp_path, cfg)

    class FailingBackend(FakeBackend):
        def generate(self, ctx, c, todo):
            self.calls.append(list(todo))
            raise icp.IcpError(icp.ICP_ERR_DEVICE, "c->b_mass.ensure(...) failed: out of memory (injected)")

    with pytest.raises(icp.IcpError, match="out of memory"):
        ds.run(["--config", str(path), "--execute"], backend=FailingBackend(icp))
    assert not (root / ".batch.lock").exists()
    assert not (root / "receipts").exists() or not any((root / "receipts").iterdir())
    if (root / "records").exists():
        assert not list((root / "records").rglob("*.part"))
    fake = FakeBackend(icp)
    assert ds.run(["--config", str(path), "--execute", "--resume"], backend=fake) == 0
    assert json.loads((root / "progress.json").read_text())["completed"] == 4


@pytest.mark.gpu
def test_batched_dataset_on_gpu(ds, icp, tmp_path):
    cfg = copy.deepcopy(CONFIG)
    cfg["output_root"] = str(tmp_path / "a")
    assert ds.run(["--config", str(_write(tmp_path, cfg)), "--execute"]) == 0
    other = copy.deepcopy(cfg)
    other["output_root"] = str(tmp_path / "b")
    other["b200"]["batch_records"] = 1
    assert ds.run(["--config", str(_write(tmp_path, other)), "--execute"]) == 0
    for ii in range(2):
        for ll in range(2):
            a = validate_record(tmp_path / f"a/records/i{ii:04d}/w{ll:04d}")
            b = validate_record(tmp_path / f"b/records/i{ii:04d}/w{ll:04d}")
            # records do not depend on how the conditions were batched
            assert np.abs(a["cell_probability"] - b["cell_probability"]).sum() <= 1e-12
            m = a["metadata"]
            assert m["incident_inclination_degrees"] == [-15.0, 15.0][ii]
            assert m["wavelength_nm"] == float(np.float32([500.0, 600.0][ll]))
            t = m["transport_audit"]
            assert abs((t["escaped_mm2"] + t["unresolved_mm2"]) / t["incident_mm2"] - 1) <= 1e-12
    assert ds.run(["--config", str(_write(tmp_path, cfg)), "--execute", "--resume"]) == 0


def test_lattice_stage_command_is_the_reference_orchestrators(ds, tmp_path):
    """A patch-model record is one rainbow_generate process with the options the reference's
    orchestrator passes (tools/generate_phase_dataset.py:296-311)."""
    cfg = copy.deepcopy(CONFIG)
    cfg["solver"].update(stage="diffraction", allow_underresolved=True)
    c = ds.normalized_config(cfg)
    args = ds.lattice_command("gen", tmp_path / "rec", c, 1, 0)
    assert args[0] == "gen" and "--allow-underresolved" in args and "--sphere" not in args
    pairs = dict(zip(args[1:-1:2], args[2:-1:2]))
    assert pairs["--stage"] == "diffraction" and pairs["--grid"] == "129" and pairs["--material"] == "water"
    assert pairs["--wavelength-nm"] == c["wavelength_nm"][0] and pairs["--inclination-deg"] == c["inclination_degrees"][1]
    assert pairs["--focal-offsets"] == "0,0,0,0" and pairs["--out"] == str(tmp_path / "rec")


@pytest.mark.gpu
def test_lattice_stage_dataset_on_gpu(ds, tmp_path):
    """Stage path through the orchestrator: one rainbow_generate per record, every record verified,
    receipted and re-verified on --resume."""
    cfg = copy.deepcopy(CONFIG)
    cfg["radius_mm"] = 0.5
    cfg["solver"].update(stage="path", grid=33, query_theta=36, query_phi=72, cdf_theta=18, cdf_phi=36)
    cfg["output_root"] = str(tmp_path / "out")
    path = _write(tmp_path, cfg)
    assert ds.run(["--config", str(path), "--execute"]) == 0
    recs = sorted((tmp_path / "out" / "records").glob("i*/w*"))
    assert len(recs) == 4
    for r in recs:
        m = validate_record(r)["metadata"]
        assert m["stage"] == "path" and m["generator_version"] == "icp_b200.rainbow.lattice.v1"
    plan = json.loads((tmp_path / "out" / "batch_plan.json").read_text())
    assert "rainbow_generate" in plan["binary_sha256"]
    assert ds.run(["--config", str(path), "--execute", "--resume"]) == 0
