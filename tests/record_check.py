"""Record validation for the tests: every record this repository writes is held to the contract
the reference's record reader enforces (python/rainbow_dataset/record.py:19-158,
PhaseRecord(validate=True)).  Where the reference checkout is present (ICP_REFERENCE_ROOT, by
default the checkout this build was made against), validate_record also opens the record with
that reader itself, unchanged; on hosts without it (the GPU box) the restatement below stands in.

The contract, as checked here: a complete v1/v2 record (not a .part directory); fixed layout
strings; positive int32 grid sizes; three <f8 C-order arrays of the right shapes with no
trailing bytes; a right-handed orthonormal sampling frame (2e-12); strictly increasing u edges
from 0 to 1; a marginal CDF from 0 to 1, non-decreasing; conditional CDFs in [0, 1] from 0 to 1,
non-decreasing; for v2, the HG label is the first moment of the saved cells (5e-12, mass 1e-10).
"""
from __future__ import annotations

import importlib.util
import json
import os
from pathlib import Path

import numpy as np

REFERENCE = Path(os.environ.get("ICP_REFERENCE_ROOT", "/root/reference"))
_READER: list = []


def reference_reader():
    """The reference's PhaseRecord class, imported by path from its checkout, or None."""
    if not _READER:
        path = REFERENCE / "python" / "rainbow_dataset" / "record.py"
        cls = None
        if path.is_file():
            spec = importlib.util.spec_from_file_location("reference_rainbow_record", path)
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            cls = mod.PhaseRecord
        _READER.append(cls)
    return _READER[0]

FIXED = {"dtype": "<f8", "order": "C", "density_measure": "solid_angle_sr",
         "cell_model": "constant_density_per_spherical_cell", "coordinates": "u=(1-cos(theta))/2; v=(phi+pi)/(2*pi)",
         "normalization": "integral_p_domega_equals_one", "input_polarization": "unpolarized",
         "cdf_axis_order": ["phi_cell", "theta_edge"]}
HG = {"method": "first_moment_of_saved_cell_pdf", "target": "saved_cdf",
      "cosine_convention": "dot(incident_propagation,outgoing_propagation)"}


def _array(path: Path, shape: tuple) -> np.ndarray:
    a = np.load(path, mmap_mode="r", allow_pickle=False)
    ok = a.dtype.str == "<f8" and a.shape == shape and a.flags.c_contiguous
    if not ok or path.stat().st_size != a.offset + a.nbytes:
        raise ValueError(f"{path.name}: layout or length differs from the record contract")
    return np.array(a)


def _fail(what: str) -> None:
    raise ValueError(f"record contract: {what}")


def validate_record(directory: str | Path) -> dict:
    d = Path(directory)
    reader = reference_reader()
    if reader is not None:
        rec = reader(d, validate=True)  # raises on any violation of its contract
        close = getattr(rec, "close", None)
        if close:
            close()
    if d.name.endswith(".part"):
        _fail("a .part directory is incomplete")
    m = json.loads((d / "metadata.json").read_text(encoding="utf-8"))
    v2 = m.get("schema") == "rainbow.phase_cdf.numpy.v2"
    if not (v2 or m.get("schema") == "rainbow.phase_cdf.numpy.v1") or m.get("complete") is not True:
        _fail("schema / completeness")
    for key in (k for k, v in FIXED.items() if m.get(k) != v):
        _fail(f"field {key}")
    nt, np_ = m["theta_count"], m["phi_count"]
    if not all(type(n) is int and 0 < n < 2 ** 31 for n in (nt, np_)):
        _fail("grid size")
    a = _array(d / "phi_cdf.npy", (np_ + 1,))
    t = _array(d / "theta_given_phi_cdf.npy", (np_, nt + 1))
    u = _array(d / "u_edges.npy", (nt + 1,))
    f = np.asarray(m["sampling_frame_columns"], dtype=np.float64)
    dt = np.diff(t, axis=1)
    checks = {
        "sampling frame": f.shape == (3, 3) and np.isfinite(f).all()
        and np.max(np.abs(f.T @ f - np.eye(3))) <= 2e-12 and abs(np.linalg.det(f) - 1) <= 2e-12,
        "u edges": np.isfinite(u).all() and u[0] == 0 and u[-1] == 1 and bool(np.all(np.diff(u) > 0)),
        "marginal CDF": np.isfinite(a).all() and a[0] == 0 and a[-1] == 1 and bool(np.all(np.diff(a) >= 0)),
        "conditional CDF range": np.isfinite(t).all() and bool(np.all((t >= 0) & (t <= 1))),
        "conditional CDF ends": bool(np.all(t[:, 0] == 0) and np.all(t[:, -1] == 1)),
        "conditional CDF order": bool(np.all(dt >= 0)),
    }
    for what in (k for k, ok in checks.items() if not ok):
        _fail(what)
    cells = np.diff(a)[:, None] * dt
    if v2:
        hg = m.get("hg", {})
        if any(hg.get(k) != v for k, v in HG.items()):
            _fail("HG convention")
        g = hg.get("g")
        if type(g) not in (int, float) or not np.isfinite(g) or not -1 < g < 1:
            _fail("HG value")
        q = cells.astype(np.longdouble)
        total = q.sum()
        axial = (q * (1.0 - (u[:-1] + u[1:])).astype(np.longdouble)[None, :]).sum()
        if abs(float(total) - 1.0) > 1e-10 or abs(float(axial / total) - float(g)) > 5e-12:
            _fail("HG label differs from the saved CDF's first moment")
    return {"metadata": m, "phi": a, "theta": t, "u": u, "cell_probability": cells}
