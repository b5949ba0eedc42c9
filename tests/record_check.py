"""Record validation used by the tests: the checks of the reference's record reader
(python/rainbow_dataset/record.py:19-158, PhaseRecord(validate=True)) restated, so that every
record this repository writes is held to the consumer's contract on hosts without the
reference checkout.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

SCHEMAS = {"rainbow.phase_cdf.numpy.v1", "rainbow.phase_cdf.numpy.v2"}


def load_npy(path: Path, shape: tuple) -> np.ndarray:
    a = np.load(path, mmap_mode="r", allow_pickle=False)
    if a.dtype.str != "<f8" or a.shape != shape or not a.flags.c_contiguous:
        raise ValueError(f"Unexpected shape/dtype/order in {path.name}")
    if path.stat().st_size != a.offset + a.nbytes:
        raise ValueError(f"Truncated or trailing data in {path.name}")
    return np.array(a)


def validate_record(directory: str | Path) -> dict:
    d = Path(directory)
    if d.name.endswith(".part"):
        raise ValueError("An incomplete .part directory is not a dataset record")
    m = json.loads((d / "metadata.json").read_text(encoding="utf-8"))
    if m.get("schema") not in SCHEMAS or m.get("complete") is not True:
        raise ValueError("Unknown schema or incomplete record")
    for key, expected in {"dtype": "<f8", "order": "C", "density_measure": "solid_angle_sr",
                          "cell_model": "constant_density_per_spherical_cell",
                          "coordinates": "u=(1-cos(theta))/2; v=(phi+pi)/(2*pi)",
                          "normalization": "integral_p_domega_equals_one", "input_polarization": "unpolarized"}.items():
        if m.get(key) != expected:
            raise ValueError(f"Unsupported {key}: {m.get(key)!r}")
    if m.get("cdf_axis_order") != ["phi_cell", "theta_edge"]:
        raise ValueError("Conditional CDF axes are not phi_cell, theta_edge")
    nt, np_ = m["theta_count"], m["phi_count"]
    if type(nt) is not int or type(np_) is not int or not (1 <= nt <= 0x7FFFFFFF and 1 <= np_ <= 0x7FFFFFFF):
        raise ValueError("Invalid angular dimension")
    a = load_npy(d / "phi_cdf.npy", (np_ + 1,))
    t = load_npy(d / "theta_given_phi_cdf.npy", (np_, nt + 1))
    u = load_npy(d / "u_edges.npy", (nt + 1,))
    frame = np.asarray(m["sampling_frame_columns"], dtype=np.float64)
    if (frame.shape != (3, 3) or not np.isfinite(frame).all()
            or not np.allclose(frame.T @ frame, np.eye(3), rtol=0, atol=2e-12)
            or not np.isclose(np.linalg.det(frame), 1.0, rtol=0, atol=2e-12)):
        raise ValueError("Sampling frame must be a right-handed orthonormal frame")
    if not np.isfinite(u).all() or u[0] != 0 or u[-1] != 1 or not np.all(np.diff(u) > 0):
        raise ValueError("u_edges are not strictly increasing from 0 to 1")
    if not np.isfinite(a).all() or a[0] != 0 or a[-1] != 1 or not np.all(np.diff(a) >= 0):
        raise ValueError("Marginal CDF is invalid")
    if not np.isfinite(t).all() or np.any(t < 0) or np.any(t > 1):
        raise ValueError("Conditional CDF contains nonfinite or out-of-range data")
    if np.any(t[:, 0] != 0) or np.any(t[:, -1] != 1):
        raise ValueError("Conditional CDF endpoints must be 0 and 1")
    if np.any(np.diff(t, axis=1) < 0):
        raise ValueError("Conditional CDF decreases; refusing to repair it")
    if m["schema"].endswith(".v2"):
        hg = m.get("hg", {})
        if (hg.get("method") != "first_moment_of_saved_cell_pdf" or hg.get("target") != "saved_cdf"
                or hg.get("cosine_convention") != "dot(incident_propagation,outgoing_propagation)"):
            raise ValueError("Unsupported HG moment convention")
        g = hg.get("g")
        if type(g) not in (int, float) or not np.isfinite(g) or not -1 < g < 1:
            raise ValueError("Invalid HG first moment")
        mean_mu = (1.0 - (u[:-1] + u[1:])).astype(np.longdouble)
        q = np.diff(a).astype(np.longdouble)[:, None] * np.diff(t, axis=1).astype(np.longdouble)
        mass = q.sum(dtype=np.longdouble)
        axial = (q * mean_mu[None, :]).sum(dtype=np.longdouble)
        if abs(float(mass) - 1.0) > 1e-10 or abs(float(axial / mass) - float(g)) > 5e-12:
            raise ValueError("HG label is inconsistent with saved CDF")
    return {"metadata": m, "phi": a, "theta": t, "u": u, "cell_probability": np.diff(a)[:, None] * np.diff(t, axis=1)}
