"""Deterministic single-particle atlas on the B200: precompute and orientation composition.

Drop-in for the reference's M3/M4 atlas path:
  * ``precompute`` replaces ice_precompute_atlas (hex_atlas/apps/precompute_atlas.cpp): for every
    incident node of the symmetry domain, the projected-area quadrature rays are traced on the
    device (icp_atlas_trace_node) and the node's raw cell flux (mm^2) is stored in the same
    directory contract -- metadata.json (schema ice.single_particle_atlas.v1), mass_mm2.npy
    [incident_theta, incident_phi, theta, phi] and u_edges.npy -- written through <dir>.part and
    renamed when complete.  The ice index comes from the Warren & Brandt (2008) table
    (icp_ice_index) unless a constant index is given explicitly.
  * ``compose`` replaces compose_atlas.py / atlas_math.py: the fixed orientation product rule
    (orientation_rule), the coupling weights of each incident direction (icp_atlas_coupling,
    one device thread per orientation, exact fixed-point sums, the analytic azimuth average at
    exact vertical incidence) and the direct cyclic convolution (icp_atlas_compose), then the
    ordered CDF build (icp_phase_cdf_build) -- records in rainbow.phase_cdf.numpy.v2 under
    records/i####/w####, batch_plan.json last, all through <out>.part.

No random numbers: entry points come from a quadrature, orientations from a product rule.

    python -m ice_crystal_phase_b200.atlas precompute --out DIR --radius-mm R --length-mm L --wavelength-nm NM ...
    python -m ice_crystal_phase_b200.atlas compose --atlas DIR [DIR ...] --config CONFIG.json --out OUT
    python -m ice_crystal_phase_b200.atlas spectrum --plan PLAN.json --atlas-root DIR --out OUT [--reuse] [--dry-run]

``spectrum`` replaces hex_atlas/tools/run_spectrum.py: one dispersive-ice atlas per wavelength
(cached with a job receipt, reused only for an identical request and library build), then one
composition over all wavelengths.
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import json
import math
import sys
import time
from pathlib import Path
from typing import Any

import numpy as np

import ice_crystal_phase_b200 as icp

PI = math.pi
EPS = float(np.finfo(np.float64).eps)
ATLAS_SCHEMA = "ice.single_particle_atlas.v1"
SYMMETRY = "D6h_O3_full_24_scalar_unpolarized"
RECONSTRUCTION = "bilinear_theta_phi_in_spherical_incident_frame"
GENERATOR = "icp_b200.deterministic_atlas.v1"


# ------------------------------------------------------------------ orientation rule
def count_in(x: Any, name: str, top: int = 1_000_000) -> int:
    """A JSON integer (not a bool, not a float) in 1..top."""
    if type(x) is int and 0 < x <= top:
        return x
    raise ValueError(f"{name}: expected an integer from 1 to {top}, got {x!r}")


def unit(v: Any) -> np.ndarray:
    """v scaled by its largest component, then by its length (the tracer's normalisation)."""
    a = np.asarray(v, dtype=np.float64)
    big = float(np.max(np.abs(a))) if a.shape == (3,) and np.isfinite(a).all() else 0.0
    if big == 0.0:
        raise ValueError("Expected finite nonzero three-vector")
    a = a / big
    return a / math.sqrt(float(a @ a))


def gaussian_tilt_nodes(count: int, sigma_deg: float) -> np.ndarray:
    """Tilts beta of the horizontal Gaussian model: the midpoints in probability of `count`
    equal-probability strata of N(pi/2, sigma^2) truncated to [0, pi], density in d beta (no
    sin beta factor), found by 64 bisection steps of the erf CDF; sigma = 0 is an exact delta
    (atlas_math.py:75-106)."""
    count_in(count, "tilt count")
    sigma = math.radians(float(sigma_deg))
    if not math.isfinite(sigma) or sigma < 0:
        raise ValueError("sigma_deg must be finite and nonnegative")
    if sigma == 0:
        return np.full(count, PI / 2)
    norm = math.erf(PI / (2 * math.sqrt(2) * sigma))
    if not norm > 0:
        raise ValueError("Gaussian normalization is not representable")
    out = np.empty(count)
    for i in range(count):
        goal = 2 * ((i + .5) / count) - 1
        lo, hi = 0.0, PI
        for _ in range(64):
            mid = (lo + hi) / 2
            if math.erf((mid - PI / 2) / (math.sqrt(2) * sigma)) / norm < goal:
                lo = mid
            else:
                hi = mid
        out[i] = (lo + hi) / 2
    if count > 1 and np.any(np.diff(out) <= 0):
        raise ValueError("Positive Gaussian width is below angular resolution; use explicit sigma_deg=0 for a delta")
    return out


def _ry(a: np.ndarray) -> np.ndarray:
    c, s = np.cos(a), np.sin(a)
    z, o = np.zeros_like(a), np.ones_like(a)
    return np.stack([np.stack([c, z, s], -1), np.stack([z, o, z], -1), np.stack([-s, z, c], -1)], -2)


def _rz(a: np.ndarray) -> np.ndarray:
    c, s = np.cos(a), np.sin(a)
    z, o = np.zeros_like(a), np.ones_like(a)
    return np.stack([np.stack([c, -s, z], -1), np.stack([s, c, z], -1), np.stack([z, z, o], -1)], -2)


def quaternion_matrix(q: Any) -> np.ndarray:
    q = np.asarray(q, dtype=np.float64)
    if q.shape != (4,) or not np.isfinite(q).all() or abs(float(q @ q) - 1) > 2e-12:
        raise ValueError("Fixed quaternion must be unit wxyz")
    w, x, y, z = q / math.sqrt(float(q @ q))
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def validate_rotations(r: np.ndarray, w: np.ndarray) -> None:
    """Proper rotations (R^T R = I and det R = 1 to 2e-12) with positive finite number weights
    summing to one (2e-12)."""
    shaped = r.ndim == 3 and r.shape[1:] == (3, 3) and len(r) > 0 and w.shape == (len(r),)
    if not shaped:
        raise ValueError("Malformed orientation quadrature")
    finite = np.isfinite(r).all() and np.isfinite(w).all()
    if not (finite and bool(np.all(w > 0)) and abs(math.fsum(w) - 1) <= 2e-12):
        raise ValueError("Nonfinite / nonpositive / unnormalized orientation weights")
    gram_error = np.max(np.abs(np.einsum("nki,nkj->nij", r, r) - np.eye(3)))
    if gram_error > 2e-12 or np.max(np.abs(np.linalg.det(r) - 1)) > 2e-12:
        raise ValueError("Orientation nodes must be proper orthogonal rotations")


def orientation_rule(config: dict[str, Any]) -> tuple[np.ndarray, np.ndarray, dict[str, Any]]:
    """Rotations R = Ry(alpha) Rz(beta) Ry(gamma) (body +y axis -> ensemble) and NUMBER weights
    of the fixed product rule: alpha midpoints of [0, 2 pi), beta from the model (isotropic:
    arccos of cos-midpoints; horizontal_gaussian: gaussian_tilt_nodes), gamma midpoints of
    [0, pi/3) (uniform spin of a hexagonal prism); a fixed component is one quaternion.  Each
    component keeps its fraction (atlas_math.py:109-161)."""
    if set(config) != {"quadrature", "components"}:
        raise ValueError("orientation keys must be quadrature and components")
    q = config["quadrature"]
    if set(q) != {"azimuth", "tilt", "spin"}:
        raise ValueError("quadrature keys must be azimuth, tilt, spin")
    na, nb, ng = (count_in(q[k], k, 4096) for k in ("azimuth", "tilt", "spin"))
    comps = config["components"]
    if not isinstance(comps, list) or not comps:
        raise ValueError("Nonempty orientation components required")
    fractions = [float(c["fraction"]) for c in comps]
    if any(not math.isfinite(f) or not 0 < f <= 1 for f in fractions) or abs(math.fsum(fractions) - 1) > 1e-12:
        raise ValueError("Positive NUMBER fractions must sum to one")
    mats, wts, counts = [], [], []
    for c, f in zip(comps, fractions):
        kind = c["kind"]
        keys = {"kind", "fraction"} | ({"sigma_deg"} if kind == "horizontal_gaussian" else
                                       {"quaternion_wxyz"} if kind == "fixed" else set())
        if set(c) != keys:
            raise ValueError(f"Unknown/missing component keys for {kind}")
        if kind == "fixed":
            mats.append(quaternion_matrix(c["quaternion_wxyz"])[None])
            wts.append(np.array([f]))
            counts.append(1)
            continue
        if kind == "isotropic":
            betas = np.arccos(1 - 2 * (np.arange(nb) + .5) / nb)
        elif kind == "horizontal_gaussian":
            betas = gaussian_tilt_nodes(nb, c["sigma_deg"])
        else:
            raise ValueError("Supported models: isotropic, horizontal_gaussian, fixed")
        if na * nb * ng > 2_000_000:
            raise ValueError("Too many explicit quadrature nodes")
        left = _ry(2 * PI * (np.arange(na) + .5) / na)
        tilted = left[:, None] @ _rz(betas)[None, :]
        spin = _ry((PI / 3) * (np.arange(ng) + .5) / ng)
        mats.append((tilted[:, :, None] @ spin[None, None, :]).reshape(-1, 3, 3))
        wts.append(np.full(na * nb * ng, f / (na * nb * ng)))
        counts.append(na * nb * ng)
    r, w = np.concatenate(mats), np.concatenate(wts)
    validate_rotations(r, w)
    return r, w, {"kind": "deterministic_probability_midpoint_product_quadrature", "config": config,
                  "component_nodes": counts, "rotation": "Ry(alpha)_Rz(beta)_Ry(gamma)_body_to_ensemble",
                  "horizontal_density_measure": "d_beta; truncated normal on [0,pi]", "uniform_spin_range": [0, PI / 3],
                  "randomness": False, "cdf_weights_analytic": True, "optical_integral_analytic": False}


def incidents(config: dict[str, Any]) -> list[tuple[np.ndarray, dict[str, Any]]]:
    """Incident directions: inclinations alpha -> ki = (cos alpha, -sin alpha, 0), exactly
    (0, -+1, 0) at +-90; or explicit direction vectors (compose_atlas.py:38-59)."""
    if ("inclinations_deg" in config) == ("directions" in config):
        raise ValueError("Specify exactly one of inclinations_deg or directions")

    def inclined(value: Any) -> tuple[np.ndarray, dict[str, Any]]:
        a = float(value)
        if not (math.isfinite(a) and abs(a) <= 90):
            raise ValueError("Inclination must be in [-90,90] degrees")
        r = math.radians(a)
        k = [0.0, -math.copysign(1.0, a), 0.0] if abs(a) == 90 else [math.cos(r), -math.sin(r), 0.0]
        return unit(k), {"inclination_deg": a}

    out = ([inclined(v) for v in config["inclinations_deg"]] if "inclinations_deg" in config
           else [(unit(k), {}) for k in config["directions"]])
    if not 0 < len(out) <= 10000:
        raise ValueError("Require 1..10000 incident conditions")
    return out


def projected_area(radius: float, length: float, k: Any) -> float:
    u = unit(k)
    s3 = math.sqrt(3)
    normals = np.array([[1, 0, 0], [.5, 0, s3 / 2], [-.5, 0, s3 / 2], [-1, 0, 0], [-.5, 0, -s3 / 2], [.5, 0, -s3 / 2],
                        [0, 1, 0], [0, -1, 0]])
    areas = np.array([radius * length] * 6 + [3 * s3 * radius * radius / 2] * 2)
    return float(areas @ np.maximum(0, -normals @ u))


def canonical_frame(theta: float, phi: float) -> np.ndarray:
    st, ct, sp, cp = math.sin(theta), math.cos(theta), math.sin(phi), math.cos(phi)
    k = np.array([st * cp, ct, st * sp])
    e = np.array([ct * cp, -st, ct * sp])
    return np.column_stack((e, np.cross(k, e), k))


# ------------------------------------------------------------------ files
def sha256_file(path: Path) -> str:
    h = hashlib.sha256()
    with path.open("rb") as f:
        for block in iter(lambda: f.read(1 << 20), b""):
            h.update(block)
    return h.hexdigest()


def _write_json(path: Path, value: Any) -> None:
    with path.open("x", encoding="utf-8", newline="\n") as f:
        json.dump(value, f, ensure_ascii=True, allow_nan=False, indent=2)
        f.write("\n")


def _write_npy(path: Path, value: np.ndarray) -> None:
    with path.open("xb") as f:
        np.save(f, np.ascontiguousarray(value, dtype="<f8"), allow_pickle=False)


def _staging(out: Path) -> Path:
    if out.name in ("", ".", "..") or out.name.endswith(".part") or out.exists():
        raise ValueError("Output must be a new named directory, not .part")
    part = out.with_name(out.name + ".part")
    out.parent.mkdir(parents=True, exist_ok=True)
    part.mkdir()  # exclusive: an existing incomplete run is neither removed nor adopted
    return part


def material_json(wavelength_nm: float, interior_index: float | None, exterior_index: float) -> dict[str, Any]:
    """Material block of the atlas metadata (write_material_json, hex_atlas/src/ice_optics.cpp:31-47)."""
    if interior_index is None:
        s = icp.evaluate_ice_optics(wavelength_nm)
        return {"model": "ice_ih_warren_brandt_2008_real_only", "wavelength_convention": "vacuum_nm",
                "wavelength_nm": wavelength_nm, "wavelength_requested_nm": wavelength_nm,
                "wavelength_evaluated_nm": wavelength_nm, "interior_index": s.n, "exterior_index": exterior_index,
                "interior_index_evaluated_fp64": s.n, "interior_index_solver_fp64": s.n,
                "automatic_ice_dispersion": True, "absorption": False, "birefringence": False,
                "absorption_model": "ignored_k_equals_zero", "kappa_solver": 0, "source_doi": "10.1029/2007JD009744",
                "reference_state": "ice_Ih_near_melting_compilation", "supported_nm": [200, 1100],
                "n_interpolation": "linear_n_in_log_vacuum_wavelength",
                "kappa_interpolation": "linear_log_kappa_in_log_vacuum_wavelength",
                "temperature_dependence_computed": False, "kappa_evaluated_not_used": s.kappa,
                "bracket_nm": [s.lower_nm, s.upper_nm], "log_wavelength_fraction": s.log_wavelength_fraction}
    return {"model": "constant", "wavelength_convention": "vacuum_nm", "wavelength_nm": wavelength_nm,
            "wavelength_requested_nm": wavelength_nm, "wavelength_evaluated_nm": wavelength_nm,
            "interior_index": interior_index, "exterior_index": exterior_index,
            "interior_index_evaluated_fp64": interior_index, "interior_index_solver_fp64": interior_index,
            "automatic_ice_dispersion": False, "absorption": False, "birefringence": False,
            "absorption_model": "ignored_k_equals_zero", "kappa_solver": 0}


# ------------------------------------------------------------------ precompute
def settings(circumradius_mm: float, length_mm: float, interior_index: float, theta_intervals: int,
             phi_intervals: int, nt: int, np_: int, subdivisions: int, exterior_index: float = 1.0,
             max_internal_hits: int = 2048, tail_tolerance: float = 1e-12, max_unresolved_fraction: float = 1e-10,
             max_balance_error: float = 1e-10) -> icp.AtlasSettings:
    return icp.AtlasSettings(float(circumradius_mm), float(length_mm), float(interior_index), float(exterior_index),
                             int(theta_intervals), int(phi_intervals), int(nt), int(np_), int(subdivisions),
                             int(max_internal_hits), float(tail_tolerance), float(max_unresolved_fraction),
                             float(max_balance_error))


def trace_node(ctx: icp.Context, s: icp.AtlasSettings, i: int, j: int,
               mass: icp.DeviceArray | None = None) -> tuple[np.ndarray, icp.AtlasNodeReport]:
    """Cell masses (mm^2, [nt][np]) and report of incident node (i, j)."""
    m = mass or icp.DeviceArray(ctx, s.nt * s.np)
    rep = icp.AtlasNodeReport()
    icp.check(icp.LIB.icp_atlas_trace_node(ctx.handle, C.byref(s), int(i), int(j), m.ptr, C.byref(rep)))
    return m.download().reshape(s.nt, s.np), rep


def precompute(ctx: icp.Context, out: Path, s: icp.AtlasSettings, wavelength_nm: float,
               constant_index: bool = False, log=print) -> Path:
    """Writes one atlas directory (every incident node traced on the device)."""
    if not (wavelength_nm > 0 and math.isfinite(wavelength_nm)):
        raise ValueError("--wavelength-nm is required (vacuum nm).")
    material = material_json(wavelength_nm, s.interior_index if constant_index else None, s.exterior_index)
    if not constant_index:
        s.interior_index = material["interior_index"]
    part = _staging(Path(out))
    ni, nj = s.theta_intervals + 1, s.phi_intervals + 1
    mass = np.lib.format.open_memmap(part / "mass_mm2.npy", mode="w+", dtype="<f8", shape=(ni, nj, s.nt, s.np))
    _write_npy(part / "u_edges.npy", icp.u_edges(s.nt))
    dev = icp.DeviceArray(ctx, s.nt * s.np)
    nodes, total = [], 0
    for i in range(ni):
        for j in range(nj):
            m, rep = trace_node(ctx, s, i, j, dev)
            mass[i, j] = m
            node = icp.atlas_incident_node(s.theta_intervals, s.phi_intervals, i, j)
            nodes.append({"i": i, "j": j, "theta": node.theta, "phi": node.phi, "ki": list(node.ki),
                          "e0": list(node.e0), "projected_area_mm2": rep.projected_area_mm2,
                          "escaped_mm2": rep.escaped_mm2, "unresolved_mm2": rep.unresolved_mm2,
                          "histogram_relative_error": rep.histogram_relative_error, "rays": rep.rays,
                          "outputs": rep.outputs, "max_balance_error": rep.max_balance_error,
                          "max_interface_balance_error": rep.max_interface_balance_error})
            total += rep.rays
            log(f"atlas_node={i},{j} rays={rep.rays} residual={rep.unresolved_mm2 / rep.projected_area_mm2:.17g}")
    mass.flush()
    del mass
    dev.free()
    meta = {"schema": ATLAS_SCHEMA, "complete": True, "backend": "cuda_fixed_point_exact_histogram",
            "generator_version": GENERATOR, "dtype": "<f8", "order": "C",
            "mass_axes": ["incident_theta", "incident_phi", "theta", "phi"],
            "incident_theta_intervals": s.theta_intervals, "incident_phi_intervals": s.phi_intervals,
            "theta_count": s.nt, "phi_count": s.np,
            "geometry": {"shape": "regular_hexagonal_prism", "circumradius_mm": s.circumradius_mm,
                         "full_length_mm": s.length_mm, "body_long_axis": [0, 1, 0]},
            "material": material, "symmetry": SYMMETRY, "incident_reconstruction": RECONSTRUCTION,
            "incident_formula": "k=(sin(t)cos(p),cos(t),sin(t)sin(p));e0=(cos(t)cos(p),-sin(t),cos(t)sin(p));e1=k_cross_e0",
            "area_quadrature": {"rule": "composite_equal_area_GL2xGL3", "subdivisions": s.subdivisions,
                                "randomness": False},
            "transport": {"path_rule": "R_and_T_R_power_m_T", "polarization": "two_input_JonesFlux",
                          "interference": False, "diffraction": False, "tail_tolerance": s.tail_tolerance,
                          "max_internal_hits": s.max_internal_hits,
                          "max_unresolved_fraction": s.max_unresolved_fraction,
                          "max_balance_error": s.max_balance_error},
            "pole_policy": "axis_mass_uniform_in_azimuth_in_histogram_end_cap",
            "accumulation": "exact_64bit_fixed_point_2^-62_of_node_quadrature_weight",
            "nodes": nodes, "total_rays": total, "numerical_convergence_certified": False}
    _write_json(part / "metadata.json", meta)
    part.rename(out)
    log(f"atlas_complete nodes={ni * nj} rays={total}")
    return Path(out)


# ------------------------------------------------------------------ reader
class Atlas:
    """A complete atlas directory, validated as the reference's composer does (atlas_math.py:235-269)."""

    def __init__(self, directory: str | Path):
        self.directory = d = Path(directory)
        if d.name.endswith(".part"):
            raise ValueError("Incomplete atlas directory")
        self.meta = m = json.loads((d / "metadata.json").read_text(encoding="utf-8"))
        if m.get("schema") != ATLAS_SCHEMA or m.get("complete") is not True:
            raise ValueError("Incomplete or unknown atlas schema")
        if (m.get("incident_reconstruction"), m.get("symmetry")) != (RECONSTRUCTION, SYMMETRY):
            raise ValueError("Unsupported atlas frame/interpolation/symmetry")
        self.it = count_in(m["incident_theta_intervals"], "incident_theta_intervals", 4096)
        self.ip = count_in(m["incident_phi_intervals"], "incident_phi_intervals", 4096)
        self.nt, self.np = count_in(m["theta_count"], "theta_count"), count_in(m["phi_count"], "phi_count")
        self.mass = np.load(d / "mass_mm2.npy", mmap_mode="r", allow_pickle=False)
        self.edges = e = np.load(d / "u_edges.npy", allow_pickle=False)
        g = m["geometry"]
        self.radius, self.length = float(g["circumradius_mm"]), float(g["full_length_mm"])
        grid = (self.it + 1, self.ip + 1)
        layout = [
            ("Atlas mass layout does not match metadata", self.mass.shape == (*grid, self.nt, self.np)
             and self.mass.dtype.str == "<f8" and self.mass.flags.c_contiguous),
            ("Invalid atlas u edges", e.shape == (self.nt + 1,) and e.dtype.str == "<f8" and np.isfinite(e).all()
             and e[0] == 0 and e[-1] == 1 and bool(np.all(np.diff(e) > 0))),
            ("Missing incident atlas nodes", len(m["nodes"]) == grid[0] * grid[1]),
            ("Unsupported geometry", g["shape"] == "regular_hexagonal_prism" and self.radius > 0 and self.length > 0),
        ]
        for what, ok in layout:
            if not ok:
                raise ValueError(what)
        nodes = m["nodes"]
        if [(n["i"], n["j"]) for n in nodes] != [divmod(k, grid[1]) for k in range(len(nodes))]:
            raise ValueError("Node order mismatch")
        acct = np.array([[float(n[k]) for k in ("projected_area_mm2", "unresolved_mm2", "escaped_mm2")]
                         for n in nodes])
        area, residual, escaped = acct.T
        for k, n in enumerate(nodes):
            i, j = divmod(k, grid[1])
            f = canonical_frame(i * (PI / 2) / self.it, j * (PI / 6) / self.ip)
            if max(np.max(np.abs(np.array(n["ki"]) - f[:, 2])), np.max(np.abs(np.array(n["e0"]) - f[:, 0]))) > 2e-12:
                raise ValueError("Node frame mismatch")
            cell = self.mass[i, j]
            if not (np.isfinite(cell).all() and bool(np.all(cell >= 0))):
                raise ValueError("Invalid atlas cell mass")
            if not (np.isfinite(acct[k]).all() and area[k] > 0 and escaped[k] > 0 and residual[k] >= 0):
                raise ValueError("Invalid node accounting")
            audits = (abs((escaped[k] + residual[k]) / area[k] - 1) <= 2e-10,
                      abs(float(np.sum(cell)) / escaped[k] - 1) <= 2e-10,
                      abs(area[k] / projected_area(self.radius, self.length, n["ki"]) - 1) <= 2e-12)
            if not all(audits):
                raise ValueError("Node area / mass / residual audit failed")
        self.area, self.residual = area.reshape(grid), residual.reshape(grid)
        self.hashes = {n: sha256_file(d / n) for n in ("metadata.json", "mass_mm2.npy", "u_edges.npy")}

    @property
    def nodes(self) -> int:
        return (self.it + 1) * (self.ip + 1)


# ------------------------------------------------------------------ composition
class Composer:
    """Device state of one composition run: the rule's rotations and weights, one atlas's node
    masses, the coupling and composed-mass buffers."""

    def __init__(self, ctx: icp.Context, first: Atlas):
        self.ctx, self.first = ctx, first
        self.coupling = icp.DeviceArray(ctx, first.nodes * 2 * first.np)
        self.out = icp.DeviceArray(ctx, first.nt * first.np)
        self.mass = icp.DeviceArray(ctx, first.nodes * first.nt * first.np)
        self.loaded: Atlas | None = None
        self._rule: tuple[np.ndarray, np.ndarray, icp.DeviceArray, icp.DeviceArray] | None = None

    def _upload(self, rot: np.ndarray, w: np.ndarray) -> tuple[icp.DeviceArray, icp.DeviceArray]:
        """Device copies of a rule's rotations / weights; the last rule stays resident (kept
        together with its host arrays, compared by identity)."""
        if self._rule is not None and self._rule[0] is rot and self._rule[1] is w:
            return self._rule[2], self._rule[3]
        r = np.ascontiguousarray(rot.reshape(-1, 9), dtype=np.float64)
        d = (icp.DeviceArray(self.ctx, r.size).upload(r),
             icp.DeviceArray(self.ctx, len(w)).upload(np.asarray(w, np.float64)))
        self._rule = (rot, w, *d)
        return d

    def add_coupling(self, rot: np.ndarray, w: np.ndarray, ki: np.ndarray, fraction: float, orbit: bool) -> float:
        a = self.first
        d_rot, d_w = self._upload(rot, w)
        n = len(w)
        k = (C.c_double * 3)(*map(float, ki))
        area = np.ascontiguousarray(a.area.reshape(-1))
        expected = C.c_double()
        icp.check(icp.LIB.icp_atlas_coupling(self.ctx.handle, a.it, a.ip, a.np, a.radius, a.length,
                                             area.ctypes.data_as(icp._D), d_rot.ptr, d_w.ptr, n, k, float(fraction),
                                             int(orbit), self.coupling.ptr, C.byref(expected)))
        return expected.value

    def coupling_for_rule(self, rot: np.ndarray, w: np.ndarray, ki: Any, rule_meta: dict[str, Any]
                          ) -> tuple[np.ndarray, float, np.ndarray, dict[str, Any]]:
        """Coupling weights of one incident direction (coupling_for_rule, atlas_math.py:313-428):
        at exact vertical incidence the uniform world azimuth of isotropic / horizontal_gaussian
        components is integrated exactly (one alpha node, the row mean); fixed poses and every
        other direction use the rule's own nodes."""
        k = unit(ki)
        f = _output_frame(k)
        vertical = bool(k[0] == 0.0 and k[2] == 0.0)
        comps = rule_meta["config"]["components"]
        eligible = [c["kind"] in ("isotropic", "horizontal_gaussian") for c in comps]
        self.coupling.zero()
        if not vertical or not any(eligible):
            area = self.add_coupling(rot, w, k, 1.0, False)
            info = {"method": "original_fixed_orientation_quadrature", "exact_vertical_incidence": vertical,
                    "analytic_uniform_azimuth_components": [], "effective_pose_evaluations": len(rot),
                    "symmetry_axis_ensemble": [0, 1, 0], "direction_snapped": False, "output_post_filter": False}
        else:
            ref_rot, ref_w, _ = orientation_rule(rule_meta["config"])
            if not np.array_equal(rot, ref_rot) or not np.array_equal(w, ref_w):
                raise ValueError("Analytic azimuth requires the declared orientation_rule arrays")
            parts, evaluations, modes = [], 0, []
            for comp, analytic in zip(comps, eligible):
                quad = dict(rule_meta["config"]["quadrature"])
                if analytic:
                    quad["azimuth"] = 1
                r1, w1, _ = orientation_rule({"quadrature": quad, "components": [dict(comp, fraction=1.0)]})
                parts.append(float(comp["fraction"]) * self.add_coupling(r1, w1, k, float(comp["fraction"]),
                                                                          analytic))
                evaluations += len(r1)
                modes.append("analytic_uniform_alpha" if analytic else "fixed_pose")
            area = math.fsum(parts)
            info = {"method": "analytic_uniform_world_azimuth_at_vertical_incidence", "exact_vertical_incidence": True,
                    "analytic_uniform_azimuth_components": [i for i, x in enumerate(eligible) if x],
                    "component_methods": modes, "reference_pose_count": len(rot),
                    "effective_pose_evaluations": evaluations, "symmetry_axis_ensemble": [0, 1, 0],
                    "direction_snapped": False, "output_post_filter": False,
                    "tilt_spin_and_atlas_interpolation_remain_numerical": True}
        wts = self.coupling.download().reshape(self.first.nodes, 2, self.first.np)
        represented = float(np.sum(np.sum(wts, axis=(1, 2)) * self.first.area.reshape(-1)))
        if not area > 0 or not np.isfinite(wts).all() or np.any(wts < 0) or abs(represented / area - 1) > 1e-11:
            raise ValueError("Orientation-to-convolution area audit failed")
        return wts, area, f, info

    def compose(self, atlas: Atlas, wts: np.ndarray) -> tuple[icp.DeviceArray, float]:
        """Composed cell masses (device, [nt][np]) of `atlas` under the current coupling, and the
        propagated unresolved area."""
        if self.loaded is not atlas:
            self.mass.upload(np.ascontiguousarray(atlas.mass).reshape(-1))
            self.loaded = atlas
        icp.check(icp.LIB.icp_atlas_compose(self.ctx.handle, atlas.nodes, atlas.nt, atlas.np, self.mass.ptr,
                                            self.coupling.ptr, self.out.ptr))
        residual = float(np.sum(np.sum(wts, axis=(1, 2)) * atlas.residual.reshape(-1)))
        return self.out, residual


def _output_frame(k: np.ndarray) -> np.ndarray:
    kk, e0, e1 = icp.make_frame(k)
    return np.column_stack((np.array(e0), np.array(e1), np.array(kk)))


def cdf(ctx: icp.Context, mass: icp.DeviceArray, nt: int, np_: int) -> tuple[np.ndarray, np.ndarray, dict]:
    """Ordered FP64 phi marginal and theta|phi CDFs of the composed masses, audited
    (icp_phase_cdf_build at the full grid: l1 <= 1e-10, lost <= 1e-12)."""
    res = icp.PhaseCdf(ctx).build(mass, nt, np_)
    return res.phi, res.theta, res.report


def record_metadata(a: Atlas, expected: float, residual: float, rep: dict, frame: np.ndarray,
                    plan_hash: str, rule_meta: dict, condition: dict, info: dict, contract: str,
                    total: float) -> dict[str, Any]:
    g = rep["g_stored"]
    material = dict(a.meta["material"])
    material.setdefault("wavelength_convention", "vacuum_nm")
    geom = dict(a.meta["geometry"], projected_area_mm2=expected, projected_area_m2=expected * 1e-6,
                projected_area_method="deterministic_orientation_quadrature_of_exact_facet_projection")
    meta = {"schema": "rainbow.phase_cdf.numpy.v2", "complete": True, "generator_version": GENERATOR,
            "backend": "b200_deterministic_atlas_convolution", "dtype": "<f8", "order": "C",
            "theta_count": a.nt, "phi_count": a.np, "density_measure": "solid_angle_sr",
            "cell_model": "constant_density_per_spherical_cell", "coordinates": "u=(1-cos(theta))/2; v=(phi+pi)/(2*pi)",
            "cdf_axis_order": ["phi_cell", "theta_edge"], "normalization": "integral_p_domega_equals_one",
            "input_polarization": "unpolarized", "direction_convention": "physical_propagation",
            "theta_zero": "forward", "theta_pi": "backward", "azimuth_periodic": True, "phi_range_rad": [-PI, PI],
            "coordinate_contract_id": ("rainbow.phase_cdf.coordinates.v1" if contract == "rainbow"
                                       else "ice.phase_cdf.ensemble_coordinates.v1"),
            "sampling_frame_layout": "rows_xyz_columns_e0_e1_k",
            "sampling_frame_map": ("local_column_to_particle_column" if contract == "rainbow"
                                   else "local_column_to_ensemble_reference_column"),
            "sampling_frame_columns": frame.tolist(), "query_frame_axis": frame[:, 2].tolist(),
            "query_frame_e0": frame[:, 0].tolist(), "particle_up_axis": [0, 1, 0], "shape_polar_axis": [0, -1, 0],
            "wavelength_nm": material["wavelength_nm"], "interior_index": material["interior_index"],
            "exterior_index": material["exterior_index"], "geometry": geom, "material": material,
            "cross_sections": {"model": "geometric_nonabsorbing", "scattering_mm2": expected, "extinction_mm2": expected,
                               "absorption_mm2": 0, "scattering_m2": expected * 1e-6, "extinction_m2": expected * 1e-6,
                               "absorption_m2": 0, "wave_scattering_cross_section_computed": False},
            "single_scattering_albedo": 1, "stage": "incoherent",
            "diffraction_policy": {"computed": False, "selected_output_includes_diffraction": False},
            "inter_path_interference": False, "tir_relative_phase_retained": True,
            "orientation": {"representation": "deterministic_SO3_number_quadrature", "rule": rule_meta,
                            "plan_sha256": plan_hash, "randomness": False, "azimuth_integration": info},
            "atlas": {"files_sha256": a.hashes, "incident_theta_intervals": a.it, "incident_phi_intervals": a.ip,
                      "angular_reconstruction": "A_normalized_bilinear_theta_phi_in_incident_spherical_frame",
                      "symmetry": "D6h_including_reflections", "transform": "phi_shift_or_phi_reflection_then_shift",
                      "azimuth_remap": "exact_overlap_of_piecewise_constant_equal_width_cells", "no_retracing": True},
            "transport_audit": {"escaped_mm2": total, "unresolved_mm2": residual,
                                "unresolved_fraction": residual / expected, "balance_error": (total + residual) / expected - 1,
                                "cdf_normalized_to_resolved_escaped_mass": True},
            "storage_processing": {"gaussian_sigma_degrees": 0, "coarsening_tv": 0,
                                   "mass_conservative_aggregation": False, "g_source": g, "g_stored": g},
            "hg": {"g": g, "axis_particle_frame": frame[:, 2].tolist(), "method": "first_moment_of_saved_cell_pdf",
                   "target": "saved_cdf", "cosine_convention": "dot(incident_propagation,outgoing_propagation)"},
            "condition": condition,
            "quality": {"cdf_mass": rep["cdf_mass"], "cdf_l1_mass_error": rep["l1_error"],
                        "cdf_lost_probability_mass": rep["lost_mass"],
                        "cdf_maximum_cell_mass_error": rep["maximum_cell_error"],
                        "orientation_convergence_certified": False, "incident_atlas_convergence_certified": False,
                        "angular_convergence_certified": False, "maximum_accepted_l1_mass_error": 1e-10,
                        "maximum_accepted_lost_probability_mass": 1e-12}}
    if contract == "rainbow":
        k = frame[:, 2]
        meta["incident_inclination_degrees"] = math.degrees(math.atan2(-k[1], max(0.0, k[0])))
    return meta


def compose(ctx: icp.Context, atlas_paths: list[Path], config_path: Path, out: Path,
            output_contract: str = "rainbow", log=print) -> Path:
    """Records for every (incident direction, atlas wavelength) of the configuration."""
    with Path(config_path).open(encoding="utf-8") as f:
        config = json.load(f)
    if set(config) - {"orientation", "inclinations_deg", "directions"} or "orientation" not in config:
        raise ValueError("Unknown/missing composition configuration keys")
    if output_contract not in ("rainbow", "ensemble"):
        raise ValueError("Unknown output contract")
    cases = incidents(config)
    atlases = [Atlas(p) for p in atlas_paths]
    if not atlases:
        raise ValueError("At least one atlas is required")
    first = atlases[0]
    rot, w, rule_meta = orientation_rule(config["orientation"])
    if output_contract == "rainbow":
        for k, _ in cases:
            if abs(k[2]) > 2e-14 or k[0] < -2e-14:
                raise ValueError("Noncanonical incident direction is not RainbowReference-compatible; "
                                 "select --output-contract ensemble explicitly")
    for a in atlases[1:]:
        if ((a.it, a.ip, a.nt, a.np) != (first.it, first.ip, first.nt, first.np) or
                a.meta["geometry"] != first.meta["geometry"] or not np.array_equal(a.edges, first.edges) or
                not np.array_equal(a.area, first.area)):
            raise ValueError("Batch atlases must share geometry, angular grids, and areas")
        for key in ("model", "exterior_index", "absorption", "birefringence"):
            if a.meta["material"].get(key) != first.meta["material"].get(key):
                raise ValueError("A spectral batch must use one material model and exterior medium")
        if a.meta["transport"] != first.meta["transport"]:
            raise ValueError("A spectral batch must use one transport/audit policy")
    wavelengths = [float(a.meta["material"]["wavelength_nm"]) for a in atlases]
    if len(set(wavelengths)) != len(wavelengths):
        raise ValueError("Unique positive wavelength per atlas required")
    part = _staging(Path(out))
    _write_json(part / "orientation_model.json", rule_meta)
    _write_npy(part / "orientation_rotations.npy", rot)
    _write_npy(part / "orientation_weights.npy", w)
    plan_files = {n: sha256_file(part / n) for n in ("orientation_model.json", "orientation_rotations.npy",
                                                     "orientation_weights.npy")}
    plan_hash = hashlib.sha256(json.dumps(plan_files, sort_keys=True).encode("ascii")).hexdigest()
    plan: dict[str, Any] = {"schema": "ice.deterministic_phase_dataset.v1", "complete": False,
                            "output_contract": output_contract, "per_record_schema": "rainbow.phase_cdf.numpy.v2",
                            "condition_axes": ["incident", "wavelength"],
                            "incident_directions": [k.tolist() for k, _ in cases], "wavelengths_nm": wavelengths,
                            "orientation_plan_sha256": plan_hash, "orientation_files_sha256": plan_files,
                            "input_config": config, "atlases": [a.hashes for a in atlases],
                            "computation": "deterministic_offline_mass_convolution_no_raytracing", "records": []}
    _write_json(part / "generation_plan.json", plan)
    comp = Composer(ctx, first)
    for i, (ki, condition) in enumerate(cases):
        wts, expected, frame, info = comp.coupling_for_rule(rot, w, ki, rule_meta)
        for wi, a in enumerate(atlases):
            mass, residual = comp.compose(a, wts)
            host = mass.download()
            total = math.fsum(host)
            if (abs((total + residual) / expected - 1) > 2e-10 or
                    residual / expected > a.meta["transport"]["max_unresolved_fraction"] + 2e-15):
                raise ValueError("Composed mass and unresolved area fail the transport audit")
            phi, theta, rep = cdf(ctx, mass, a.nt, a.np)
            rel = Path("records") / f"i{i:04d}" / f"w{wi:04d}"
            rec = part / rel
            rec.mkdir(parents=True)
            _write_npy(rec / "phi_cdf.npy", phi)
            _write_npy(rec / "theta_given_phi_cdf.npy", theta)
            _write_npy(rec / "u_edges.npy", a.edges)
            _write_json(rec / "metadata.json", record_metadata(a, expected, residual, rep, frame, plan_hash, rule_meta,
                                                               condition, info, output_contract, total))
            hashes = {n: sha256_file(rec / n) for n in ("metadata.json", "phi_cdf.npy", "theta_given_phi_cdf.npy",
                                                        "u_edges.npy")}
            plan["records"].append({"incident_index": i, "wavelength_index": wi, "path": rel.as_posix(),
                                    "condition": [wavelengths[wi], -float(ki[1])], "ki": ki.tolist(),
                                    "wavelength_nm": wavelengths[wi], "g": rep["g_stored"], "files_sha256": hashes,
                                    "azimuth_integration": info})
            log(f"record i={i} w={wi} g={rep['g_stored']:.17g} A={expected:.17g}")
    plan["complete"] = True
    _write_json(part / "batch_plan.json", plan)
    if Path(out).exists():
        raise FileExistsError("Destination appeared while composing")
    part.rename(out)
    return Path(out)


# ------------------------------------------------------------------ spectral runner
SPECTRUM_REQUIRED = {"radius_mm", "length_mm", "incident_theta_intervals", "incident_phi_intervals", "theta", "phi",
                     "area_subdivisions", "batch_rays", "max_work_mib"}
SPECTRUM_OPTIONAL = {"max_internal_hits", "tail_tolerance", "max_unresolved_fraction", "max_balance_error"}
SPECTRUM_INTEGERS = {"incident_theta_intervals", "incident_phi_intervals", "theta", "phi", "area_subdivisions",
                     "batch_rays", "max_work_mib", "max_internal_hits"}


def read_spectrum_plan(path: Path) -> dict[str, Any]:
    """A spectral plan: wavelengths_nm (unique, ascending, 200..1100), precompute settings of one
    ice prism, and one composition (inclinations and orientation model); everything is
    validated before any work (run_spectrum.py:29-63).  batch_rays / max_work_mib size the
    reference's per-ray histogram columns: required and validated, but they limit nothing here
    (the device histogram is exact fixed point without per-ray columns)."""
    with Path(path).open(encoding="utf-8") as f:
        plan = json.load(f)
    if set(plan) != {"wavelengths_nm", "precompute", "composition"}:
        raise ValueError("Plan requires only wavelengths_nm, precompute, composition")
    st = plan["precompute"]
    if not isinstance(st, dict) or not SPECTRUM_REQUIRED <= set(st) <= SPECTRUM_REQUIRED | SPECTRUM_OPTIONAL:
        raise ValueError("Missing/unknown precompute parameter")
    for k, v in st.items():
        if k in SPECTRUM_INTEGERS:
            if type(v) is not int or v <= 0:
                raise ValueError(f"{k} must be a positive integer")
        elif type(v) not in (int, float) or not math.isfinite(v) or v < 0:
            raise ValueError(f"{k} must be a finite nonnegative number")
    if min(st["radius_mm"], st["length_mm"]) <= 0:
        raise ValueError("Particle dimensions must be positive")
    waves = plan["wavelengths_nm"]
    if (not isinstance(waves, list) or not waves or len(set(waves)) != len(waves) or
            any(type(w) not in (int, float) or not math.isfinite(w) or not 200 <= w <= 1100 for w in waves)):
        raise ValueError("Unique vacuum wavelengths in 200..1100 nm are required")
    if sorted(waves) != waves:
        raise ValueError("Wavelengths must be listed in increasing order (stable w-index)")
    cfg = plan["composition"]
    if set(cfg) != {"inclinations_deg", "orientation"}:
        raise ValueError("This fixed-condition runner requires inclination angles and one orientation model")
    if len(set(cfg["inclinations_deg"])) != len(incidents(cfg)):
        raise ValueError("Duplicate incident conditions")
    orientation_rule(cfg["orientation"])
    return plan


def atlas_name(wavelength: float) -> str:
    return "lambda_" + format(float(wavelength), ".17g").replace(".", "p") + "_nm"


def verify_spectral_atlas(path: Path, wave: float, st: dict[str, Any]) -> dict[str, Any]:
    """A cached atlas is the requested dispersive-ice calculation (run_spectrum.py:70-95); the
    Atlas reader then audits every node."""
    if path.name.endswith(".part"):
        raise ValueError("Incomplete atlas")
    m = json.loads((path / "metadata.json").read_text(encoding="utf-8"))
    if m.get("complete") is not True or m.get("schema") != ATLAS_SCHEMA:
        raise ValueError("Incomplete/unknown cached atlas")
    mat = m["material"]
    if (mat.get("model") != "ice_ih_warren_brandt_2008_real_only" or mat.get("automatic_ice_dispersion") is not True
            or mat.get("wavelength_nm") != wave or mat.get("exterior_index") != 1):
        raise ValueError("Cached atlas is not the requested dispersive ice calculation")
    grid = {"incident_theta_intervals": st["incident_theta_intervals"],
            "incident_phi_intervals": st["incident_phi_intervals"], "theta_count": st["theta"], "phi_count": st["phi"]}
    if any(m.get(k) != v for k, v in grid.items()):
        raise ValueError("Cached angular grid differs from request")
    if (m["geometry"]["circumradius_mm"] != st["radius_mm"] or m["geometry"]["full_length_mm"] != st["length_mm"]
            or m["area_quadrature"]["subdivisions"] != st["area_subdivisions"]):
        raise ValueError("Cached geometry/area quadrature differs from request")
    for f in ("mass_mm2.npy", "u_edges.npy"):
        if not (path / f).is_file():
            raise ValueError("Missing cached atlas array")
    return m


def spectrum(plan_path: Path, atlas_root: Path, out: Path, reuse: bool = False, dry_run: bool = False,
             device: int = 0, log=print) -> None:
    """Atlases of every wavelength (ice index from the table), cached under atlas_root with a job
    receipt each and reused only when the request and the library build match, then one
    composition over all of them (run_spectrum.py:98-169)."""
    plan = read_spectrum_plan(plan_path)
    out, atlas_root = Path(out), Path(atlas_root)
    if out.exists() or out.with_name(out.name + ".part").exists():
        raise ValueError("Use a new CDF output directory; existing output/.part is never replaced")
    st = plan["precompute"]
    raw = 8 * (st["incident_theta_intervals"] + 1) * (st["incident_phi_intervals"] + 1) * st["theta"] * st["phi"]
    waves = plan["wavelengths_nm"]
    log(f"PLAN: {len(waves)} wavelengths x {len(plan['composition']['inclinations_deg'])} incidents")
    log(f"RAW ATLAS: {raw / 1024 ** 3:.3f} GiB/wavelength; {raw * len(waves) / 1024 ** 3:.3f} GiB total "
        "(plus headers/metadata/CDFs)")
    paths = [atlas_root / atlas_name(w) for w in waves]
    if dry_run:
        for w, p in zip(waves, paths):
            log(f"python -m ice_crystal_phase_b200.atlas precompute --material ice --wavelength-nm {w} "
                f"--radius-mm {st['radius_mm']} --length-mm {st['length_mm']} "
                f"--incident-theta-intervals {st['incident_theta_intervals']} "
                f"--incident-phi-intervals {st['incident_phi_intervals']} --theta {st['theta']} --phi {st['phi']} "
                f"--area-subdivisions {st['area_subdivisions']} --out {p}")
        log("DRY RUN: no files were created and no data were generated")
        return
    build = {"library_sha256": sha256_file(icp.LIB_PATH)}
    atlas_root.mkdir(parents=True, exist_ok=True)
    with icp.Context(device) as ctx:
        for index, (wave, path) in enumerate(zip(waves, paths)):
            receipt = path.with_name(path.name + ".job.json")
            expected = {"schema": "ice.spectral_atlas_job.v1", "wavelength_nm": wave, "precompute": st,
                        "material": "ice", "build": build}
            if path.exists():
                if not reuse:
                    raise FileExistsError("Atlas exists; use --reuse for validated matching jobs: " + str(path))
                old = json.loads(receipt.read_text(encoding="utf-8"))
                if old.get("request") != expected or old.get("complete") is not True:
                    raise ValueError("Cached atlas arguments/build differ; use another atlas-root")
                if old.get("metadata_sha256") != sha256_file(path / "metadata.json"):
                    raise ValueError("Cached metadata changed since the recorded job")
                verify_spectral_atlas(path, wave, st)
                log(f"REUSE {index + 1}/{len(paths)}: wavelength_nm={wave}")
                continue
            if receipt.exists() or path.with_name(path.name + ".part").exists():
                raise FileExistsError("Unfinished job or stale receipt; inspect it before retrying: " + str(path))
            s = settings(st["radius_mm"], st["length_mm"], 0.0, st["incident_theta_intervals"],
                         st["incident_phi_intervals"], st["theta"], st["phi"], st["area_subdivisions"],
                         max_internal_hits=st.get("max_internal_hits", 2048),
                         tail_tolerance=st.get("tail_tolerance", 1e-12),
                         max_unresolved_fraction=st.get("max_unresolved_fraction", 1e-10),
                         max_balance_error=st.get("max_balance_error", 1e-10))
            started = time.perf_counter()
            with path.with_name(path.name + ".log").open("w", encoding="utf-8") as job_log:
                precompute(ctx, path, s, float(wave), log=lambda line: print(line, file=job_log))
            verify_spectral_atlas(path, wave, st)
            _write_json(receipt, {"complete": True, "request": expected,
                                  "metadata_sha256": sha256_file(path / "metadata.json"),
                                  "seconds": time.perf_counter() - started})
            log(f"ATLAS {index + 1}/{len(paths)}: wavelength_nm={wave}; seconds={time.perf_counter() - started:.3f}")
        payload = json.dumps(plan["composition"], sort_keys=True, ensure_ascii=True, allow_nan=False).encode("ascii")
        cfg_path = atlas_root / ("composition_" + hashlib.sha256(payload).hexdigest() + ".json")
        if cfg_path.exists():
            if json.loads(cfg_path.read_text(encoding="utf-8")) != plan["composition"]:
                raise ValueError("Composition configuration cache mismatch")
        else:
            _write_json(cfg_path, plan["composition"])
        compose(ctx, paths, cfg_path, out, "rainbow", log=log)
    log("COMPLETE: " + ascii(str(out)))


# ------------------------------------------------------------------ CLI
def main(argv: list[str] | None = None) -> int:
    p = argparse.ArgumentParser(prog="python -m ice_crystal_phase_b200.atlas", description=__doc__.split("\n\n")[0])
    sub = p.add_subparsers(dest="cmd", required=True)
    q = sub.add_parser("precompute")
    q.add_argument("--out", type=Path, required=True)
    q.add_argument("--radius-mm", type=float, required=True)
    q.add_argument("--length-mm", type=float, required=True)
    q.add_argument("--wavelength-nm", type=float, required=True)
    q.add_argument("--material", choices=["ice", "constant"], default="ice")
    q.add_argument("--ior", type=float)
    q.add_argument("--exterior-ior", type=float, default=1.0)
    q.add_argument("--incident-theta-intervals", type=int, required=True)
    q.add_argument("--incident-phi-intervals", type=int, required=True)
    q.add_argument("--theta", type=int, required=True)
    q.add_argument("--phi", type=int, required=True)
    q.add_argument("--area-subdivisions", type=int, required=True)
    q.add_argument("--max-internal-hits", type=int, default=2048)
    q.add_argument("--tail-tolerance", type=float, default=1e-12)
    q.add_argument("--max-unresolved-fraction", type=float, default=1e-10)
    q.add_argument("--max-balance-error", type=float, default=1e-10)
    q.add_argument("--device", type=int, default=0)
    c = sub.add_parser("compose")
    c.add_argument("--atlas", nargs="+", type=Path, required=True)
    c.add_argument("--config", type=Path, required=True)
    c.add_argument("--out", type=Path, required=True)
    c.add_argument("--output-contract", choices=["rainbow", "ensemble"], default="rainbow")
    c.add_argument("--device", type=int, default=0)
    sp = sub.add_parser("spectrum")
    sp.add_argument("--plan", type=Path, required=True)
    sp.add_argument("--atlas-root", type=Path, required=True)
    sp.add_argument("--out", type=Path, required=True)
    sp.add_argument("--reuse", action="store_true")
    sp.add_argument("--dry-run", action="store_true")
    sp.add_argument("--device", type=int, default=0)
    a = p.parse_args(argv)
    if a.cmd == "spectrum":
        try:
            spectrum(a.plan, a.atlas_root, a.out, a.reuse, a.dry_run, a.device)
        except Exception as e:  # noqa: BLE001
            print("SPECTRAL GENERATION FAILED: " + ascii(str(e)), file=sys.stderr)
            return 2
        return 0
    try:
        if a.cmd == "precompute":
            if a.material == "ice" and a.ior is not None:
                raise ValueError("Ice index is evaluated from wavelength; --ior requires explicit --material constant.")
            if a.material == "constant" and a.ior is None:
                raise ValueError("Constant material requires --ior.")
        with icp.Context(a.device) as ctx:
            if a.cmd == "precompute":
                s = settings(a.radius_mm, a.length_mm, a.ior or 0.0, a.incident_theta_intervals,
                             a.incident_phi_intervals, a.theta, a.phi, a.area_subdivisions, a.exterior_ior,
                             a.max_internal_hits, a.tail_tolerance, a.max_unresolved_fraction, a.max_balance_error)
                precompute(ctx, a.out, s, a.wavelength_nm, constant_index=a.material == "constant")
            else:
                compose(ctx, a.atlas, a.config, a.out, a.output_contract)
    except Exception as e:  # noqa: BLE001 -- the CLI reports and exits 2 like the reference's tools
        print(f"ice_crystal_phase_b200.atlas {a.cmd} failed: {e!a}", file=sys.stderr)
        return 2
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
