"""Resumable condition-grid dataset generation on the batched B200 drop path.

Drop-in for the reference's orchestrator (tools/generate_phase_dataset.py): the same config
file (output_root, generator, radius_mm, force_sphere, temperature_c, pressure_pa, wavelengths,
inclinations, solver, reserve_gib; an optional "b200" object adds rays, seed, precision,
max_internal_hits, diffraction and batch_records), the same command line, the same on-disk
contract -- batch_plan.json with a signature, a .batch.lock, records/i####/w#### written through
<record>.part -> rename, receipts/<job>.json verified on --resume, progress.json, a free-space
reserve -- and the same refusal to lower precision, skip or delete anything on failure.

What changes: the reference runs one rainbow_generate process per condition, one at a time
(generate_phase_dataset.py:296-311).  Here the ray-model records (stage "incoherent") go to the
GPU in batches of `batch_records` through one persistent launch (icp_drop_batch_generate); every
record keeps its own seed (derived from the condition indices), so a record does not depend on
how the run was batched, limited or resumed.  The patch-model stages (path, focal, diffraction)
run rainbow_generate once per record with the reference's options, as the reference does.
Records are written in rainbow_generate's format.

    python -m ice_crystal_phase_b200.dataset --config CONFIG.json [--execute] [--resume] [--limit N]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import math
import os
import shutil
import struct
import subprocess
import sys
import time
from contextlib import contextmanager
from decimal import Decimal, InvalidOperation
from pathlib import Path
from typing import Any, Iterator

import numpy as np

VERSION = "rainbow.condition_batch.v1"
GENERATOR_VERSION = "icp_b200.rainbow.v1"                # ray-model records (the batched library)
LATTICE_GENERATOR_VERSION = "icp_b200.rainbow.lattice.v1"  # patch-model records (rainbow_generate)
ARRAYS = ("phi_cdf.npy", "theta_given_phi_cdf.npy", "u_edges.npy")
B200_DEFAULTS = {"rays": 10_000_000, "seed": 12345, "precision": "fp32", "max_internal_hits": 1024,
                 "diffraction": False, "batch_records": 32, "max_unresolved_fraction": 1e-4}


# ------------------------------------------------------------------ config contract
# The accepted config file is the reference orchestrator's (generate_phase_dataset.py:33-152):
# exact decimal parsing of every number, JSON NaN / Infinity refused, booleans only where a
# flag is meant, the same ranges and the same condition grids.  Field tables drive the checks.
TOP_KEYS = frozenset({"output_root", "generator", "radius_mm", "force_sphere", "temperature_c", "pressure_pa",
                      "wavelengths", "inclinations", "solver", "reserve_gib"})
TOP_FIELDS = {"radius_mm": ("real", 1e-9, 3), "force_sphere": ("bool",), "temperature_c": ("real", 0, 60),
              "pressure_pa": ("real", 50000, 100000000)}
SOLVER_FIELDS = {"grid": ("int", 2, 32767), "query_theta": ("int", 1, 32767), "query_phi": ("int", 1, 32767),
                 "cdf_theta": ("int", 1, 32767), "cdf_phi": ("int", 1, 32767), "device": ("int", 0, 128),
                 "allow_underresolved": ("bool",), "maximum_coarsening_tv": ("real", 0, 1),
                 "cdf_max_l1": ("real", 0, 1), "cdf_max_lost_mass": ("real", 0, 1)}
SOLVER_KEYS = frozenset(SOLVER_FIELDS) | {"stage", "focal_offsets"}
B200_FIELDS = {"rays": ("int", 1, 10 ** 12), "seed": ("int", 0, 2 ** 62), "max_internal_hits": ("int", 1, 1 << 20),
               "diffraction": ("bool",), "batch_records": ("int", 1, 4096),
               "max_unresolved_fraction": ("real", 0, 0.999999)}
STAGES = ("diffraction", "focal", "path", "incoherent")


def _refuse_constant(name: str) -> None:
    raise ValueError(f"Nonfinite JSON constant: {name}")


def read_json_object(path: Path, limit: int = 8 << 20) -> dict[str, Any]:
    """A JSON object from a file of at most `limit` bytes (a UTF-8 BOM allowed, NaN refused)."""
    if path.stat().st_size > limit:
        raise ValueError(f"JSON too large: {path}")
    value = json.loads(path.read_text(encoding="utf-8-sig"), parse_constant=_refuse_constant)
    if not isinstance(value, dict):
        raise ValueError(f"Expected JSON object: {path}")
    return value


def field(value: Any, kind: str, low: Any = None, high: Any = None) -> Any:
    """One config value: "bool" (JSON true / false only), or a number read exactly as a decimal
    -- "dec" (any finite), "int" (integral in [low, high]) or "real" ([low, high], as float)."""
    if kind == "bool":
        if type(value) is not bool:
            raise ValueError("Expected JSON true or false")
        return value
    if type(value) is bool:
        raise ValueError("Boolean is not a numerical parameter")
    try:
        d = Decimal(str(value))
    except InvalidOperation as exc:
        raise ValueError(f"Invalid decimal: {value}") from exc
    if not d.is_finite():
        raise ValueError("Nonfinite parameter")
    if kind == "dec":
        return d
    if kind == "int":
        if d != d.to_integral_value() or not low <= d <= high:
            raise ValueError(f"Expected integer in [{low}, {high}]")
        return int(d)
    if not Decimal(str(low)) <= d <= Decimal(str(high)):
        raise ValueError(f"Parameter {value} is outside [{low}, {high}]")
    return float(d)


def real_field(value: Any, low: float, high: float) -> float:
    return field(value, "real", low, high)


def fp32(x: float) -> float:
    return float(np.float32(x))


def wavelength_grid(spec: dict[str, Any]) -> list[str]:
    """Wavelengths start, start + step, ..., stop (stop reached exactly) as decimal strings; no
    two may round to the same binary32 solver value (generate_phase_dataset.py:83-99)."""
    if set(spec) != {"start_nm", "stop_nm", "step_nm"}:
        raise ValueError("wavelengths needs start_nm, stop_nm, step_nm")
    start, stop, step = (field(spec[k], "dec") for k in ("start_nm", "stop_nm", "step_nm"))
    if step <= 0 or not 380 <= start <= stop <= 830:
        raise ValueError("Require 380 <= start <= stop <= 830 and positive step")
    steps, rest = divmod(stop - start, step)
    if rest:
        raise ValueError("The wavelength range must contain an integer number of steps; no silent endpoint truncation")
    if steps >= 100000:
        raise ValueError("Too many wavelengths")
    values = [format(start + step * i, "f") for i in range(int(steps) + 1)]
    if np.unique(np.array([float(v) for v in values], dtype=np.float32)).size != len(values):
        raise ValueError("Distinct wavelengths collapse to the same FP32 solver value")
    return values


def inclination_grid(spec: dict[str, Any]) -> list[str]:
    """Centres of `count` equal cells of [min, max] degrees as decimal strings, each computed as
    min + (max - min) (i + 1/2) / count (generate_phase_dataset.py:102-111)."""
    if set(spec) != {"min_degrees", "max_degrees", "count", "placement"}:
        raise ValueError("inclinations needs min_degrees, max_degrees, count, placement")
    if spec["placement"] != "linear_angle_cell_centers":
        raise ValueError("Only explicit linear_angle_cell_centers is supported")
    low, high = field(spec["min_degrees"], "dec"), field(spec["max_degrees"], "dec")
    count = field(spec["count"], "int", 1, 100000)
    if not -90 <= low < high <= 90:
        raise ValueError("Canonical inclination domain is [-90,90], NOT [0,180]")
    half = Decimal("0.5")
    return [format(low + (high - low) * (Decimal(i) + half) / count, "f") for i in range(count)]


def normalized_config(raw: dict[str, Any]) -> dict[str, Any]:
    """The checked, normalised conditions of a config file.  Beyond the reference's keys an
    optional "b200" object sets rays, seed, precision, max_internal_hits, diffraction and
    batch_records: the ray model of stage "incoherent".  The other stages (path, focal,
    diffraction) are the reference's patch model, one rainbow_generate process per record as in
    the reference; the "b200" settings do not apply to them."""
    keys = set(raw) - {"b200"}
    if keys != TOP_KEYS:
        raise ValueError(f"Unexpected/missing config keys: {keys ^ TOP_KEYS}")
    solver = raw["solver"]
    if not isinstance(solver, dict) or set(solver) != SOLVER_KEYS:
        raise ValueError("Invalid solver keys")
    out = {k: field(solver[k], *spec) for k, spec in SOLVER_FIELDS.items()}
    if 4 * out["grid"] ** 2 > 0xFFFFFFFF:
        raise ValueError("Source index range exceeds the existing solver contract")
    if any(out["cdf_" + a] > out["query_" + a] or out["query_" + a] % out["cdf_" + a] for a in ("theta", "phi")):
        raise ValueError("CDF grids must divide query grids")
    if solver["stage"] not in STAGES:
        raise ValueError("Unknown stage")
    out["stage"] = solver["stage"]
    offsets = solver["focal_offsets"]
    if not isinstance(offsets, list) or len(offsets) != 4:
        raise ValueError("Four focal offsets required")
    out["focal_offsets"] = [field(v, "int", 0, 3) for v in offsets]
    extra = raw.get("b200", {})
    if not isinstance(extra, dict) or not set(extra) <= set(B200_DEFAULTS):
        raise ValueError(f"b200 accepts only {sorted(B200_DEFAULTS)}")
    b = {**B200_DEFAULTS, **extra}
    b200 = {k: field(b[k], *spec) for k, spec in B200_FIELDS.items()}
    if b["precision"] not in ("fp32", "fp64"):
        raise ValueError("b200.precision must be fp32 or fp64")
    b200["precision"] = b["precision"]
    top = {k: field(raw[k], *spec) for k, spec in TOP_FIELDS.items()}
    return {**top, "wavelength_nm": wavelength_grid(raw["wavelengths"]),
            "inclination_degrees": inclination_grid(raw["inclinations"]),
            "inclination_placement": "linear_angle_cell_centers", "material": "water", "solver": out, "b200": b200}


def condition_seed(base: int, ii: int, ll: int) -> int:
    """Seed of condition (ii, ll): a SplitMix64 mix of the base seed and the indices."""
    x = (base + 0x9E3779B97F4A7C15 * (1 + ii * 100003 + ll)) & 0xFFFFFFFFFFFFFFFF
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return x ^ (x >> 31)


# ------------------------------------------------------------------ files
def sha256(path: Path) -> str:
    h = hashlib.sha256()
    with path.open("rb") as f:
        for block in iter(lambda: f.read(1 << 20), b""):
            h.update(block)
    return h.hexdigest()


def object_hash(value: Any) -> str:
    return hashlib.sha256(json.dumps(value, sort_keys=True, separators=(",", ":"), allow_nan=False).encode()).hexdigest()


def write_json(path: Path, value: Any) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_suffix(path.suffix + ".tmp")
    with tmp.open("w", encoding="utf-8", newline="\n") as f:
        json.dump(value, f, indent=2, ensure_ascii=False, allow_nan=False)
        f.write("\n")
    tmp.replace(path)


@contextmanager
def batch_lock(root: Path) -> Iterator[None]:
    """Exclusive writer lock of a dataset root (created with O_EXCL, removed on exit)."""
    lock = root / ".batch.lock"
    try:
        fd = os.open(lock, os.O_CREAT | os.O_EXCL | os.O_WRONLY, 0o644)
    except FileExistsError as exc:
        raise RuntimeError("Batch lock exists: another writer may be running. Remove a stale .batch.lock by hand "
                           "only after checking that no batch is running.") from exc
    with os.fdopen(fd, "w", encoding="ascii") as f:
        f.write(f"pid={os.getpid()}\n")
    try:
        yield
    finally:
        lock.unlink()


def write_npy(path: Path, array: np.ndarray) -> None:
    """NPY v1, <f8, C order, header padded to a 64-byte boundary, dictionary text as the
    command-line writers format it (bytes identical to rainbow_generate's files)."""
    a = np.ascontiguousarray(array, dtype="<f8")
    header = "{'descr': '<f8', 'fortran_order': False, 'shape': (" + "".join(f"{d}, " for d in a.shape) + "), }"
    header += " " * ((64 - (10 + len(header) + 1) % 64) % 64) + "\n"
    with path.open("xb") as f:
        f.write(b"\x93NUMPY\x01\x00" + struct.pack("<H", len(header)) + header.encode("latin1"))
        f.write(a.tobytes())


def npy_size(path: Path, expected_shape: tuple[int, ...]) -> int:
    """Byte size of a record array after checking its header (v1 or v2, <f8, C order, the
    expected shape) and that the file holds exactly that many values (no trailing data)."""
    fmt = np.lib.format
    with path.open("rb") as f:
        try:
            version = fmt.read_magic(f)
        except ValueError as exc:
            raise ValueError(f"Not NPY: {path}") from exc
        if version not in ((1, 0), (2, 0)):
            raise ValueError("Unsupported NPY version")
        try:
            shape, fortran, dtype = (fmt.read_array_header_1_0 if version == (1, 0) else fmt.read_array_header_2_0)(f)
        except ValueError as exc:
            raise ValueError(f"Invalid NPY header: {path}") from exc
        if dtype.str != "<f8" or fortran or tuple(shape) != tuple(expected_shape):
            raise ValueError(f"Wrong NPY layout: {path}")
        end = f.tell() + 8 * math.prod(expected_shape)
    if path.stat().st_size != end:
        raise ValueError(f"Truncated or trailing NPY data: {path}")
    return end


def near(a: Any, b: float, tol: float = 1e-12) -> bool:
    return type(a) in (int, float) and math.isfinite(a) and abs(a - b) <= tol * max(1.0, abs(b))


def _is_number(x: Any) -> bool:
    return type(x) in (int, float) and math.isfinite(x)


def _frame_ok(rows: Any, alpha_deg: float) -> str | None:
    """None, or what is wrong with sampling_frame_columns: a right-handed orthonormal 3x3 frame
    (columns e0, e1, k to 2e-12) whose k is (cos a, -sin a, 0) to 2e-6."""
    if not (isinstance(rows, list) and len(rows) == 3 and all(isinstance(r, list) and len(r) == 3 for r in rows)):
        return "frame shape"
    if not all(_is_number(v) for r in rows for v in r):
        return "frame values"
    cols = [[rows[r][j] for r in range(3)] for j in range(3)]
    if not all(near(sum(x * y for x, y in zip(cols[j], cols[k])), float(j == k), 2e-12)
               for j in range(3) for k in range(3)):
        return "frame orthogonality"
    e0, e1, kk = cols
    det = sum(c * d for c, d in zip((e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2],
                                     e0[0] * e1[1] - e0[1] * e1[0]), kk))
    if not det > 1 - 2e-12:
        return "frame handedness"
    a = math.radians(alpha_deg)
    if any(abs(v - w) >= 2e-6 for v, w in zip(kk, (math.cos(a), -math.sin(a), 0.0))):
        return "incident direction/sign"
    return None


def verify_record(path: Path, plan: dict[str, Any], ii: int, ll: int) -> dict[str, Any]:
    """The record checks the reference's orchestrator makes before it trusts a record on resume
    (generate_phase_dataset.py:227-287): the contract fields, the condition, the water model,
    the frame, the area and cross sections, the quality and storage gates, the array files.
    Returns the receipt digest of the record."""
    c, s = plan["conditions"], plan["conditions"]["solver"]
    m = read_json_object(path / "metadata.json", 1 << 20)
    alpha = float(c["inclination_degrees"][ii])
    geometry, cs, q = m.get("geometry", {}), m.get("cross_sections", {}), m.get("quality", {})
    sp, hg, material = m.get("storage_processing", {}), m.get("hg", {}), m.get("material", {})
    area = geometry.get("projected_area_mm2")
    version = GENERATOR_VERSION if s["stage"] == "incoherent" else LATTICE_GENERATOR_VERSION
    fields = {"complete": True, "schema": "rainbow.phase_cdf.numpy.v2", "generator_version": version,
              "coordinate_contract_id": "rainbow.phase_cdf.coordinates.v1",
              "direction_convention": "physical_propagation", "dtype": "<f8", "order": "C",
              "density_measure": "solid_angle_sr", "cdf_axis_order": ["phi_cell", "theta_edge"],
              "theta_count": s["cdf_theta"], "phi_count": s["cdf_phi"], "query_grid": [s["query_theta"], s["query_phi"]],
              "incident_grid": [s["grid"], s["grid"]], "stage": s["stage"], "force_sphere": c["force_sphere"],
              "focal_quarter_turn_offsets": s["focal_offsets"]}
    checks = [(f"mismatched {k}", m.get(k) == v) for k, v in fields.items()]
    checks += [("radius", near(m.get("radius_mm"), fp32(c["radius_mm"]))),
               ("wavelength", near(m.get("wavelength_nm"), fp32(float(c["wavelength_nm"][ll])))),
               ("inclination", near(m.get("incident_inclination_degrees"), alpha)),
               ("material", material.get("model") == "water_iapws_r9_97"),
               ("temperature", near(material.get("temperature_kelvin"), c["temperature_c"] + 273.15)),
               ("pressure", near(material.get("pressure_pascal"), c["pressure_pa"]))]
    for what, ok in checks:
        if not ok:
            raise ValueError(f"{path}: {what}")
    bad_frame = _frame_ok(m.get("sampling_frame_columns", []), alpha)
    lim = {"cdf_l1_mass_error": s["cdf_max_l1"], "cdf_lost_probability_mass": s["cdf_max_lost_mass"]}
    tv = sp.get("coarsening_tv")
    checks = [(bad_frame or "", bad_frame is None),
              ("projected area", _is_number(area) and area > 0),
              ("area validation", geometry.get("projected_area_converged") is True
               and geometry.get("convexity_verified") is True),
              ("cross-section model", cs.get("model") == "geometric_nonabsorbing"
               and cs.get("wave_scattering_cross_section_computed") is False),
              ("cross sections", cs.get("scattering_mm2") == area and cs.get("extinction_mm2") == area
               and cs.get("absorption_mm2") == 0),
              ("invalid optical data", q.get("invalid_values") == 0 and q.get("incomplete_directions") == 0),
              ("underresolution policy", q.get("allow_underresolved") is s["allow_underresolved"]),
              ("underresolution not authorized", s["allow_underresolved"] or q.get("underresolved_directions") == 0)]
    checks += [(k, _is_number(q.get(k)) and 0 <= q.get(k) <= bound) for k, bound in lim.items()]
    checks += [("unexpected global smoothing", sp.get("additional_filter") == "none"),
               ("coarsening error", _is_number(tv) and 0 <= tv <= s["maximum_coarsening_tv"]),
               ("HG target", hg.get("target") == "saved_cdf" and type(hg.get("g")) in (float, int)
                and -1 < hg["g"] < 1)]
    for what, ok in checks:
        if not ok:
            raise ValueError(f"{path}: {what}")
    nt, np_ = s["cdf_theta"], s["cdf_phi"]
    shapes = ((np_ + 1,), (np_, nt + 1), (nt + 1,))
    return {"metadata_sha256": sha256(path / "metadata.json"),
            "npy_sizes": {name: npy_size(path / name, shape) for name, shape in zip(ARRAYS, shapes)},
            "hg_g": hg["g"], "projected_area_mm2": area, "underresolved_directions": q.get("underresolved_directions"),
            "coarsening_tv": tv}


# ------------------------------------------------------------------ records
def record_metadata(c: dict, ii: int, ll: int, spec, rep, water) -> dict:
    """metadata.json in the layout rainbow_generate writes (apps/rainbow_generate.cpp)."""
    s, b = c["solver"], c["b200"]
    k, e0, e1 = list(rep.ki), list(rep.e0), list(rep.e1)
    area = rep.projected_area_mm2
    coeff = list(spec.coefficients)
    sphere = all(x == 0 for x in coeff[1:])
    t = rep.trace
    statuses = ["exhausted", "tail_tolerance_reached", "interaction_limit", "ambiguous_boundary", "invalid_input",
                "numerical_failure", "output_overflow", "replay_mismatch"]
    lam_f = fp32(float(c["wavelength_nm"][ll]))
    return {
        "coordinate_contract_id": "rainbow.phase_cdf.coordinates.v1", "direction_convention": "physical_propagation",
        "particle_frame_handedness": "right", "particle_up_axis": [0, 1, 0], "shape_polar_axis": [0, -1, 0],
        "sampling_frame_layout": "rows_xyz_columns_e0_e1_k", "sampling_frame_map": "local_column_to_particle_column",
        "theta_zero": "forward", "theta_pi": "backward", "azimuth_periodic": True,
        "inclination_definition": "ki=(cos(alpha),-sin(alpha),0); alpha=0 is +x; positive alpha points downward",
        "geometry": {"projected_area_mm2": area, "projected_area_m2": area * 1e-6,
                     "projected_area_method": "analytic_sphere" if sphere else
                     "convex_surface_integral_azimuth_analytic_gauss_legendre",
                     "projected_area_shape": "solver_shape_coefficients_promoted_to_fp64",
                     "projected_area_converged": True, "projected_area_error_is_rigorous_bound": False,
                     "convexity_verified": True,
                     "convexity_method": "analytic_sphere" if sphere else "dense_curvature_sampling",
                     "incident_axis_particle_frame": k, "sampled_disk_area_mm2": rep.sampled_area_mm2,
                     "traced_hit_area_mm2": rep.incident_area_mm2},
        "cross_sections": {"model": "geometric_nonabsorbing", "scattering_mm2": area, "extinction_mm2": area,
                           "absorption_mm2": 0, "scattering_m2": area * 1e-6, "extinction_m2": area * 1e-6,
                           "absorption_m2": 0, "assignment": "Csca=Cext=Aproj; Cabs=0 (transport model assumption)",
                           "wave_scattering_cross_section_computed": False},
        "material": {"model": "water_iapws_r9_97", "wavelength_convention": "vacuum_nm",
                     "wavelength_requested_nm": float(c["wavelength_nm"][ll]), "wavelength_evaluated_nm": lam_f,
                     "ambient_model": "unit_absolute_index_air_approximation",
                     "absorption_model": "ignored_k_equals_zero", "interior_index_evaluated_fp64": water.refractive_index,
                     "interior_index_solver_fp32": spec.interior_index, "exterior_index_solver": 1,
                     "refractive_index_release": "IAPWS R9-97",
                     "density_model": "IAPWS R6-95(2018) liquid pressure EOS inversion",
                     "temperature_kelvin": c["temperature_c"] + 273.15, "pressure_pascal": c["pressure_pa"],
                     "density_kg_m3": water.density_kg_m3,
                     "density_pressure_residual_pascal": water.density_pressure_residual_pascal,
                     "density_bracket_width_kg_m3": water.density_bracket_width_kg_m3},
        "diffraction_policy": {"name": "fraunhofer_equal_area_circle_v1" if spec.diffraction else "none",
                               "computed": bool(spec.diffraction),
                               "selected_output_includes_diffraction": bool(spec.diffraction),
                               "primary_sigma_degrees": None, "secondary_sigma_degrees": None,
                               "power_mm2": rep.diffraction_area_mm2,
                               "query_dtheta_degrees": 180.0 / s["query_theta"],
                               "query_dphi_degrees": 360.0 / s["query_phi"]},
        "schema": "rainbow.phase_cdf.numpy.v2", "complete": True, "dtype": "<f8", "order": "C",
        "theta_count": s["cdf_theta"], "phi_count": s["cdf_phi"], "density_measure": "solid_angle_sr",
        "cell_model": "constant_density_per_spherical_cell", "coordinates": "u=(1-cos(theta))/2; v=(phi+pi)/(2*pi)",
        "theta_definition": "angle_between_incident_and_outgoing_propagation_directions",
        "cdf_axis_order": ["phi_cell", "theta_edge"], "phi_range_rad": [-math.pi, math.pi],
        "normalization": "integral_p_domega_equals_one", "input_polarization": "unpolarized",
        "incident_total_intensity": 1, "single_scattering_albedo": 1, "collision_model": "geometric_projected_area",
        "projected_area_storage": "metadata.geometry.projected_area_mm2", "stage": s["stage"],
        "radius_mm": spec.radius_mm, "wavelength_nm": lam_f, "exterior_index": 1,
        "interior_index": spec.interior_index, "force_sphere": c["force_sphere"],
        "incident_grid": [s["grid"], s["grid"]], "incident_grid_used": False,
        "query_frame_axis": [fp32(x) for x in k], "query_frame_e0": [fp32(x) for x in e0],
        "sampling_frame_columns": [[e0[r], e1[r], k[r]] for r in range(3)], "shape_coefficients": coeff,
        "shape_source": "sphere" if c["force_sphere"] else "Sadeghi2012_TableI",
        "focal_quarter_turn_offsets": s["focal_offsets"], "diffraction_transition_contrast": 0,
        "generator_version": GENERATOR_VERSION,
        "backend": f"b200_batched_trace_{b['precision']}_fixed_point_histogram_cooperative_cdf",
        "sampling": {"generator": "counter_splitmix64_open52_v1", "method": "uniform_disk_covering_silhouette",
                     "rays": spec.rays, "seed": spec.seed, "missed_rays": t.missed, "outgoing_samples": t.outputs,
                     "weight": "disk_area / rays * path_power", "trace_precision": b["precision"]},
        "transport_audit": {"incident_mm2": rep.incident_area_mm2, "escaped_mm2": rep.escaped_area_mm2,
                            "unresolved_mm2": rep.unresolved_area_mm2,
                            "unresolved_fraction": rep.unresolved_area_mm2 / rep.incident_area_mm2,
                            "maximum_balance_error": t.max_ray_balance,
                            "maximum_interface_balance_error": t.max_interface_balance,
                            "max_internal_hits": b["max_internal_hits"], "tail_tolerance_per_ray": 1e-12,
                            "max_unresolved_fraction": b["max_unresolved_fraction"], "internal_encounters": t.encounters,
                            "status_counts": {statuses[i]: int(t.status_counts[i]) for i in range(8)}},
        "histogram": {"theta_count": s["query_theta"], "phi_count": s["query_phi"], "mass_mm2": rep.histogram_mass_mm2,
                      "relative_mass_audit_error": rep.histogram_relative_error,
                      "forward_axis_mass_mm2": rep.forward_mass_mm2, "backward_axis_mass_mm2": rep.backward_mass_mm2,
                      "boundary_snapped_samples": t.snapped},
        "quality": {"source_coverage_certified": False, "angular_convergence_certified": False,
                    "missing_source_cells": 0, "invalid_values": int(t.invalid), "incomplete_directions": 0,
                    "underresolved_directions": 0, "allow_underresolved": s["allow_underresolved"],
                    "cdf_l1_mass_error": rep.cdf.l1_error, "cdf_maximum_cell_mass_error": rep.cdf.maximum_cell_error,
                    "cdf_lost_positive_cells": int(rep.cdf.lost_cells), "cdf_lost_probability_mass": rep.cdf.lost_mass,
                    "maximum_accepted_l1_mass_error": s["cdf_max_l1"],
                    "maximum_accepted_lost_probability_mass": s["cdf_max_lost_mass"]},
        "incident_inclination_degrees": float(c["inclination_degrees"][ii]),
        "query_grid": [s["query_theta"], s["query_phi"]],
        "storage_processing": {"additional_filter": "none", "additional_filter_is_paper_diffraction": False,
                               "sigma_degrees": 0, "aggregation": "nested_solid_angle_mass_preserving",
                               "aggregation_integral_relative_change": rep.cdf.aggregation_relative_error,
                               "coarsening_tv": rep.cdf.coarsening_tv,
                               "maximum_accepted_coarsening_tv": s["maximum_coarsening_tv"]},
        "hg": {"g": rep.cdf.g_stored, "method": "first_moment_of_saved_cell_pdf", "target": "saved_cdf",
               "cosine_convention": "dot(incident_propagation,outgoing_propagation)", "axis_particle_frame": k,
               "g_source": rep.cdf.g_source, "cdf_mass_check": rep.cdf.cdf_mass},
        "timing": {"batch_seconds": rep.seconds_trace},
    }


def accept(rep, c: dict) -> None:
    """rainbow_generate's record gates: statuses other than exhausted / tail / interaction
    limit, balance, unbinnable exits, the global unresolved budget, the histogram audit."""
    t = rep.trace
    if (t.invalid or any(t.status_counts[i] for i in range(3, 8)) or not rep.incident_area_mm2 > 0
            or not rep.escaped_area_mm2 > 0 or not t.max_ray_balance <= 1e-10):
        raise RuntimeError("Drop trace is NOT accepted. Inspect per-ray statuses and unresolved power; "
                           "do not renormalize it away.")
    if rep.unresolved_area_mm2 / rep.incident_area_mm2 > c["b200"]["max_unresolved_fraction"]:
        raise RuntimeError("Unresolved light exceeds explicit global budget.")
    if abs((rep.escaped_area_mm2 + rep.unresolved_area_mm2) / rep.incident_area_mm2 - 1) > 1e-10:
        raise RuntimeError("Energy balance failed.")
    if rep.histogram_relative_error > 1e-10:
        raise RuntimeError("Histogram mass differs from independent escaped-ray audit.")


def write_record(path: Path, phi, theta, u, metadata: dict) -> None:
    part = Path(str(path) + ".part")
    if path.exists():
        raise FileExistsError(f"Dataset already exists; refusing to overwrite: {path}")
    part.mkdir(parents=True, exist_ok=False)
    write_npy(part / "phi_cdf.npy", phi)
    write_npy(part / "theta_given_phi_cdf.npy", theta)
    write_npy(part / "u_edges.npy", u)
    with (part / "metadata.json").open("x", encoding="utf-8", newline="\n") as f:
        json.dump(metadata, f, indent=2, allow_nan=False)
        f.write("\n")
    part.rename(path)


def lattice_command(exe: Path, out: Path, c: dict, ii: int, ll: int) -> list[str]:
    """The rainbow_generate command of one patch-model record: the options the reference's
    orchestrator passes (tools/generate_phase_dataset.py:296-311), so a record is the CLI's."""
    s = c["solver"]
    values = {"out": str(out), "material": "water", "radius-mm": str(c["radius_mm"]),
              "wavelength-nm": c["wavelength_nm"][ll], "inclination-deg": c["inclination_degrees"][ii],
              "temperature-c": str(c["temperature_c"]), "pressure-pa": str(c["pressure_pa"]),
              "grid": s["grid"], "query-theta": s["query_theta"], "query-phi": s["query_phi"],
              "cdf-theta": s["cdf_theta"], "cdf-phi": s["cdf_phi"], "stage": s["stage"],
              "device": s["device"], "max-coarsening-tv": s["maximum_coarsening_tv"],
              "cdf-max-l1": s["cdf_max_l1"], "cdf-max-lost-mass": s["cdf_max_lost_mass"],
              "focal-offsets": ",".join(map(str, s["focal_offsets"]))}
    args = [str(exe)]
    for k, v in values.items():
        args += ["--" + k, str(v)]
    if c["force_sphere"]:
        args.append("--sphere")
    if s["allow_underresolved"]:
        args.append("--allow-underresolved")
    return args


class GpuBackend:
    """The batched device library (a context for the run and one persistent launch per batch of
    ray-model records) and rainbow_generate for the patch-model stages."""

    def __init__(self, generator: Path | None = None):
        import ice_crystal_phase_b200 as icp  # noqa: PLC0415 (only needed to execute)

        self.icp = icp
        self.generator = Path(generator) if generator else Path(icp.__file__).resolve().parent / "bin" / "rainbow_generate"

    def library_sha256(self) -> str:
        return sha256(self.icp.LIB_PATH)

    def generator_sha256(self) -> str:
        return sha256(self.generator)

    def lattice_record(self, c: dict, ii: int, ll: int, path: Path) -> None:
        """One patch-model record written by rainbow_generate (through its own .part directory)."""
        r = subprocess.run(lattice_command(self.generator, path, c, ii, ll), capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"rainbow_generate failed for {path}: {(r.stderr or r.stdout).strip()[-2000:]}")

    def context(self, device: int):
        return self.icp.Context(device)

    def generate(self, ctx, c: dict, todo: list) -> list:
        return generate(self.icp, ctx, c, todo)


def generate(icp, ctx, c: dict, todo: list) -> list:
    """One GPU batch: todo = [(ii, ll), ...] -> (spec, water, phi, theta, u, report) per condition."""
    s, b = c["solver"], c["b200"]
    radius = fp32(c["radius_mm"])
    shape = icp.RaindropShape.make(radius, c["force_sphere"]).coefficients
    specs, waters = [], []
    for ii, ll in todo:
        lam = fp32(float(c["wavelength_nm"][ll]))
        water = icp.evaluate_water_optics(lam, c["temperature_c"], c["pressure_pa"])
        n = fp32(water.refractive_index)
        if not 1.0 <= n <= 2.0:
            raise ValueError("interior_index must be in [1,2]; exterior_index is 1.")
        specs.append(icp.DropSpec(shape, radius, n, b["rays"], seed=condition_seed(b["seed"], ii, ll),
                                  inclination_deg=float(c["inclination_degrees"][ii]), wavelength_nm=lam,
                                  diffraction=b["diffraction"]))
        waters.append(water)
    settings = icp.batch_settings(s["query_theta"], s["query_phi"], s["cdf_theta"], s["cdf_phi"],
                                  max_internal_hits=b["max_internal_hits"],
                                  precision=icp.ICP_FP64 if b["precision"] == "fp64" else icp.ICP_FP32,
                                  max_l1_error=s["cdf_max_l1"], max_lost_mass=s["cdf_max_lost_mass"],
                                  max_coarsening_tv=s["maximum_coarsening_tv"])
    out = icp.generate_drop_batch(ctx, specs, settings)
    return [(specs[i], waters[i], out.phi[i], out.theta[i], out.u_edges, out.reports[i]) for i in range(len(todo))]


def _arguments(argv: list[str] | None) -> argparse.Namespace:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--config", type=Path, required=True)
    ap.add_argument("--out-root", type=Path)
    ap.add_argument("--generator", type=Path, help="rainbow_generate for the patch-model stages (default: the "
                    "package's bin/rainbow_generate); ray-model records come from the batched library")
    ap.add_argument("--wavelength-range", nargs=3, metavar=("START_NM", "STOP_NM", "STEP_NM"))
    ap.add_argument("--radius-mm")
    ap.add_argument("--inclination-count", type=int)
    ap.add_argument("--allow-underresolved", action="store_true")
    ap.add_argument("--resume", action="store_true")
    ap.add_argument("--limit", type=int, help="run at most this many NEW records, without changing the planned dataset")
    mode = ap.add_mutually_exclusive_group()
    mode.add_argument("--execute", action="store_true", help="actually start the simulations; default is a dry run")
    mode.add_argument("--dry-run", action="store_true")
    args = ap.parse_args(argv)
    if args.limit is not None and args.limit <= 0:
        raise ValueError("limit must be positive")
    return args


class DatasetRun:
    """One invocation over a dataset root: the plan (conditions + library hash, signed), the scan
    of what exists (every existing record re-verified against its receipt), then the pending
    conditions in GPU batches, each record written through .part, verified and receipted."""

    def __init__(self, args: argparse.Namespace, backend=None):
        raw = read_json_object(args.config)
        overrides = {"radius_mm": args.radius_mm}
        if args.wavelength_range:
            raw["wavelengths"] = dict(zip(("start_nm", "stop_nm", "step_nm"), args.wavelength_range))
        raw.update({k: v for k, v in overrides.items() if v is not None})
        if args.inclination_count is not None:
            raw["inclinations"]["count"] = args.inclination_count
        if args.allow_underresolved:
            raw["solver"]["allow_underresolved"] = True
        self.args, self.backend = args, backend
        self.c = normalized_config(raw)
        root = Path(args.out_root or raw["output_root"])
        self.root = (root if root.is_absolute() else Path.cwd() / root).resolve()
        self.reserve = int(real_field(raw["reserve_gib"], 0, 1000000) * (1 << 30))
        nt, np_ = self.c["solver"]["cdf_theta"], self.c["solver"]["cdf_phi"]
        self.payload = 8 * ((np_ + 1) + np_ * (nt + 1) + (nt + 1))
        self.per_record = self.payload + (128 << 10)  # arrays + metadata, receipt and progress allowance
        self.ni, self.nl = len(self.c["inclination_degrees"]), len(self.c["wavelength_nm"])

    def summary(self) -> None:
        c, n = self.c, self.ni * self.nl
        s, b = c["solver"], c["b200"]
        print(f"conditions={self.ni} x {self.nl} = {n}; CDF={s['cdf_theta']}x{s['cdf_phi']}; "
              f"array_bytes_per_record={self.payload}")
        print(f"array_total_TB={self.payload * n / 1e12:.6f}; output={self.root}")
        print(f"inclination_centers=[{c['inclination_degrees'][0]}, {c['inclination_degrees'][-1]}] degrees")
        print(f"wavelengths=[{c['wavelength_nm'][0]}, {c['wavelength_nm'][-1]}] nm; inclusive exact-step endpoints")
        if s["stage"] == "incoherent":
            print(f"Batches of {b['batch_records']} records per persistent GPU launch; {b['rays']} rays per record "
                  f"({b['precision']}).")
        else:
            print(f"Stage {s['stage']}: one rainbow_generate process per record (lattice {s['grid']} x {s['grid']}, "
                  f"query {s['query_theta']} x {s['query_phi']}).")
        if s["maximum_coarsening_tv"] == 1:
            print("WARNING: maximum_coarsening_tv=1 is not an accuracy acceptance threshold.")

    def plan(self) -> tuple[dict, str]:
        """The signed plan, written on first use and required to be identical on --resume."""
        binaries = {"libicp_b200": self.backend.library_sha256()}
        if self.c["solver"]["stage"] != "incoherent":
            binaries["rainbow_generate"] = self.backend.generator_sha256()
        spec = {"version": VERSION, "conditions": self.c, "binary_sha256": binaries}
        signature = object_hash(spec)
        plan = {**spec, "signature": signature, "record_layout": "records/i{incident_index:04d}/w{wavelength_index:04d}"}
        manifest = self.root / "batch_plan.json"
        if manifest.exists():
            if not self.args.resume:
                raise FileExistsError("Dataset plan exists; use --resume with identical configuration and binaries")
            if read_json_object(manifest) != json.loads(json.dumps(plan)):
                raise ValueError("Resume rejected: configuration/binaries differ from batch_plan.json")
        else:
            if any(p.name != ".batch.lock" for p in self.root.iterdir()):
                raise ValueError("Refusing to adopt a nonempty directory without this batch plan")
            write_json(manifest, plan)
        return read_json_object(manifest), signature

    def scan(self, plan: dict, signature: str) -> tuple[list, int]:
        """(pending conditions, number of existing records verified against their receipts)."""
        pending, verified = [], 0
        for ii in range(self.ni):
            for ll in range(self.nl):
                job = f"i{ii:04d}_w{ll:04d}"
                path = self.root / "records" / f"i{ii:04d}" / f"w{ll:04d}"
                receipt = self.root / "receipts" / f"{job}.json"
                if path.with_name(path.name + ".part").exists():
                    raise ValueError(f"Incomplete .part exists: {path}.part; inspect and move it manually before retrying")
                if not path.exists():
                    if receipt.exists():
                        raise ValueError(f"Receipt exists but record missing: {path}")
                    pending.append((ii, ll, job, path, receipt))
                    continue
                if not self.args.resume or not receipt.exists():
                    raise ValueError(f"Existing record without authorized resume/receipt: {path}")
                saved = read_json_object(receipt)
                expected = {"signature": signature, "incident_index": ii, "wavelength_index": ll,
                            "record": verify_record(path, plan, ii, ll)}
                if any(saved.get(k) != v for k, v in expected.items()):
                    raise ValueError(f"Resume receipt/content mismatch: {path}")
                verified += 1
        return pending, verified

    def execute(self) -> None:
        self.root.mkdir(parents=True, exist_ok=True)
        with batch_lock(self.root):
            plan, signature = self.plan()
            pending, verified = self.scan(plan, signature)
            todo = pending if self.args.limit is None else pending[:self.args.limit]
            free = shutil.disk_usage(self.root).free
            print(f"verified_existing={verified}; pending={len(pending)}; this_run={len(todo)}; "
                  f"free_TB={free / 1e12:.3f}")
            needed = len(todo) * self.per_record + self.reserve
            if needed > free:
                raise RuntimeError(f"Insufficient free space: estimated {needed} bytes including reserve; "
                                   f"available {free}")
            total, started, done = self.ni * self.nl, time.monotonic(), 0
            lattice = self.c["solver"]["stage"] != "incoherent"
            per = 1 if lattice else self.c["b200"]["batch_records"]
            with self.backend.context(self.c["solver"]["device"]) as ctx:
                for batch in (todo[k:k + per] for k in range(0, len(todo), per)):
                    if shutil.disk_usage(self.root).free < len(batch) * self.per_record + self.reserve:
                        raise RuntimeError("Free-space reserve reached; stopping without lowering precision")
                    if lattice:
                        results = [None] * len(batch)
                    else:
                        results = self.backend.generate(ctx, self.c, [(ii, ll) for ii, ll, *_ in batch])
                    for (ii, ll, job, path, receipt), result in zip(batch, results):
                        path.parent.mkdir(parents=True, exist_ok=True)
                        if lattice:
                            self.backend.lattice_record(self.c, ii, ll, path)
                        else:
                            sp, water, phi, theta, u, rep = result
                            accept(rep, self.c)
                            write_record(path, phi, theta, u, record_metadata(self.c, ii, ll, sp, rep, water))
                        digest = verify_record(path, plan, ii, ll)
                        write_json(receipt, {"signature": signature, "incident_index": ii, "wavelength_index": ll,
                                             "record": digest})
                        done += 1
                        write_json(self.root / "progress.json",
                                   {"completed": verified + done, "total": total, "last_record": job,
                                    "elapsed_seconds_this_run": time.monotonic() - started})
                        print(f"[{verified + done}/{total}] {job}: alpha={self.c['inclination_degrees'][ii]} "
                              f"lambda={self.c['wavelength_nm'][ll]} g={digest['hg_g']:.9g} "
                              f"Aproj_mm2={digest['projected_area_mm2']:.9g}", flush=True)
            complete = verified + len(todo) == total
            write_json(self.root / "progress.json", {"completed": verified + len(todo), "total": total,
                                                     "complete": complete,
                                                     "elapsed_seconds_this_run": time.monotonic() - started})
            print("Dataset complete." if complete else
                  "Requested subset finished. Repeat with --resume to continue the same plan.")


def run(argv: list[str] | None = None, backend=None) -> int:
    args = _arguments(argv)
    job = DatasetRun(args, backend)
    job.summary()
    if not args.execute:
        print("DRY RUN: no simulations or files written. Add --execute to start.")
        return 0
    job.backend = backend or GpuBackend(args.generator)
    job.execute()
    return 0


def main() -> None:
    try:
        raise SystemExit(run())
    except KeyboardInterrupt:
        print("Interrupted. No automatic cleanup of records/.part directories.", file=sys.stderr)
        raise SystemExit(130)
    except (OSError, ValueError, RuntimeError, KeyError, TypeError, struct.error) as exc:
        print(f"generate_phase_dataset: {exc}", file=sys.stderr)
        raise SystemExit(1)


if __name__ == "__main__":
    main()
