"""Python access to the CPU oracle (oracle/icp_oracle.c) and the reference build (oracle/_ref).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py as the checker; the product (ice_crystal_phase_b200) never
imports it.

The composition below follows the reference CPU CLI
hex_phase/apps/generate_hex_phase.cpp:79-140 (preflight areas, per-node batches,
PhaseMassAccumulator, validate_composition, build_host_cdf).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libicp_oracle.so"
REF_DIR = HERE / "_ref"

_D = C.POINTER(C.c_double)
_U = C.POINTER(C.c_uint64)


def build() -> None:
    subprocess.run([str(HERE / "build_oracle.sh")], check=True, stdout=subprocess.DEVNULL)


def _lib() -> C.CDLL:
    if not LIB_PATH.exists():
        build()
    lib = C.CDLL(str(LIB_PATH))
    lib.icpo_sample_uniform.restype = C.c_double
    lib.icpo_sample_uniform.argtypes = [C.c_uint64, C.c_uint64, C.c_uint]
    lib.icpo_hex_projected_area.restype = C.c_double
    lib.icpo_hex_projected_area.argtypes = [C.c_double, C.c_double, _D]
    lib.icpo_u_edges.argtypes = [C.c_uint32, _D]
    lib.icpo_rotation_from_quaternion.argtypes = [C.c_double] * 4 + [_D]
    lib.icpo_make_frame.argtypes = [_D, _D, _D, _D]
    lib.icpo_hex_node_area.restype = C.c_double
    lib.icpo_hex_node_area.argtypes = [C.c_double, C.c_double, _D, _D]
    lib.icpo_hex_accumulate.argtypes = [_D, C.c_uint64, C.c_uint64, C.c_uint32, _D, C.c_uint32, C.c_uint32, _D, _D,
                                        C.c_uint64, C.c_uint64, C.c_uint64, _D, _D, _U, C.c_double]
    lib.icpo_hex_trace_rays.argtypes = [_D, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint32,
                                        _D, _D]
    lib.icpo_masses.argtypes = [_D, C.c_uint32, C.c_uint32, _D, _D]
    lib.icpo_measure_mass.argtypes = [_D, C.c_uint32, C.c_uint32, _D, _D]
    lib.icpo_build_cdf.argtypes = [_D, C.c_uint32, C.c_uint32, _D, C.c_uint32, C.c_uint32, C.c_double, C.c_double,
                                   C.c_double, _D, _D, _D, _D]
    lib.icpo_drop_accumulate.argtypes = [_D, _D, C.c_uint64, C.c_uint64, C.c_uint32, _D, C.c_uint32, C.c_uint32,
                                         C.c_uint64, C.c_uint64, _D, _D, _U]
    lib.icpo_drop_trace_rays.argtypes = [_D, _D, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint64,
                                         C.c_uint32, _D, _D]
    lib.icpo_drop_trace_from.argtypes = [_D, _D, _D, _D, C.c_uint32, C.c_uint32, _D, _D]
    lib.icpo_drop_intersect.argtypes = [_D, _D, _D, C.c_int, _D]
    lib.icpo_drop_frame.argtypes = [C.c_double, _D, _D, _D]
    lib.icpo_rainbow_table_sigma.argtypes = [C.c_float, _D]
    lib.icpo_rainbow_config_ok.argtypes = [C.c_uint32, C.c_uint32, _D]
    lib.icpo_rainbow_distance.restype = C.c_double
    lib.icpo_rainbow_distance.argtypes = [C.c_double] * 3
    lib.icpo_rainbow_detect.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, _D, C.c_void_p]
    lib.icpo_rainbow_filter.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, _D, C.c_void_p]
    lib.icpo_rainbow_filter_at.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, _D, C.c_void_p,
                                           C.c_uint64, C.c_void_p]
    lib.icpo_patch_optics.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.icpo_bilinear_intersect.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.icpo_patch_query.restype = C.c_uint64
    lib.icpo_patch_query.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                     C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.icpo_patch_build.restype = C.c_uint32
    lib.icpo_patch_build.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_float, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p]
    lib.icpo_atlas_node.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint32, _D, _D,
                                    _D, _D, C.c_uint64, _D, C.c_uint32, C.c_uint32, C.c_double, _D, _D]
    return lib


_LIB: C.CDLL | None = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = _lib()
    return _LIB


def _p(a: np.ndarray):
    return a.ctypes.data_as(_D if a.dtype == np.float64 else _U)


def sample_uniform(seed: int, ray: int, dim: int) -> float:
    return lib().icpo_sample_uniform(seed, ray, dim)


def u_edges(n: int) -> np.ndarray:
    e = np.empty(n + 1)
    if lib().icpo_u_edges(n, _p(e)):
        raise ValueError("u edges not representable")
    return e


def make_frame(k) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    kin = np.asarray(k, dtype=np.float64)
    ko, e0, e1 = np.empty(3), np.empty(3), np.empty(3)
    if lib().icpo_make_frame(_p(kin), _p(ko), _p(e0), _p(e1)):
        raise ValueError("invalid incident direction")
    return ko, e0, e1


def rotation_from_quaternion(q) -> np.ndarray:
    """Columns body->ensemble, returned as a 3x3 matrix M with M[:, c] = column c."""
    out = np.empty(9)
    if lib().icpo_rotation_from_quaternion(*map(float, q), _p(out)):
        raise ValueError("Quaternion must be unit length (w,x,y,z).")
    return out.reshape(3, 3).T.copy()


def hex_projected_area(R: float, L: float, k) -> float:
    kk = np.asarray(k, dtype=np.float64)
    return lib().icpo_hex_projected_area(R, L, _p(kk))


@dataclass
class Node:
    q: tuple[float, float, float, float]
    weight: float
    samples: int
    seed: int


def parse_plan(text: str) -> list[Node]:
    """Orientation CSV (hex_phase/src/orientation_plan.cpp:69-120) without the SHA digest."""
    nodes, header = [], False
    for raw in text.splitlines():
        line = raw.strip(" \t\r")
        if not line or line.startswith("#"):
            continue
        if not header:
            if line != "qw,qx,qy,qz,weight,samples,seed":
                raise ValueError("Expected CSV header qw,qx,qy,qz,weight,samples,seed.")
            header = True
            continue
        cols = line.split(",")
        if len(cols) != 7:
            raise ValueError("Expected seven CSV fields.")
        nodes.append(Node(tuple(float(c) for c in cols[:4]), float(cols[4]), int(cols[5]), int(cols[6])))
    total = math.fsum(n.weight for n in nodes)
    if not nodes or abs(total - 1) > 2e-12:
        raise ValueError("Orientation number-probability weights must sum to one (within 2e-12).")
    # Kahan sum of weights as in the reference (orientation_plan.cpp:286, 295)
    s, c = 0.0, 0.0
    for n in nodes:
        y = n.weight - c
        t = s + y
        c = (t - s) - y
        s = t
    for n in nodes:
        n.weight /= s
    return nodes


@dataclass
class HexRecord:
    masses: np.ndarray
    point_mass: float
    point_axial: float
    forward: float
    backward: float
    expected_area: float
    escaped_area: float
    unresolved_area: float
    max_balance: float
    max_iface: float
    counts: dict = field(default_factory=dict)


def hex_record(R: float, L: float, ki, n_int: float, n_ext: float, nt: int, np_: int, nodes: list[Node],
               max_hits: int = 1024, tail: float = 1e-12, batch: int = 4096,
               balance_tol: float = 1e-10) -> HexRecord:
    """Cell masses and audits of one record, in the reference CLI's order of operations."""
    L_ = lib()
    edges = u_edges(nt)
    ko, e0, e1 = make_frame(ki)
    grid_frame = np.concatenate([ko, e0, e1])
    cells = np.zeros(2 * nt * np_)
    stats = np.zeros(18)
    counts = np.zeros(13, dtype=np.uint64)
    expected_s, expected_c = 0.0, 0.0
    rots = []
    for n in nodes:
        rot = rotation_from_quaternion(n.q).T.reshape(-1).copy()  # column-major body->ensemble
        area = L_.icpo_hex_node_area(R, L, _p(rot), _p(ko))
        if not area > 0:
            raise ValueError("Invalid node geometry")
        rots.append(rot)
        y = n.weight * area - expected_c
        t = expected_s + y
        expected_c = (t - expected_s) - y
        expected_s = t
    for n, rot in zip(nodes, rots):
        node = np.array([R, L, n_ext, n_int, tail, n.weight])
        rc = L_.icpo_hex_accumulate(_p(node), n.seed, n.samples, max_hits, _p(edges), nt, np_, _p(grid_frame),
                                    _p(rot), 0, n.samples, batch, _p(cells), _p(stats), _p(counts), balance_tol)
        if rc:
            raise RuntimeError(f"oracle accumulate failed ({rc})")
    masses = np.empty(nt * np_)
    if L_.icpo_masses(_p(cells), nt, np_, _p(stats), _p(masses)):
        raise RuntimeError("Pole weight underflow.")
    names = ["samples", "snapped", "outputs", "rays"] + [f"status{i}" for i in range(8)] + ["rejected_batches"]
    return HexRecord(masses, stats[0], stats[2], stats[4], stats[6], expected_s, stats[14], stats[16], stats[10],
                     stats[11], {k: int(v) for k, v in zip(names, counts)})


def hex_trace_rays(R, L, k_body, n_int, n_ext, seed, total, max_hits, tail, first, count, max_out=64):
    node = np.array([R, L, k_body[0], k_body[1], k_body[2], n_ext, n_int, tail, 1.0])
    info = np.zeros((count, 6))
    exits = np.zeros((count, max_out, 4))
    if lib().icpo_hex_trace_rays(_p(node), seed, total, max_hits, first, count, max_out, _p(info), _p(exits)):
        raise RuntimeError("invalid trace settings")
    return info, exits


@dataclass
class Cdf:
    phi: np.ndarray
    theta: np.ndarray
    edges: np.ndarray
    report: dict


def build_cdf(mass: np.ndarray, nt: int, np_: int, ct: int | None = None, cp: int | None = None,
              max_l1: float = 1e-10, max_lost: float = 1e-12, max_tv: float = 1.0) -> Cdf:
    ct = ct or nt
    cp = cp or np_
    edges = u_edges(nt)
    m = np.ascontiguousarray(mass, dtype=np.float64)
    phi = np.zeros(cp + 1)
    theta = np.zeros(cp * (ct + 1))
    ced = np.zeros(ct + 1)
    rep = np.zeros(9)
    rc = lib().icpo_build_cdf(_p(edges), nt, np_, _p(m), ct, cp, max_l1, max_lost, max_tv, _p(phi), _p(theta),
                              _p(ced), _p(rep))
    names = ["g_source", "g_stored", "coarsening_tv", "cdf_mass", "l1_error", "lost_mass", "maximum_cell_error",
             "aggregation_relative_error", "lost_cells"]
    report = dict(zip(names, rep.tolist()))
    report["status"] = rc
    return Cdf(phi, theta.reshape(cp, ct + 1), ced, report)


# ------------------------------------------------------------------ reference (_ref)
def atlas_node(R: float, L: float, n_int: float, k, e0, e1, faces, points, weights, nt: int, np_: int,
               n_ext: float = 1.0, tail: float = 1e-12, max_hits: int = 2048, balance_tol: float = 1e-10):
    """One atlas node from its quadrature rays (atlas::trace_cpu, hex_atlas/src/atlas.cpp:140-153):
    (cell masses [nt][np] in mm^2, stats: escaped_mm2, unresolved_mm2, rays, outputs, max balance,
    max interface balance, first rejected ray or -1, its status)."""
    rays = np.ascontiguousarray(np.column_stack([np.asarray(faces, float), np.asarray(points, float),
                                                 np.asarray(weights, float)]))
    edges = u_edges(nt)
    cells = np.zeros(nt * np_)
    stats = np.zeros(8)
    k3, a3, b3 = (np.ascontiguousarray(v, dtype=np.float64) for v in (k, e0, e1))
    st = lib().icpo_atlas_node(R, L, n_ext, n_int, tail, max_hits, _p(k3), _p(a3), _p(b3), _p(rays), len(rays),
                               _p(edges), nt, np_, balance_tol, _p(cells), _p(stats))
    if st:
        raise RuntimeError(f"icpo_atlas_node failed ({st})")
    return cells.reshape(nt, np_), stats


def ref_available() -> bool:
    return (REF_DIR / "ref_hex_harness").exists()


def ref_masses(R, L, ki, n_int, n_ext, nt, np_, plan_csv: Path, max_hits=1024, tail=1e-12, batch=4096,
               workdir: Path | None = None) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    out = Path(workdir or "/tmp") / f"ref_masses_{os.getpid()}.bin"
    args = [str(REF_DIR / "ref_hex_harness"), "masses", repr(R), repr(L), *map(repr, map(float, ki)), repr(n_int),
            repr(n_ext), str(nt), str(np_), str(max_hits), repr(tail), str(plan_csv), str(batch), str(out)]
    subprocess.run(args, check=True)
    raw = out.read_bytes()
    out.unlink()
    n = nt * np_
    masses = np.frombuffer(raw[:8 * n], dtype="<f8").copy()
    d = np.frombuffer(raw[8 * n:8 * n + 72], dtype="<f8").copy()
    u = np.frombuffer(raw[8 * n + 72:], dtype="<u8").copy()
    return masses, d, u


# ------------------------------------------------------------------ water drops
@dataclass
class DropGeometry:
    """Drop in units of its equal-volume radius and the sampling disk that covers it."""
    coefficients: np.ndarray
    radius_mm: float
    r_center: float
    r_out: float
    r_in: float
    sphere: bool
    disk: float
    back: float

    def vector(self, n_int: float, n_ext: float = 1.0, tail: float = 1e-12, scale: float = 1.0) -> np.ndarray:
        return np.array([*self.coefficients, self.r_center, self.r_out, self.r_in, float(self.sphere), self.disk,
                         self.back, n_ext, n_int, tail, scale, self.radius_mm])

    @property
    def disk_area_mm2(self) -> float:
        return math.pi * self.disk * self.disk * self.radius_mm * self.radius_mm


def drop_geometry(coefficients, radius_mm: float) -> DropGeometry:
    """Bounding radii from |T_n| <= 1; rays are sampled on the disk of the exact sphere radius
    (spheres) or of the conservative outer radius, 2 r_out + 1 before the centre."""
    c = np.zeros(8)
    given = np.asarray(coefficients, dtype=np.float64).reshape(-1)
    if given.size > 8:
        raise ValueError("At most eight shape coefficients.")
    c[:given.size] = given
    sphere = bool(np.all(c[1:] == 0))
    r_center = 1 + c[0]
    s = 0.0
    for x in c[1:]:
        s += abs(float(x))
    r_out = (1 + c[0] + s) * (1 + 1e-6) + 1e-6
    r_in = 1 + c[0] - s
    disk = r_center if sphere else r_out
    return DropGeometry(c, radius_mm, r_center, r_out, r_in, sphere, disk, 2 * r_out + 1)


def drop_frame(inclination_deg: float) -> np.ndarray:
    """k, e0, e1 of an inclination as a (3, 3) array of rows."""
    k, e0, e1 = np.empty(3), np.empty(3), np.empty(3)
    if lib().icpo_drop_frame(inclination_deg, _p(k), _p(e0), _p(e1)):
        raise ValueError("invalid inclination")
    return np.stack([k, e0, e1])


@dataclass
class DropRecord:
    masses: np.ndarray         # cell masses with the pole caps spread over the end rows (mm^2)
    forward: float
    backward: float
    escaped_area: float
    unresolved_area: float
    incident_area: float       # hits x disk area / rays
    point_axial: float
    max_balance: float
    max_iface: float
    counts: dict = field(default_factory=dict)
    cells: np.ndarray | None = None  # cell masses before the pole caps are spread (mm^2)


def drop_record(geo: DropGeometry, frame: np.ndarray, n_int: float, nt: int, np_: int, rays: int, seed: int,
                max_hits: int = 1024, tail: float = 1e-12, n_ext: float = 1.0, first: int = 0,
                count: int | None = None) -> DropRecord:
    count = rays - first if count is None else count
    scale = geo.disk_area_mm2 / rays
    drop = geo.vector(n_int, n_ext, tail, scale)
    f9 = np.ascontiguousarray(frame, dtype=np.float64).reshape(-1)
    edges = u_edges(nt)
    cells = np.zeros(2 * nt * np_)
    stats = np.zeros(14)
    counts = np.zeros(14, dtype=np.uint64)
    rc = lib().icpo_drop_accumulate(_p(drop), _p(f9), seed, rays, max_hits, _p(edges), nt, np_, first, count,
                                    _p(cells), _p(stats), _p(counts))
    if rc:
        raise RuntimeError(f"oracle drop accumulate failed ({rc})")
    hist = np.zeros(18)
    hist[[0, 2, 4, 6]] = stats[[0, 2, 4, 6]]
    masses = np.empty(nt * np_)
    if lib().icpo_masses(_p(cells), nt, np_, _p(hist), _p(masses)):
        raise RuntimeError("Pole weight underflow.")
    names = ["samples", "snapped", "outputs", "rays"] + [f"status{i}" for i in range(8)] + ["missed", "encounters"]
    cnt = {k: int(v) for k, v in zip(names, counts)}
    hits = cnt["rays"] - cnt["missed"]
    return DropRecord(masses, stats[4], stats[6], scale * stats[8], scale * stats[10], scale * hits, stats[2],
                      stats[12], stats[13], cnt, cells[0::2].copy())


def drop_record_sharded(geo: DropGeometry, frame: np.ndarray, n_int: float, nt: int, np_: int, rays: int, seed: int,
                        max_hits: int = 1024, tail: float = 1e-12, first: int = 0, count: int | None = None,
                        workers: int | None = None) -> DropRecord:
    """drop_record over rays [first, first + count) of a `rays`-ray record, cut into disjoint
    ray-id slices traced on threads (the C oracle keeps no global state and ctypes releases the
    GIL during the call).  The counter RNG makes every ray independent of the cut, so the merged
    masses equal the single-call record's up to the order of the FP64 cell sums; counts are
    exact."""
    count = rays - first if count is None else count
    workers = max(1, min(workers or os.cpu_count() or 1, max(1, count // 10000)))
    bounds = [first + count * k // workers for k in range(workers + 1)]
    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(max_workers=workers) as pool:
        parts = list(pool.map(lambda k: drop_record(geo, frame, n_int, nt, np_, rays, seed, max_hits, tail,
                                                    first=bounds[k], count=bounds[k + 1] - bounds[k]),
                              range(workers)))
    out = parts[0]
    for p in parts[1:]:
        out.masses = out.masses + p.masses
        out.cells = out.cells + p.cells
        out.forward += p.forward
        out.backward += p.backward
        out.escaped_area += p.escaped_area
        out.unresolved_area += p.unresolved_area
        out.incident_area += p.incident_area
        out.point_axial += p.point_axial
        out.max_balance = max(out.max_balance, p.max_balance)
        out.max_iface = max(out.max_iface, p.max_iface)
        out.counts = {k: out.counts[k] + p.counts[k] for k in out.counts}
    return out


def drop_trace_rays(geo: DropGeometry, frame, n_int, seed, total, first, count, max_hits=1024, tail=1e-12,
                    n_ext=1.0, max_out=64):
    """Per-ray info (status, outputs, escaped, unresolved, hits, max_iface, missed, tir) and
    exits (direction, power, interaction index)."""
    drop = geo.vector(n_int, n_ext, tail)
    f9 = np.ascontiguousarray(frame, dtype=np.float64).reshape(-1)
    info = np.zeros((count, 8))
    exits = np.zeros((count, max_out, 5))
    if lib().icpo_drop_trace_rays(_p(drop), _p(f9), seed, total, max_hits, first, count, max_out, _p(info),
                                  _p(exits)):
        raise RuntimeError("invalid drop settings")
    return info, exits


def drop_trace_from(geo: DropGeometry, origin, k, e0, n_int, max_hits=3, n_ext=1.0, tail=0.0, max_out=16):
    drop = geo.vector(n_int, n_ext, tail)
    o, kk, ee = (np.ascontiguousarray(v, dtype=np.float64) for v in (origin, k, e0))
    info = np.zeros(8)
    exits = np.zeros((max_out, 5))
    if lib().icpo_drop_trace_from(_p(drop), _p(o), _p(kk), _p(ee), max_hits, max_out, _p(info), _p(exits)):
        raise RuntimeError("invalid drop settings")
    return info, exits[: min(int(info[1]), max_out)]


def drop_intersect(geo: DropGeometry, origin, d, inside: bool) -> np.ndarray:
    out = np.zeros(8)
    o, dd = (np.ascontiguousarray(v, dtype=np.float64) for v in (origin, d))
    if lib().icpo_drop_intersect(_p(geo.vector(1.33)), _p(o), _p(dd), int(inside), _p(out)):
        raise RuntimeError("invalid drop query")
    return out


def ref_drop_available() -> bool:
    return (REF_DIR / "ref_drop_harness").exists()


def ref_drop_lines(mode: str, lines: list[str]) -> list[list[float]]:
    """Runs the reference drop harness in a line mode (water, shape, area, frame)."""
    r = subprocess.run([str(REF_DIR / "ref_drop_harness"), mode], input="\n".join(lines) + "\n",
                       capture_output=True, text=True, check=True)
    return [[float(x) for x in line.split()] for line in r.stdout.splitlines()]


def ref_drop_families(radius_mm: float, sphere: bool, n_int: float, k, grid: int,
                      workdir: Path | None = None) -> np.ndarray:
    """The reference four-family tracer over its vertex lattice: (grid^2, 41) float64 rows."""
    out = Path(workdir or "/tmp") / f"ref_families_{os.getpid()}.bin"
    args = [str(REF_DIR / "ref_drop_harness"), "families", repr(float(radius_mm)), str(int(sphere)),
            repr(float(n_int)), *map(repr, map(float, k)), str(grid), str(out)]
    subprocess.run(args, check=True)
    a = np.fromfile(out, dtype="<f8").reshape(-1, 41)
    out.unlink()
    return a


# ------------------------------------------------------- Table-II rainbow diffraction
# rainbow::FocalOpticalResult (include/rainbow/wave_optics_data.hpp:27-40) and
# rainbow::DiffractionResult (:66-78) as numpy records.
FOCAL_DTYPE = np.dtype([("field", "<f8", 4), ("intensity_s", "<f8"), ("intensity_p", "<f8"),
                        ("family_incoherent", "<f8", 4), ("family_hits", "<u4", 4), ("corrected_hits", "<u4"),
                        ("extra_quarter_turn_hits", "<u4"), ("flags", "<u4"), ("first_problem_patch_id", "<u4"),
                        ("field_second", "<f8", 4)])
RESULT_DTYPE = np.dtype([("intensity_s", "<f8"), ("intensity_p", "<f8"), ("sigma_rad", "<f8"), ("blend", "<f8"),
                         ("flags", "<u4"), ("transition_kind", "<u4")])
assert FOCAL_DTYPE.itemsize == 144 and RESULT_DTYPE.itemsize == 40


def _cfg(config) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(config, dtype=np.float64).reshape(4))


def rainbow_table_sigma(radius: float) -> float | None:
    """Table-II primary width (degrees) of a float32 radius in mm, None outside the table."""
    out = np.zeros(1)
    return float(out[0]) if lib().icpo_rainbow_table_sigma(float(radius), _p(out)) else None


def rainbow_config_ok(nt: int, np_: int, config) -> bool:
    return bool(lib().icpo_rainbow_config_ok(nt, np_, _p(_cfg(config))))


def rainbow_distance(a: float, b: float, phi: float) -> float:
    return float(lib().icpo_rainbow_distance(a, b, phi))


def rainbow_detect(focal: np.ndarray, nt: int, np_: int, config) -> np.ndarray:
    """Transition labels (uint32 [nt*np]) of a focal grid (FOCAL_DTYPE [nt*np]); config =
    (primary sigma rad, support sigma, transition contrast, inner blend sigma)."""
    f = np.ascontiguousarray(focal, dtype=FOCAL_DTYPE).reshape(-1)
    assert f.size == nt * np_
    edges = np.zeros(nt * np_, dtype=np.uint32)
    lib().icpo_rainbow_detect(f.ctypes.data, nt, np_, _p(_cfg(config)), edges.ctypes.data)
    return edges


def rainbow_filter(focal: np.ndarray, edges: np.ndarray, nt: int, np_: int, config) -> np.ndarray:
    """Diffraction results (RESULT_DTYPE [nt*np]) of a focal grid under the given labels."""
    f = np.ascontiguousarray(focal, dtype=FOCAL_DTYPE).reshape(-1)
    e = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1)
    assert f.size == e.size == nt * np_
    out = np.zeros(nt * np_, dtype=RESULT_DTYPE)
    lib().icpo_rainbow_filter(f.ctypes.data, e.ctypes.data, nt, np_, _p(_cfg(config)), out.ctypes.data)
    return out


def rainbow_filter_at(focal: np.ndarray, edges: np.ndarray, nt: int, np_: int, config, index) -> np.ndarray:
    """The diffraction results at the given direction indices only."""
    f = np.ascontiguousarray(focal, dtype=FOCAL_DTYPE).reshape(-1)
    e = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1)
    idx = np.ascontiguousarray(index, dtype=np.uint64).reshape(-1)
    assert f.size == e.size == nt * np_ and (idx < nt * np_).all()
    out = np.zeros(idx.size, dtype=RESULT_DTYPE)
    lib().icpo_rainbow_filter_at(f.ctypes.data, e.ctypes.data, nt, np_, _p(_cfg(config)), idx.ctypes.data, idx.size,
                                 out.ctypes.data)
    return out


def ref_rainbow_available() -> bool:
    return (REF_DIR / "ref_rainbow_harness").exists()


def ref_rainbow_table(radii) -> list[tuple[bool, float]]:
    """The reference's table_sigma_degrees on float32 radii (given as decimal strings or floats)."""
    text = "\n".join(repr(float(np.float32(r))) for r in radii) + "\n"
    r = subprocess.run([str(REF_DIR / "ref_rainbow_harness"), "table"], input=text, capture_output=True, text=True,
                       check=True)
    return [(line.split()[0] == "1", float.fromhex(line.split()[1])) for line in r.stdout.splitlines()]


def ref_rainbow_grid(focal: np.ndarray, nt: int, np_: int, config, edges: np.ndarray | None = None,
                     workdir: Path | None = None) -> tuple[np.ndarray, np.ndarray]:
    """The reference's detect (unless edges are given) and filter over a whole focal grid."""
    f = np.ascontiguousarray(focal, dtype=FOCAL_DTYPE).reshape(-1)
    base = Path(workdir or "/tmp") / f"ref_rainbow_{os.getpid()}"
    src, dst = base.with_suffix(".in"), base.with_suffix(".out")
    with open(src, "wb") as fh:
        fh.write(np.array([nt, np_], dtype="<u4").tobytes() + _cfg(config).tobytes())
        fh.write(np.array([0 if edges is None else 1, 0], dtype="<u4").tobytes() + f.tobytes())
        if edges is not None:
            fh.write(np.ascontiguousarray(edges, dtype="<u4").tobytes())
    subprocess.run([str(REF_DIR / "ref_rainbow_harness"), "grid", str(src), str(dst)], check=True)
    raw = dst.read_bytes()
    src.unlink()
    dst.unlink()
    n = nt * np_
    return (np.frombuffer(raw[: 4 * n], dtype="<u4").copy(),
            np.frombuffer(raw[4 * n:], dtype=RESULT_DTYPE).copy())


# ----------------------------------------------------------------------- patch optics
class _Vec3f(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class _OpticsInput(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("patches", C.c_void_p), ("directions", C.c_void_p),
                ("offsets", C.c_void_p), ("summaries", C.c_void_p), ("hits", C.c_void_p), ("second", C.c_void_p),
                ("hit_storage", C.c_uint64), ("vertex_count", C.c_uint32), ("patch_count", C.c_uint32),
                ("direction_count", C.c_uint32), ("second_count", C.c_uint32), ("incident", _Vec3f),
                ("incident_basis", _Vec3f), ("polarization", C.c_uint32), ("reserved", C.c_uint32)]


class _FocalConfig(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("half_extent", C.c_float), ("reserved", C.c_uint32),
                ("offsets", C.c_uint32 * 4)]


OPTICAL_DTYPE = np.dtype([("path_field", "<f8", 4), ("incoherent_s", "<f8"), ("incoherent_p", "<f8"),
                          ("path_s", "<f8"), ("path_p", "<f8")] +
                         [(k, "<u4") for k in ("hit_count", "evaluated_hits", "rejected_hits", "refinement_hits",
                                               "boundary_hits", "singular_hits", "flags", "query_flags",
                                               "first_problem_patch_id", "folded_hits")] +
                         [("path_field_second", "<f8", 4)])


def patch_optics(case) -> tuple[np.ndarray, np.ndarray | None]:
    """Per-direction optics of an optics input (tests/optics_cases.OpticsInput): the
    PatchOpticalResult records, and the FocalOpticalResult records when it has a focal layout."""
    keep = []

    def ptr(a):
        if a is None:
            return None
        a = np.ascontiguousarray(a)
        keep.append(a)
        return a.ctypes.data

    n = case.count
    inp = _OpticsInput(ptr(case.vertices), ptr(case.patches), ptr(np.asarray(case.directions, dtype=np.float32)),
                       ptr(case.offsets.astype(np.uint64)), ptr(case.summaries), ptr(case.hits),
                       ptr(None if case.second is None else np.asarray(case.second, dtype=np.float32)),
                       len(case.hits), len(case.vertices), len(case.patches), n, case.second_len(),
                       _Vec3f(*map(float, case.incident)), _Vec3f(*map(float, case.basis)), case.polarization, 0)
    out = np.zeros(n, dtype=OPTICAL_DTYPE)
    focal = np.zeros(n, dtype=FOCAL_DTYPE) if case.focal else None
    cfg = None
    if case.focal:
        w, h, e, o = case.focal
        cfg = _FocalConfig(w, h, e, 0, (C.c_uint32 * 4)(*o))
    lib().icpo_patch_optics(C.addressof(inp), C.addressof(cfg) if cfg is not None else None, out.ctypes.data,
                            focal.ctypes.data if focal is not None else None)
    return out, focal


def ref_optics_available() -> bool:
    return (REF_DIR / "ref_optics_harness").exists()


def ref_patch_optics(blob: bytes, count: int, with_focal: bool,
                     workdir: Path | None = None) -> tuple[np.ndarray, np.ndarray | None]:
    """The reference's evaluator over a serialized optics input (tests/optics_cases.serialize)."""
    base = Path(workdir or "/tmp") / f"ref_optics_{os.getpid()}"
    src, dst = base.with_suffix(".in"), base.with_suffix(".out")
    src.write_bytes(blob)
    subprocess.run([str(REF_DIR / "ref_optics_harness"), str(src), str(dst)], check=True)
    raw = dst.read_bytes()
    src.unlink()
    dst.unlink()
    out = np.frombuffer(raw[: 136 * count], dtype=OPTICAL_DTYPE).copy()
    focal = np.frombuffer(raw[136 * count:], dtype=FOCAL_DTYPE).copy() if with_focal else None
    return out, focal


PATCH_DTYPE = np.dtype([("vertex_indices", "<u4", 4), ("patch_id", "<u4"), ("status", "<u4"),
                        ("signed_solid_angle_sr", "<f4"), ("incident_area_drop2", "<f4")])
AABB_DTYPE = np.dtype([(k, "<f4") for k in ("min_x", "min_y", "min_z", "max_x", "max_y", "max_z")])


def patch_build(vertices: np.ndarray, width: int, height: int, half_extent: float):
    """(statuses [cells], patches with geometry in patch_id order, their boxes, status histogram)."""
    cells = 4 * (width - 1) * (height - 1)
    v = np.ascontiguousarray(vertices)
    st = np.zeros(cells, dtype=np.uint32)
    pa = np.zeros(cells, dtype=PATCH_DTYPE)
    bx = np.zeros(cells, dtype=AABB_DTYPE)
    hist = np.zeros(8, dtype=np.uint32)
    n = lib().icpo_patch_build(v.ctypes.data, width, height, float(half_extent), st.ctypes.data, pa.ctypes.data,
                               bx.ctypes.data, hist.ctypes.data)
    if n == 0xFFFFFFFF:
        raise ValueError("invalid patch layout")
    return st, pa[:n].copy(), bx[:n].copy(), hist


def ref_patch_build(blob: bytes, cells: int, workdir: Path | None = None):
    base = Path(workdir or "/tmp") / f"ref_patch_{os.getpid()}"
    src, dst = base.with_suffix(".in"), base.with_suffix(".out")
    src.write_bytes(blob)
    subprocess.run([str(REF_DIR / "ref_patch_harness"), str(src), str(dst)], check=True)
    raw = dst.read_bytes()
    src.unlink()
    dst.unlink()
    st = np.frombuffer(raw[:4 * cells], "<u4").copy()
    n = int(np.frombuffer(raw[4 * cells:4 * cells + 4], "<u4")[0])
    hist = np.frombuffer(raw[4 * cells + 4:4 * cells + 36], "<u4").copy()
    off = 4 * cells + 36
    pa = np.frombuffer(raw[off:off + 32 * n], PATCH_DTYPE).copy()
    bx = np.frombuffer(raw[off + 32 * n:off + 56 * n], AABB_DTYPE).copy()
    return st, pa, bx, hist


BILINEAR_HITS_DTYPE = np.dtype([("hits", [("u", "<f4"), ("v", "<f4"), ("t", "<f4"), ("residual", "<f4"),
                                          ("flags", "<u4")], 2), ("count", "<u4"), ("flags", "<u4")])
assert BILINEAR_HITS_DTYPE.itemsize == 48


def bilinear_intersect(corners: np.ndarray, directions: np.ndarray) -> np.ndarray:
    """Ray / bilinear patch hits for rows of (corners [n, 4, 3], directions [n, 3]), float32."""
    c = np.ascontiguousarray(corners, dtype=np.float32).reshape(-1, 12)
    d = np.ascontiguousarray(directions, dtype=np.float32).reshape(-1, 3)
    out = np.zeros(len(c), dtype=BILINEAR_HITS_DTYPE)
    for i in range(len(c)):
        lib().icpo_bilinear_intersect(c[i].ctypes.data, d[i].ctypes.data, out[i:i + 1].ctypes.data)
    return out


def ref_bilinear_intersect(corners: np.ndarray, directions: np.ndarray, workdir: Path | None = None) -> np.ndarray:
    c = np.ascontiguousarray(corners, dtype=np.float32).reshape(-1, 12)
    d = np.ascontiguousarray(directions, dtype=np.float32).reshape(-1, 3)
    base = Path(workdir or "/tmp") / f"ref_isect_{os.getpid()}"
    src, dst = base.with_suffix(".in"), base.with_suffix(".out")
    src.write_bytes(np.array([len(c)], "<u4").tobytes() + np.hstack([c, d]).astype("<f4").tobytes())
    subprocess.run([str(REF_DIR / "ref_query_harness"), "intersect", str(src), str(dst)], check=True)
    out = np.frombuffer(dst.read_bytes(), dtype=BILINEAR_HITS_DTYPE).copy()
    src.unlink()
    dst.unlink()
    return out


SUMMARY_DTYPE = np.dtype([(k, "<u4") for k in ("candidate_count", "hit_count", "regular_hits", "refinement_hits",
                                               "boundary_hits", "flags", "first_problem_patch_id", "reserved")])
HIT_DTYPE = np.dtype([("compact_index", "<u4"), ("patch_id", "<u4"), ("root_index", "<u4"), ("flags", "<u4"),
                      ("u", "<f4"), ("v", "<f4"), ("t", "<f4"), ("residual", "<f4")])


def patch_query(vertices, patches, aabbs, directions):
    """All-hit query by brute force over every patch: (offsets [n + 1], summaries [n], hits)."""
    v = np.ascontiguousarray(vertices)
    p = np.ascontiguousarray(patches, dtype=PATCH_DTYPE)
    b = np.ascontiguousarray(aabbs, dtype=AABB_DTYPE)
    d = np.ascontiguousarray(directions, dtype=np.float32).reshape(-1, 3)
    n = len(d)
    offsets = np.zeros(n + 1, dtype=np.uint64)
    summaries = np.zeros(n, dtype=SUMMARY_DTYPE)
    total = lib().icpo_patch_query(v.ctypes.data, len(v), p.ctypes.data, b.ctypes.data, len(p), d.ctypes.data, n,
                                   offsets.ctypes.data, summaries.ctypes.data, None)
    hits = np.zeros(max(1, total), dtype=HIT_DTYPE)
    lib().icpo_patch_query(v.ctypes.data, len(v), p.ctypes.data, b.ctypes.data, len(p), d.ctypes.data, n,
                           offsets.ctypes.data, summaries.ctypes.data, hits.ctypes.data)
    return offsets, summaries, hits[:total]


def ref_query_directions(nt: int, np_: int, axis, e0, workdir: Path | None = None) -> np.ndarray:
    out = Path(workdir or "/tmp") / f"ref_qdirs_{os.getpid()}.bin"
    subprocess.run([str(REF_DIR / "ref_query_harness"), "directions", str(nt), str(np_),
                    *[repr(float(x)) for x in axis], *[repr(float(x)) for x in e0], str(out)], check=True)
    d = np.frombuffer(out.read_bytes(), dtype="<f4").reshape(-1, 3).copy()
    out.unlink()
    return d
