"""Synthetic inputs of the drop's patch optics (the path / focal stages' per-direction sums).

A small outgoing-ray lattice of the four path families (R, TT, TRT, TRRT) over the emitting
plane, its patches and a query of seeded directions with sorted hit lists, in the reference's
record layouts (OutgoingVertex, OutgoingPatch, PatchQueryHit, PatchQuerySummary).  Each case
mixes regular hits with every kind of rejected or pending input the reference's evaluator
distinguishes: unsorted and duplicate hits, out-of-range patch indices, invalid vertices and
phases, non-regular patches, boundary / singular hits, query errors, degenerate and non-unit
query directions, forward scattering.  `CASES` lists the fixture cases
(tests/golden/optics_reference.npz holds the reference's outputs and the SHA-256 of each
input); `serialize` writes the byte layout read by oracle/ref_optics_harness.cpp.
"""
from __future__ import annotations

import hashlib
import math
import struct
from dataclasses import dataclass

import numpy as np

VERTEX_DTYPE = np.dtype([("position", "<f4", 3), ("direction", "<f4", 3), ("basis_x", "<f4", 3),
                         ("field", "<f4", 4), ("turns", "<i4"), ("fraction", "<f4"), ("status", "<u4"),
                         ("diagnostics", "<u4")])
PATCH_DTYPE = np.dtype([("vertex_indices", "<u4", 4), ("patch_id", "<u4"), ("status", "<u4"),
                        ("signed_solid_angle_sr", "<f4"), ("incident_area_drop2", "<f4")])
HIT_DTYPE = np.dtype([("compact_index", "<u4"), ("patch_id", "<u4"), ("root_index", "<u4"), ("flags", "<u4"),
                      ("u", "<f4"), ("v", "<f4"), ("t", "<f4"), ("residual", "<f4")])
SUMMARY_DTYPE = np.dtype([(k, "<u4") for k in ("candidate_count", "hit_count", "regular_hits", "refinement_hits",
                                               "boundary_hits", "flags", "first_problem_patch_id", "reserved")])
OPTICAL_DTYPE = np.dtype([("path_field", "<f8", 4), ("incoherent_s", "<f8"), ("incoherent_p", "<f8"),
                          ("path_s", "<f8"), ("path_p", "<f8")] +
                         [(k, "<u4") for k in ("hit_count", "evaluated_hits", "rejected_hits", "refinement_hits",
                                               "boundary_hits", "singular_hits", "flags", "query_flags",
                                               "first_problem_patch_id", "folded_hits")] +
                         [("path_field_second", "<f8", 4)])
AABB_DTYPE = np.dtype([(k, "<f4") for k in ("min_x", "min_y", "min_z", "max_x", "max_y", "max_z")])
assert (VERTEX_DTYPE.itemsize, PATCH_DTYPE.itemsize, HIT_DTYPE.itemsize, SUMMARY_DTYPE.itemsize,
        OPTICAL_DTYPE.itemsize) == (68, 32, 32, 32, 136)


@dataclass
class OpticsInput:
    vertices: np.ndarray
    patches: np.ndarray
    directions: np.ndarray      # float32 (n, 3)
    offsets: np.ndarray         # uint64 (n + 1)
    summaries: np.ndarray
    hits: np.ndarray
    second: np.ndarray | None   # float32 (vertex_count, 4) or None
    incident: np.ndarray        # float32 (3,)
    basis: np.ndarray           # float32 (3,)
    polarization: int
    focal: tuple | None         # (width, height, half_extent, offsets[4]) or None
    second_count: int | None = None  # overrides len(second) (inconsistent-input cases)

    @property
    def count(self) -> int:
        return len(self.directions)

    def second_len(self) -> int:
        if self.second_count is not None:
            return self.second_count
        return 0 if self.second is None else len(self.second)


def _f32_unit(v: np.ndarray) -> np.ndarray:
    v = np.asarray(v, dtype=np.float32)
    return (v / np.sqrt((v * v).sum(axis=-1, keepdims=True))).astype(np.float32)


def lattice_case(seed: int, width: int = 7, height: int = 7, directions: int = 150, dual: bool = True,
                 focal: bool = True, faults: bool = True, quarter_turns=(0, 1, 2, 3)) -> OpticsInput:
    rng = np.random.default_rng(seed)
    half = 1.01
    k = _f32_unit([math.cos(math.radians(20)), -math.sin(math.radians(20)), 0.0])
    e0 = np.array([0.0, 0.0, 1.0], dtype=np.float32)
    e1 = _f32_unit(np.cross(k.astype(np.float64), e0.astype(np.float64)))
    n = width * height
    cells = (width - 1) * (height - 1)
    verts = np.zeros(4 * n, dtype=VERTEX_DTYPE)
    base = [0.05, 2.9, 2.4, 2.2]  # scattering angle of each family at the lattice centre
    for f in range(4):
        iy, ix = np.divmod(np.arange(n), width)
        U = (2 * ix / (width - 1) - 1) * half
        V = (2 * iy / (height - 1) - 1) * half
        theta = base[f] + (0.15 if f != 2 else -0.2) * (U * U + V * V) + 0.01 * rng.standard_normal(n)
        phi = np.arctan2(V, U) + 0.3 * f
        d = (np.cos(theta)[:, None] * k + np.sin(theta)[:, None] *
             (np.cos(phi)[:, None] * e0 + np.sin(phi)[:, None] * e1))
        d = _f32_unit(d)
        axis = np.where(np.abs(d[:, 2:3]) < 0.9, np.array([0, 0, 1.0]), np.array([1.0, 0, 0]))
        bx = _f32_unit(axis - d * (d * axis).sum(axis=1, keepdims=True))
        sl = slice(f * n, (f + 1) * n)
        verts["position"][sl] = np.column_stack([U, V, np.full(n, 1.0)]).astype(np.float32)
        verts["direction"][sl] = d
        verts["basis_x"][sl] = bx
        verts["field"][sl] = rng.standard_normal((n, 4)).astype(np.float32)
        verts["turns"][sl] = (1000 + 40 * f + np.round(30 * (U * U + V * V))).astype(np.int32)
        fr = rng.random(n).astype(np.float32)
        fr[rng.random(n) < 0.1] = rng.choice(np.array([0.0, 0.25, 0.5, 0.75], dtype=np.float32), 1)[0]
        verts["fraction"][sl] = fr
        verts["status"][sl] = 1
    patches = np.zeros(4 * cells, dtype=PATCH_DTYPE)
    for pid in range(4 * cells):
        f, cell = divmod(pid, cells)
        iy, ix = divmod(cell, width - 1)
        first = f * n + iy * width + ix
        patches["vertex_indices"][pid] = (first, first + 1, first + width, first + width + 1)
        patches["patch_id"][pid] = pid
        patches["status"][pid] = rng.choice([1, 2])
        patches["signed_solid_angle_sr"][pid] = (1 if patches["status"][pid] == 1 else -1) * rng.uniform(1e-3, 5e-2)
        patches["incident_area_drop2"][pid] = (2 * half / (width - 1)) * (2 * half / (height - 1))
    if faults:
        m = len(patches)
        patches["status"][rng.choice(m, 3, replace=False)] = 3  # needs refinement
        patches["status"][rng.choice(m, 2, replace=False)] = 4  # missing corners
        patches["signed_solid_angle_sr"][rng.choice(m, 1)] = 0.0
        p = rng.choice(m, 2, replace=False)
        patches["vertex_indices"][p[0], 1] += 1               # not the lattice's corners (focal geometry)
        patches["vertex_indices"][p[1], 2] = 4 * n + 7       # out of range
        vb = rng.choice(4 * n, 4, replace=False)
        verts["status"][vb[0]] = 2                           # a miss
        verts["fraction"][vb[1]] = 1.0                       # invalid phase
        verts["basis_x"][vb[2]] = verts["direction"][vb[2]]  # degenerate frame
        verts["field"][vb[3], 1] = np.inf
    # query directions: around the families' cones, plus forward, backward, non-unit
    dirs = []
    for _ in range(directions):
        f = rng.integers(0, 4)
        th = base[f] + rng.uniform(-0.2, 0.3)
        ph = rng.uniform(-math.pi, math.pi)
        dirs.append(math.cos(th) * k + math.sin(th) * (math.cos(ph) * e0 + math.sin(ph) * e1))
    dirs = _f32_unit(np.array(dirs))
    if faults:
        dirs[0] = k
        dirs[1] = -k
        dirs[2] = dirs[2] * np.float32(1.1)
    hits, offsets, sums = [], [0], []
    for i in range(len(dirs)):
        count = int(rng.poisson(2.5))
        chosen = sorted(rng.choice(len(patches), count, replace=False)) if count else []
        rows = []
        for c in chosen:
            for root in range(1 if rng.random() < 0.8 else 2):
                fl = 0
                r = rng.random()
                if faults and r < 0.04:
                    fl = 1
                elif faults and r < 0.07:
                    fl = 2
                elif r < 0.12:
                    fl = 4
                u, v = rng.random(2).astype(np.float32)
                if rng.random() < 0.08:
                    u, v = np.float32(rng.integers(0, 2)), np.float32(rng.integers(0, 2))
                rows.append((c, patches["patch_id"][c], root, fl, u, v, rng.uniform(0.5, 3.0), rng.uniform(0, 1e-6)))
        rows.sort(key=lambda h: (h[1], h[0], h[2]))
        if faults and i % 37 == 5 and len(rows) >= 2:
            rows[0], rows[1] = rows[1], rows[0]              # broken ordering
        if faults and i % 41 == 7 and rows:
            rows.append(rows[-1])                            # duplicate report
        if faults and i % 43 == 9 and rows:
            rows[-1] = (len(patches) + 3,) + rows[-1][1:]    # compact index out of range
        slack = int(rng.integers(0, 2))
        s = np.zeros(1, dtype=SUMMARY_DTYPE)[0]
        s["candidate_count"] = len(rows) + slack
        s["hit_count"] = len(rows)
        s["first_problem_patch_id"] = 0xFFFFFFFF
        st = [patches["status"][h[0]] if h[0] < len(patches) else 0 for h in rows]
        s["regular_hits"] = sum(1 for x in st if x in (1, 2))
        s["refinement_hits"] = sum(1 for x in st if x == 3)
        s["boundary_hits"] = sum(1 for h in rows if h[3] & 1)
        fl = (8 if s["refinement_hits"] else 0) | (16 if s["boundary_hits"] else 0)
        fl |= 128 if any(h[3] & 2 for h in rows) else 0
        if faults and i % 29 == 3:
            fl |= 1                                          # unresolved query
            s["first_problem_patch_id"] = rows[0][1] if rows else 5
        s["flags"] = fl
        sums.append(s)
        hits.extend(rows + [(0, 0, 0, 0, 0.5, 0.5, 1.0, 0.0)] * slack)
        offsets.append(len(hits))
    hit_arr = np.zeros(len(hits), dtype=HIT_DTYPE)
    for j, h in enumerate(hits):
        hit_arr[j] = h
    second = rng.standard_normal((4 * n, 4)).astype(np.float32) if dual else None
    return OpticsInput(verts, patches, dirs, np.array(offsets, dtype=np.uint64), np.array(sums, dtype=SUMMARY_DTYPE),
                       hit_arr, second, k, e0, 1 if dual else 0,
                       (width, height, half, tuple(quarter_turns)) if focal else None)


def _bad_polarization() -> OpticsInput:
    c = lattice_case(7, directions=20, dual=False, faults=False)
    c.polarization = 1  # unpolarized without the second response column
    return c


def _bad_layout() -> OpticsInput:
    c = lattice_case(8, directions=40, faults=False)
    c.focal = (7, 7, 1.01, (0, 4, 0, 0))  # a quarter-turn offset above 3
    return c


CASES = [
    ("unpolarized_focal", lambda: lattice_case(1)),
    ("single_jones_focal", lambda: lattice_case(2, dual=False, quarter_turns=(0, 0, 0, 0))),
    ("unpolarized_path_only", lambda: lattice_case(3, focal=False)),
    ("clean_wide_lattice", lambda: lattice_case(4, width=11, height=9, directions=200, faults=False)),
    ("missing_second_column", _bad_polarization),
    ("invalid_focal_layout", _bad_layout),
]


def serialize(c: OpticsInput) -> bytes:
    fw, fh, fe, fo = c.focal if c.focal else (0, 0, 0.0, (0, 0, 0, 0))
    head = struct.pack("<Q6I6f", len(c.hits), len(c.vertices), len(c.patches), c.count, c.second_len(),
                       c.polarization, 1 if c.focal else 0, *map(float, c.incident), *map(float, c.basis))
    focal = struct.pack("<IIfI4I", fw, fh, fe, 0, *fo)
    parts = [head, focal, c.vertices.tobytes(), c.patches.tobytes(),
             np.ascontiguousarray(c.directions, dtype="<f4").tobytes(), c.offsets.astype("<u8").tobytes(),
             c.summaries.tobytes(), c.hits.tobytes()]
    if c.second is not None and c.second_len():
        parts.append(np.ascontiguousarray(c.second, dtype="<f4").tobytes())
    return b"".join(parts)


def digest(c: OpticsInput) -> str:
    return hashlib.sha256(serialize(c)).hexdigest()


# --------------------------------------------------------------- patch build lattices
def patch_lattice(seed: int, width: int = 9, height: int = 8, faults: bool = True) -> tuple[np.ndarray, tuple]:
    """A four-family lattice for the patch construction: smooth families, one whose scattering
    angle folds over the emitting plane (cells of both orientations and uncertified cells at
    the fold), misses and total internal reflections at the rim, and -- with faults -- invalid
    vertices of each kind."""
    c = lattice_case(seed, width=width, height=height, directions=1, dual=False, focal=False, faults=False)
    v = c.vertices
    rng = np.random.default_rng(seed + 1000)
    n = width * height
    half = 1.01
    k, e0 = c.incident.astype(np.float64), c.basis.astype(np.float64)
    e1 = np.cross(k, e0)
    iy, ix = np.divmod(np.arange(n), width)
    U = (2 * ix / (width - 1) - 1) * half
    V = (2 * iy / (height - 1) - 1) * half
    r2 = U * U + V * V
    theta = 2.3 + 0.6 * r2 - 0.8 * r2 * r2          # folds at r^2 = 0.375
    phi = np.arctan2(V, U)
    d = np.cos(theta)[:, None] * k + np.sin(theta)[:, None] * (np.cos(phi)[:, None] * e0 + np.sin(phi)[:, None] * e1)
    v["direction"][2 * n:3 * n] = _f32_unit(d)
    rim = r2 > 0.98 * half * half
    for f in range(4):
        sl = slice(f * n, (f + 1) * n)
        st = v["status"][sl]
        st[rim] = 2 if f != 3 else 3                      # misses; TIR on the last family
        v["status"][sl] = st
    if faults:
        pick = rng.choice(4 * n, 6, replace=False)
        v["status"][pick[0]] = 4                          # unresolved intersection
        v["status"][pick[1]] = 0                          # unwritten
        v["direction"][pick[2]] *= np.float32(1.001)      # not unit to 2^-16
        v["fraction"][pick[3]] = np.float32(np.nan)
        v["position"][pick[4], 0] = np.inf
        v["field"][pick[5], 2] = np.nan
    return v, (width, height, half)


PATCH_CASES = [
    ("fold_9x8", lambda: patch_lattice(21)),
    ("fold_17x13_clean", lambda: patch_lattice(22, width=17, height=13, faults=False)),
    ("small_2x2", lambda: patch_lattice(23, width=2, height=2, faults=False)),
    ("wide_33x5", lambda: patch_lattice(24, width=33, height=5)),
]


def serialize_lattice(vertices: np.ndarray, layout: tuple) -> bytes:
    w, h, e = layout
    return struct.pack("<IIf", w, h, e) + np.ascontiguousarray(vertices, dtype=VERTEX_DTYPE).tobytes()


# ------------------------------------------------------------- intersection pairs
def intersection_pairs(seed: int = 51, count: int = 3000) -> tuple[np.ndarray, np.ndarray]:
    """(corners [n, 4, 3], directions [n, 3]) float32: patches of a folding lattice queried at
    interior points, at points on and just outside their edges and corners, through folded
    cells, far outside, and with invalid inputs."""
    rng = np.random.default_rng(seed)
    v, (w, h, _) = patch_lattice(seed, width=12, height=11, faults=False)
    n = w * h
    corners, dirs = [], []
    cells = [(f, iy, ix) for f in range(4) for iy in range(h - 1) for ix in range(w - 1)]
    while len(corners) < count:
        f, iy, ix = cells[rng.integers(len(cells))]
        first = f * n + iy * w + ix
        idx = [first, first + 1, first + w, first + w + 1]
        if not (v["status"][idx] == 1).all():
            continue
        c = v["direction"][idx].astype(np.float32)
        kind = rng.integers(0, 6)
        if kind <= 1:
            u, t = rng.random(2)
        elif kind == 2:
            u, t = rng.choice([0.0, 1.0, 1e-7, 1 - 1e-7, 0.5]), rng.random()
        elif kind == 3:
            u, t = rng.uniform(-0.05, 1.05, 2)
        else:
            u, t = rng.uniform(-3, 4, 2)
        p = ((1 - u) * c[0] + u * c[1]) * (1 - t) + ((1 - u) * c[2] + u * c[3]) * t
        d = p / np.linalg.norm(p)
        corners.append(c)
        dirs.append(d.astype(np.float32))
    corners, dirs = np.array(corners, dtype=np.float32), np.array(dirs, dtype=np.float32)
    dirs[0] = [np.nan, 0, 1]
    dirs[1] = dirs[1] * np.float32(1.2)
    corners[2, 1] = [3.0, 0.0, 0.0]
    corners[3, :] = corners[3, 0]  # a degenerate patch
    return corners, dirs


BILINEAR_HITS_DTYPE = np.dtype([("hits", [("u", "<f4"), ("v", "<f4"), ("t", "<f4"), ("residual", "<f4"),
                                          ("flags", "<u4")], 2), ("count", "<u4"), ("flags", "<u4")])
_K20 = (0.9396926164627075, -0.3420201539993286, 0.0)  # float32 (cos 20, -sin 20, 0)
# (theta_count, phi_count, axis, e0) of the query grids pinned to the reference's QueryDirectionGrid
DIRECTION_GRIDS = [(36, 72, _K20, (0.0, 0.0, 1.0)), (7, 5, (0.0, 0.0, 1.0), (1.0, 0.0, 0.0)),
                   (90, 180, (0.0, -1.0, 0.0), (0.0, 0.0, 1.0))]


def bench_lattice(width: int, height: int, seed: int = 61) -> tuple[np.ndarray, np.ndarray, tuple]:
    """A large four-family lattice (vectorised; the bench's input): smooth families, one folding
    at the rainbow angle, misses on the rim; second response column.  (vertices, second, layout)"""
    rng = np.random.default_rng(seed)
    half = 1.01
    k = np.array([math.cos(math.radians(20)), -math.sin(math.radians(20)), 0.0])
    e0 = np.array([0.0, 0.0, 1.0])
    e1 = np.cross(k, e0)
    n = width * height
    iy, ix = np.divmod(np.arange(n), width)
    U = (2 * ix / (width - 1) - 1) * half
    V = (2 * iy / (height - 1) - 1) * half
    r2 = U * U + V * V
    phi = np.arctan2(V, U)
    v = np.zeros(4 * n, dtype=VERTEX_DTYPE)
    for f, theta in enumerate((0.05 + 0.15 * r2, 2.9 - 0.3 * r2, 2.3 + 0.6 * r2 - 0.8 * r2 * r2, 2.2 + 0.2 * r2)):
        d = np.cos(theta)[:, None] * k + np.sin(theta)[:, None] * (np.cos(phi + 0.3 * f)[:, None] * e0 +
                                                                    np.sin(phi + 0.3 * f)[:, None] * e1)
        d = _f32_unit(d)
        axis = np.where(np.abs(d[:, 2:3]) < 0.9, np.array([0, 0, 1.0]), np.array([1.0, 0, 0]))
        sl = slice(f * n, (f + 1) * n)
        v["position"][sl] = np.column_stack([U, V, np.ones(n)]).astype(np.float32)
        v["direction"][sl] = d
        v["basis_x"][sl] = _f32_unit(axis - d * (d * axis).sum(axis=1, keepdims=True))
        v["field"][sl] = rng.standard_normal((n, 4)).astype(np.float32)
        v["turns"][sl] = (1000 + 3000 * r2).astype(np.int32)
        v["fraction"][sl] = rng.random(n).astype(np.float32)
        v["status"][sl] = np.where(r2 > 0.98 * half * half, 2, 1)
    second = rng.standard_normal((4 * n, 4)).astype(np.float32)
    return v, second, (width, height, half)
