"""CPU oracle of the deterministic atlas composition -- TEST INFRASTRUCTURE ONLY.

Restates, in plain Python/NumPy, the reference's orientation composition
(hex_atlas/python/atlas_math.py): the D6h fold of a body direction (fold_direction, :186-210),
the bilinear incident interpolation (interpolation, :213-223), the exact projected area
(projected_area, :226-232), the coupling weights (coupling, :272-310; the vertical-incidence
orbit average of coupling_for_rule, :313-428) and the direct cyclic convolution (compose_mass,
:431-447), plus the ordered CDF (make_cdf, :450-488).  The coupling is written in the same
operation order as the device kernel (ice_crystal_phase_b200/csrc/icp_atlas.cu) and accumulates
in the same exact fixed point (Python integers), so that on the CPU it checks the kernel's
formulas against the reference's golden values (tests/golden/atlas_reference.npz).

Only tests/ may import this module; the product never does.
"""
from __future__ import annotations

import math

import numpy as np

PI = math.pi
EPS = float(np.finfo(np.float64).eps)
SQ3 = math.sqrt(3.0)
FIX = 2.0 ** 62
NORMALS = ((1.0, 0.0, 0.0), (0.5, 0.0, SQ3 / 2), (-0.5, 0.0, SQ3 / 2), (-1.0, 0.0, 0.0), (-0.5, 0.0, -SQ3 / 2),
           (0.5, 0.0, -SQ3 / 2), (0.0, 1.0, 0.0), (0.0, -1.0, 0.0))


class AtlasError(ValueError):
    pass


def unit3(v) -> list[float]:
    s = max(abs(v[0]), abs(v[1]), abs(v[2]))
    if not (s > 0) or not math.isfinite(s):
        raise AtlasError("Expected finite nonzero three-vector")
    a = [v[0] / s, v[1] / s, v[2] / s]
    n = math.sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2])
    return [a[0] / n, a[1] / n, a[2] / n]


def output_frame(ki) -> tuple[list[float], list[float], list[float]]:
    """(e0, e1, k): helper axis = the coordinate axis least aligned with k."""
    k = unit3(ki)
    ax, ay, az = abs(k[0]), abs(k[1]), abs(k[2])
    a = (1.0, 0.0, 0.0) if (ax <= ay and ax <= az) else ((0.0, 1.0, 0.0) if ay <= az else (0.0, 0.0, 1.0))
    d = k[0] * a[0] + k[1] * a[1] + k[2] * a[2]
    e0 = unit3([a[0] - k[0] * d, a[1] - k[1] * d, a[2] - k[2] * d])
    e1 = unit3([k[1] * e0[2] - k[2] * e0[1], k[2] * e0[0] - k[0] * e0[2], k[0] * e0[1] - k[1] * e0[0]])
    return e0, e1, k


def fold(b: list[float]) -> tuple[float, float, float, float, float, float, bool]:
    """(theta, phi, cos(-angle), sin(-angle), sy, sz, mirror) of the D6h operation
    q = Ry(-angle) diag(1, sy, sz) with q k(theta, phi) = b."""
    third, sixth, two_pi = PI / 3, PI / 6, 2 * PI
    theta = math.atan2(math.hypot(b[0], b[2]), abs(b[1]))
    az = math.fmod(math.atan2(b[2], b[0]), two_pi)
    if az < 0:
        az += two_pi
    if az == 0:
        az = 0.0
    sector = min(5, int(az / third))
    local = az - sector * third
    mirror = local > sixth
    phi = third - local if mirror else local
    if phi < -64 * EPS or phi > sixth + 64 * EPS:
        raise AtlasError("Canonical azimuth outside fundamental region")
    phi = min(sixth, max(0.0, phi))
    angle = (sector + (1 if mirror else 0)) * third
    c, s = math.cos(-angle), math.sin(-angle)
    sy = -1.0 if b[1] < 0 else 1.0
    sz = -1.0 if mirror else 1.0
    return theta, phi, c, s, sy, sz, mirror


def projected_area(R: float, L: float, b) -> float:
    u = unit3(b)
    side, cap = R * L, (3 * SQ3 / 2) * R * R
    area = 0.0
    for f, n in enumerate(NORMALS):
        proj = -(n[0] * u[0] + n[1] * u[1] + n[2] * u[2])
        area += (side if f < 6 else cap) * max(0.0, proj)
    return area


def coupling(node_area: np.ndarray, it: int, ip: int, np_: int, R: float, L: float, rotations: np.ndarray,
             weights: np.ndarray, ki, fraction: float = 1.0, orbit: bool = False,
             out: np.ndarray | None = None) -> tuple[np.ndarray, float]:
    """Coupling weights [(it+1)(ip+1)][2][np] (added to `out`, times `fraction`) and the expected
    area sum(weight x projected area)."""
    e0, e1, k = output_frame(ki)
    side, cap = R * L, (3 * SQ3 / 2) * R * R
    bound = 3 * side + cap
    inv_unit = FIX / bound
    nodes = (it + 1) * (ip + 1)
    acc = [[[0] * np_ for _ in range(2)] for _ in range(nodes)]
    expected = 0
    sixth = PI / 6
    for r, nw in zip(rotations.reshape(-1, 9), weights):
        R9 = [float(x) for x in r]
        nw = float(nw)
        b = [R9[j] * k[0] + R9[3 + j] * k[1] + R9[6 + j] * k[2] for j in range(3)]
        b = unit3(b)
        theta, phi, c, s, sy, sz, _ = fold(b)
        st, ct, sp, cp = math.sin(theta), math.cos(theta), math.sin(phi), math.cos(phi)
        kc = (st * cp, ct, st * sp)
        ec = (ct * cp, -st, ct * sp)
        qk = (c * kc[0] + s * sz * kc[2], sy * kc[1], -s * kc[0] + c * sz * kc[2])
        if max(abs(qk[0] - b[0]), abs(qk[1] - b[1]), abs(qk[2] - b[2])) > 2e-12:
            raise AtlasError("Symmetry unfolding is inconsistent")
        qe = (c * ec[0] + s * sz * ec[2], sy * ec[1], -s * ec[0] + c * sz * ec[2])
        ew = [R9[3 * i] * qe[0] + R9[3 * i + 1] * qe[1] + R9[3 * i + 2] * qe[2] for i in range(3)]
        shift = math.atan2(ew[0] * e1[0] + ew[1] * e1[1] + ew[2] * e1[2],
                           ew[0] * e0[0] + ew[1] * e0[1] + ew[2] * e0[2]) / (2 * PI) * np_
        nearest = float(round(shift))
        if abs(shift - nearest) <= 64 * EPS * np_:
            shift = nearest
        lower = math.floor(shift)
        frac = shift - lower
        parity = 1 if sy * sz < 0 else 0
        area = projected_area(R, L, b)
        if not (-64 * EPS <= theta <= PI / 2 + 64 * EPS and -64 * EPS <= phi <= sixth + 64 * EPS):
            raise AtlasError("Incident interpolation outside canonical domain")
        x = min(float(it), max(0.0, theta / (PI / 2) * it))
        y = min(float(ip), max(0.0, phi / sixth * ip))
        i0, j0 = min(it - 1, int(x)), min(ip - 1, int(y))
        ax, by = x - i0, y - j0
        s0, s1 = lower % np_, (lower + 1) % np_
        base = nw * area
        for di in (0, 1):
            for dj in (0, 1):
                mix = (ax if di else 1 - ax) * (by if dj else 1 - by)
                if not mix > 0:
                    continue
                row = acc[(i0 + di) * (ip + 1) + (j0 + dj)][parity]
                v = base * mix
                row[s0] += round(v * (1 - frac) * inv_unit)
                row[s1] += round(v * frac * inv_unit)
        expected += round(base * inv_unit)
    unit = bound / FIX
    w = np.zeros((nodes, 2, np_)) if out is None else out
    for n in range(nodes):
        scale = unit / float(node_area.reshape(-1)[n])
        for q in range(2):
            vals = np.array([float(a) * scale for a in acc[n][q]])
            if orbit:
                w[n, q] += fraction * (vals.sum() / np_)
            else:
                w[n, q] += fraction * vals
    return w, float(expected) * unit


def compose(mass: np.ndarray, w: np.ndarray) -> np.ndarray:
    """sum over nodes, parities, shifts (that order, products and sums rounded separately) of
    w * the node's cell masses, phi-reflected for parity 1, rolled by the shift."""
    nodes, nt, np_ = mass.shape
    out = np.zeros((nt, np_))
    for n in range(nodes):
        for q in range(2):
            cell = mass[n][:, ::-1] if q else mass[n]
            for s in range(np_):
                v = float(w[n, q, s])
                if v > 0:
                    out += v * np.roll(cell, s, axis=1)
    return out


def make_cdf(mass: np.ndarray, edges: np.ndarray) -> tuple[np.ndarray, np.ndarray, dict]:
    """Ordered phi marginal and theta|phi CDFs of a cell-mass grid, with the recovered-mass audit."""
    nt, np_ = mass.shape
    raw = mass / float(mass.max())
    b = np.zeros((np_, nt + 1))
    b[:, 1:] = np.cumsum(raw.T, axis=1)
    cols = b[:, -1].copy()
    a = np.zeros(np_ + 1)
    a[1:] = np.cumsum(cols)
    a /= a[-1]
    for j in range(np_):
        b[j] = b[j] / cols[j] if cols[j] > 0 else edges
    target = (mass / math.fsum(mass.flat)).T
    rec = np.diff(a)[:, None] * np.diff(b, axis=1)
    g = float(np.sum(rec * (1 - edges[:-1] - edges[1:])[None, :]) / np.sum(rec))
    return a, b, {"l1": math.fsum(np.abs(target - rec).flat), "g": g, "cdf_mass": math.fsum(rec.flat)}
