"""Synthetic focal-stage query grids for the Table-II rainbow diffraction tests.

`paper_grid` restates the reference's own diffraction fixture
(tests/wave_optics_test_cases.hpp:82-99 of the reference): a primary bow entering TRT support
at theta > 138 + 0.8 sin(phi) degrees and a secondary bow leaving TRRT support at
theta < 129 + 0.5 sin(phi), with the total intensity jumping at both.  `bow_grid` widens it
with seeded noise, wobbling bows, hit counts, and unavailable samples of every kind the
reference's sample check rejects (nonzero flags, negative, NaN and infinite intensities).
`CASES` is the list of fixture grids: tests/golden/rainbow_reference.npz (made by
tests/golden/make_golden.py) holds the reference's outputs and the SHA-256 of each input grid,
so the tests rebuild the inputs here and check that they are the ones the reference saw.
"""
from __future__ import annotations

import math

import numpy as np

FOCAL_DTYPE = np.dtype([("field", "<f8", 4), ("intensity_s", "<f8"), ("intensity_p", "<f8"),
                        ("family_incoherent", "<f8", 4), ("family_hits", "<u4", 4), ("corrected_hits", "<u4"),
                        ("extra_quarter_turn_hits", "<u4"), ("flags", "<u4"), ("first_problem_patch_id", "<u4"),
                        ("field_second", "<f8", 4)])
RESULT_DTYPE = np.dtype([("intensity_s", "<f8"), ("intensity_p", "<f8"), ("sigma_rad", "<f8"), ("blend", "<f8"),
                         ("flags", "<u4"), ("transition_kind", "<u4")])
PAPER_CONFIG = (2 * math.pi / 180, 4.0, 0.25, 3.0)


def _axes(rows: int, cols: int) -> tuple[np.ndarray, np.ndarray]:
    r = np.repeat(np.arange(rows), cols)
    c = np.tile(np.arange(cols), rows)
    return 180 * (r + 0.5) / rows, 2 * math.pi * c / cols


def paper_grid(rows: int = 180, cols: int = 72) -> np.ndarray:
    deg, phi = _axes(rows, cols)
    primary = deg > 138 + 0.8 * np.sin(phi)
    secondary = deg < 129 + 0.5 * np.sin(phi)
    total = 1 + np.where(primary, 8, 0) + np.where(secondary, 2, 0)
    f = np.zeros(rows * cols, dtype=FOCAL_DTYPE)
    f["intensity_s"] = 0.8 * total
    f["intensity_p"] = 0.2 * total
    f["family_hits"][:, 2] = np.where(primary, 2, 0)
    f["family_hits"][:, 3] = np.where(secondary, 2, 0)
    f["family_incoherent"][:, 2] = np.where(primary, 8, 0)
    f["family_incoherent"][:, 3] = np.where(secondary, 2, 0)
    return f


def bow_grid(rows: int, cols: int, seed: int, primary_deg: float = 138.0, secondary_deg: float = 129.0,
             wobble: float = 1.0, noise: float = 0.3, invalid: float = 0.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    deg, phi = _axes(rows, cols)
    primary = deg > primary_deg + wobble * (0.8 * np.sin(phi) + 0.6 * np.cos(2 * phi))
    secondary = deg < secondary_deg + wobble * (0.5 * np.sin(phi) - 0.4 * np.cos(3 * phi))
    base = 1 + np.where(primary, 8, 0) + np.where(secondary, 2, 0)
    total = base * (1 + noise * rng.standard_normal(deg.size)).clip(0.05)
    f = np.zeros(rows * cols, dtype=FOCAL_DTYPE)
    split = rng.uniform(0.2, 0.9, deg.size)
    f["intensity_s"] = split * total
    f["intensity_p"] = (1 - split) * total
    f["family_hits"][:, 2] = np.where(primary, rng.integers(1, 6, deg.size), 0)
    f["family_hits"][:, 3] = np.where(secondary, rng.integers(1, 6, deg.size), 0)
    f["family_incoherent"][:, 2] = np.where(primary, rng.uniform(0.5, 9, deg.size), 0)
    f["family_incoherent"][:, 3] = np.where(secondary, rng.uniform(0.1, 3, deg.size), 0)
    f["family_hits"][:, 1] = rng.integers(0, 3, deg.size)
    f["family_incoherent"][:, 1] = rng.uniform(0, 1, deg.size)
    if invalid > 0:
        bad = np.flatnonzero(rng.random(deg.size) < invalid)
        kind = rng.integers(0, 5, bad.size)
        f["flags"][bad[kind == 0]] = rng.choice([1, 2, 4, 8, 16], int((kind == 0).sum()))
        f["intensity_s"][bad[kind == 1]] = -rng.uniform(1e-6, 1, int((kind == 1).sum()))
        f["intensity_p"][bad[kind == 2]] = np.nan
        f["intensity_s"][bad[kind == 3]] = np.inf
        f["intensity_p"][bad[kind == 4]] = 1e308  # finite alone, s + p overflows
        f["intensity_s"][bad[kind == 4]] = 1e308
    return f


# (name, rows, cols, config, builder, labels) -- labels "detect" or an edit of the detected ones
CASES = [
    ("paper", 180, 72, PAPER_CONFIG, lambda: paper_grid(), "detect"),
    ("paper_coarse_sigma", 180, 72, (0.15 * math.pi / 180, 4.0, 0.25, 3.0), lambda: paper_grid(), "detect"),
    ("paper_hole", 180, 72, PAPER_CONFIG, lambda: _with_pending(paper_grid(), 137 * 72 + 1), "detect"),
    ("paper_unknown_label", 180, 72, PAPER_CONFIG, lambda: paper_grid(), "unknown@9865"),
    ("paper_no_labels", 180, 72, PAPER_CONFIG, lambda: paper_grid(), "none"),
    ("bows_noisy", 90, 180, (0.7 * math.pi / 180, 4.0, 0.25, 3.0), lambda: bow_grid(90, 180, 11), "detect"),
    ("bows_invalid", 120, 96, (1.1 * math.pi / 180, 4.0, 0.2, 3.0), lambda: bow_grid(120, 96, 12, invalid=0.004),
     "detect"),
    ("bows_wide_poles", 24, 40, (6.0 * math.pi / 180, 6.0, 0.1, 1.5),
     lambda: bow_grid(24, 40, 13, primary_deg=150, secondary_deg=20, wobble=4), "detect"),
    ("one_column", 60, 1, (1.5 * math.pi / 180, 4.0, 0.25, 3.0), lambda: bow_grid(60, 1, 14, wobble=0), "detect"),
    ("two_rows", 2, 9, (30.0 * math.pi / 180, 2.0, 0.0, 0.0), lambda: _two_rows(), "detect"),
    ("fine_strip", 720, 8, (0.3 * math.pi / 180, 4.0, 0.25, 3.0), lambda: bow_grid(720, 8, 15, noise=0.05), "detect"),
    ("zero_intensity", 180, 72, PAPER_CONFIG, lambda: _flat(0.0, 0.0), "of:paper"),
    ("constant", 180, 72, PAPER_CONFIG, lambda: _flat(3.25, 0.125), "of:paper"),
]


def _with_pending(f: np.ndarray, index: int) -> np.ndarray:
    f["flags"][index] = 2  # FocalInputPending
    return f


def _two_rows() -> np.ndarray:
    f = np.zeros(18, dtype=FOCAL_DTYPE)
    f["intensity_s"] = [1, 2, 3, 4, 5, 6, 7, 8, 9, 9, 1, 9, 1, 9, 1, 9, 1, 9]
    f["intensity_p"] = 0.5
    f["family_hits"][9:, 2] = 1
    f["family_incoherent"][9:, 2] = 1
    f["family_hits"][:9:2, 3] = 1
    f["family_incoherent"][:9, 3] = 1
    return f


def _flat(s: float, p: float) -> np.ndarray:
    f = paper_grid()
    f["intensity_s"] = s
    f["intensity_p"] = p
    return f


def labels_for(spec: str, detect) -> np.ndarray | None:
    """None for the pass's own labels, else the labels handed to the filter; detect(grid) gives
    the labels of a grid ("of:paper" takes the paper grid's labels for another grid)."""
    if spec == "detect":
        return None
    if spec == "of:paper":
        return detect(paper_grid())
    e = detect(None).copy()
    if spec == "none":
        e[:] = 0
    elif spec.startswith("unknown@"):
        e[int(spec.split("@")[1])] = 4  # TransitionUnknown
    return e


def digest(f: np.ndarray) -> str:
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(f, dtype=FOCAL_DTYPE).tobytes()).hexdigest()


def expected(z, name: str, focal: np.ndarray) -> np.ndarray:
    """The reference's full result array of a fixture case: unflagged directions keep their
    input intensities with zero width, blend and kind; the flagged ones are stored."""
    flags = z[f"{name}.flags"]
    out = np.zeros(flags.size, dtype=RESULT_DTYPE)
    out["intensity_s"], out["intensity_p"], out["flags"] = focal["intensity_s"], focal["intensity_p"], flags
    at = z[f"{name}.changed"].astype(np.int64)
    for k in ("intensity_s", "intensity_p", "sigma_rad", "blend", "transition_kind"):
        out[k][at] = z[f"{name}.{k}"]
    return out
