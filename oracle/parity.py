"""Same-seed parity of a traced drop record slice against the FP64 oracle.

TEST INFRASTRUCTURE ONLY (the checker).  tests/ call `drop_parity` in-process; bench.py runs
this module in a subprocess after its timed region, so the oracle library never loads into the
process that measures the device:

    python -m oracle.parity <slice.npz>        -> one JSON object on stdout

The .npz holds the device's cell masses of ray ids [first, first + count) of a `rays`-ray record
(pole caps spread over the end rows, as PhaseMassAccumulator::masses, hex_phase/src/phase_table.cpp:
41-76), its transport audit and the record's parameters.  The oracle traces the same ray ids with
the same counter-RNG seed (drop_record_sharded), and the two histograms are compared with the
metrics of the reference's record comparison (tools/phase_analysis.py:244-315: total variation of
normalised cell mass, asymmetry parameter g):

* tv        0.5 * sum |p_dev - p_oracle|, p = cell mass / total (pole rows included);
* g         sum m * mu / sum m with mu = 1 - U_i - U_{i+1} the mean cosine of row i, for each side;
* energy    |escaped + unresolved - incident| / incident of the device (ray power is exact
            fixed point on the device, so this is binary64 rounding);
* noise floor  the expected TV between two independent runs of N rays, (1/sqrt(pi)) sum_k
            sqrt(p_k / N) (the Monte Carlo floor a different seed would show), at the slice's N and
            at the full record's N.

Because every ray depends only on (seed, ray id), the slice's same-seed TV measures the
per-ray disagreement (FP32 against FP64 arithmetic: exits that fall in a neighbouring cell,
rounding of powers) independently of the record's size.
"""
from __future__ import annotations

import json
import math
import sys
from pathlib import Path

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    from oracle import oracle as O  # noqa: E402
else:
    from . import oracle as O


def row_mu(nt: int) -> np.ndarray:
    e = O.u_edges(nt)
    return 1.0 - e[:-1] - e[1:]


def g_of(masses: np.ndarray, nt: int) -> float:
    m = masses.reshape(nt, -1)
    return float((m.sum(axis=1) * row_mu(nt)).sum() / m.sum())


def noise_floor(p: np.ndarray, n: float) -> float:
    return float(np.sqrt(p / n).sum() / math.sqrt(math.pi))


def drop_parity(dev_masses: np.ndarray, cfg: dict, audit: dict, workers: int | None = None) -> dict:
    """cfg: coefficients, radius_mm, interior_index, inclination_deg, nt, np, rays, seed,
    max_internal_hits, first, count.  audit: escaped, unresolved, incident (mm^2) of the device."""
    nt, np_ = int(cfg["nt"]), int(cfg["np"])
    geo = O.drop_geometry(cfg["coefficients"], float(cfg["radius_mm"]))
    frame = O.drop_frame(float(cfg["inclination_deg"]))
    rec = O.drop_record_sharded(geo, frame, float(cfg["interior_index"]), nt, np_, int(cfg["rays"]),
                                int(cfg["seed"]), max_hits=int(cfg["max_internal_hits"]), first=int(cfg["first"]),
                                count=int(cfg["count"]), workers=workers)
    a = np.asarray(dev_masses, dtype=np.float64).reshape(-1)
    b = rec.masses
    pa, pb = a / a.sum(), b / b.sum()
    tv = 0.5 * float(np.abs(pa - pb).sum())
    ga, gb = g_of(a, nt), g_of(b, nt)
    hits = rec.counts["rays"] - rec.counts["missed"]
    energy = abs(audit["escaped"] + audit["unresolved"] - audit["incident"]) / audit["incident"]
    return {"rays": int(cfg["count"]), "first_ray": int(cfg["first"]), "record_rays": int(cfg["rays"]),
            "hit_rays": int(hits), "tv": tv, "g_device": ga, "g_oracle": gb, "g_abs_error": abs(ga - gb),
            "energy_residual_device": energy,
            "energy_residual_oracle": abs(rec.escaped_area + rec.unresolved_area - rec.incident_area)
            / rec.incident_area,
            "escaped_relative_difference": abs(audit["escaped"] / rec.escaped_area - 1),
            "missed_device": int(audit.get("missed", -1)), "missed_oracle": int(rec.counts["missed"]),
            "noise_floor_slice": noise_floor(pb, max(1, hits)),
            "noise_floor_record": noise_floor(pb, max(1.0, hits * float(cfg["rays"]) / float(cfg["count"]))),
            "oracle": "FP64 C restatement (oracle/icp_oracle.c), same seed and ray ids",
            "metric": "TV of normalised cell mass and g as tools/phase_analysis.py compare_tables"}


def main(argv: list[str]) -> int:
    z = np.load(argv[1], allow_pickle=False)
    cfg = json.loads(str(z["cfg"]))
    audit = json.loads(str(z["audit"]))
    print(json.dumps(drop_parity(z["masses"], cfg, audit)), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
