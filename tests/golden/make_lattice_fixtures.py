"""Writes tests/golden/drop_lattice_cases.npz: the REFERENCE's unpolarised lattice trace
(RaindropPathTracer::trace_vertex_unpolarized with RaindropIntersector, run on the CPU by
oracle/_ref/ref_drop_harness, which oracle/build_ref.sh compiles from the reference's sources)
for a few drops, as the bit-exact target of the device lattice trace.

    python tests/golden/make_lattice_fixtures.py [REFERENCE_ROOT]

Per case: the harness arguments, the 116-byte RaindropTraceConfig, SHA-256 digests of the full
vertex (68 B records) and second-column (16 B) buffers, the per-family status histogram, the
number of records the trace validation rejects, and the records of the lattice's middle row (all
four families) for a readable first difference.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REF = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(os.environ.get("ICP_REFERENCE_ROOT", "/root/reference"))
HARNESS = ROOT / "oracle" / "_ref" / "ref_drop_harness"

VERTEX_DTYPE = np.dtype([("position", "<f4", 3), ("direction", "<f4", 3), ("basis_x", "<f4", 3), ("field", "<f4", 4),
                         ("turns", "<i4"), ("fraction", "<f4"), ("status", "<u4"), ("diagnostics", "<u4")])

# name: radius sphere n_int kx ky kz grid wavelength [c0 .. c7]
CASES = {
    "sphere_0.5mm_700nm_25": ["0.5", "1", "1.3317", "0.9396926", "-0.3420201", "0", "25", "700"],
    "table1_1.5mm_550nm_33": ["1.5", "0", "1.3335", "1", "-0.3", "0.1", "33", "550"],
    # the benchmark drop: r/a = 1 - 0.08 cos chi - 0.02 cos 2chi + 0.005 cos 3chi, inclination 20 deg
    "oblate_1.5mm_650nm_41": ["1.5", "0", "1.3319", "0.9396926", "-0.3420201", "0", "41", "650",
                              "0", "-0.08", "-0.02", "0.005", "0", "0", "0", "0"],
    # incident direction within |k_z| >= 0.9: the transverse basis starts from the x axis
    "table1_2.5mm_450nm_steep_17": ["2.5", "0", "1.34", "0.1", "0.2", "0.97", "17", "450"],
    "table1_3mm_700nm_129": ["3.0", "0", "1.3314", "1", "0", "0", "129", "700"],
}


def main() -> None:
    subprocess.run([str(ROOT / "oracle" / "build_ref.sh"), str(REF)], check=True)
    out = {}
    with tempfile.TemporaryDirectory() as t:
        for name, args in CASES.items():
            cfg = subprocess.run([str(HARNESS), "config", *args], capture_output=True, text=True, check=True)
            cfg_bytes = bytes.fromhex(cfg.stdout.strip())
            path = Path(t) / f"{name}.bin"
            vargs = [*args[:7], str(path), *args[7:]]
            subprocess.run([str(HARNESS), "vertices", *vargs], check=True)
            raw = path.read_bytes()
            w, h = (int(x) for x in np.frombuffer(raw[:8], "<u4"))
            n = 4 * w * h
            vb = raw[36:36 + 68 * n]
            sb = raw[36 + 68 * n:]
            assert len(sb) == 16 * n
            v = np.frombuffer(vb, VERTEX_DTYPE)
            second = np.frombuffer(sb, "<f4").reshape(-1, 4)
            hist = np.zeros((4, 8), np.uint64)
            st = v["status"].reshape(4, -1)
            for f in range(4):
                hist[f] = np.bincount(np.minimum(st[f], 7), minlength=8)[:8]
            valid = v["status"] == 1
            finite = (np.isfinite(v["position"]).all(1) & np.isfinite(v["direction"]).all(1) &
                      np.isfinite(v["basis_x"]).all(1) & np.isfinite(v["field"]).all(1) & np.isfinite(second).all(1) &
                      (v["fraction"] >= 0) & (v["fraction"] < 1))
            bad = ~np.isin(v["status"], [1, 2, 3]) | (valid & ~finite)
            mid = h // 2
            rows = np.concatenate([np.arange(f * w * h + mid * w, f * w * h + mid * w + w) for f in range(4)])
            out[f"{name}.args"] = np.array(" ".join(args))
            out[f"{name}.config"] = np.frombuffer(cfg_bytes, np.uint8).copy()
            out[f"{name}.vertices_sha256"] = np.array(hashlib.sha256(vb).hexdigest())
            out[f"{name}.second_sha256"] = np.array(hashlib.sha256(sb).hexdigest())
            out[f"{name}.histogram"] = hist
            out[f"{name}.incomplete"] = np.array(int(bad.sum()), np.uint64)
            out[f"{name}.first_problem"] = np.array(int(np.flatnonzero(bad)[0]) if bad.any() else 2 ** 64 - 1,
                                                    np.uint64)
            out[f"{name}.row_index"] = rows.astype(np.uint32)
            out[f"{name}.row_vertices"] = v[rows].copy()
            out[f"{name}.row_second"] = second[rows].copy()
    np.savez_compressed(HERE / "drop_lattice_cases.npz", **out)


if __name__ == "__main__":
    main()
