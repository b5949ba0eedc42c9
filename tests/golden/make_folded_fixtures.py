"""Writes tests/golden/folded_reference.npz: the REFERENCE's folded-patch records and the per-
direction optics evaluated with them, on the reference's own lattices of real drops.

    python tests/golden/make_folded_fixtures.py [REFERENCE_ROOT]

Per case the chain is: the lattice (RaindropPathTracer::trace_vertex_unpolarized,
oracle/_ref/ref_drop_harness vertices), its patches (PatchConstruction::make,
oracle/_ref/ref_patch_harness), the query directions (QueryDirectionGrid,
oracle/_ref/ref_query_harness directions), the all-hit query (the oracle's restatement of the
reference's OptiX query and PatchHitCollector, pinned by the query fixtures), and the optics
with folded records (FoldedPatchBuilder::prepare + PatchOpticalEvaluator::evaluate_direction
with a FoldedPatchView, oracle/_ref/ref_optics_harness ... folded), with the focal stage.
Stored: the SHA-256 of the serialised optics input, the records (compact-index order) with the
record index of every patch, the optical and focal results of the directions with refinement
hits, and a SHA-256 over every direction's optical and focal counters and flags.
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
REF_BIN = ROOT / "oracle" / "_ref"
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT))

import optics_cases as OC  # noqa: E402
import rainbow_cases as RC  # noqa: E402

FOLDED_BRANCH = [("u0", "<f8"), ("u1", "<f8"), ("area_fraction", "<f8"), ("solid_angle_sr", "<f8"),
                 ("representative_u", "<f8"), ("representative_v", "<f8"), ("sign", "<i4"), ("focal_flags", "<u4"),
                 ("quarter_turns", "<u4"), ("extra_quarter_turn", "<u4")]
FOLDED_DTYPE = np.dtype([("compact_index", "<u4"), ("patch_id", "<u4"), ("flags", "<u4"), ("branch_count", "<u4"),
                         ("jacobian", "<f8", 4), ("branches", np.dtype(FOLDED_BRANCH), 4),
                         ("largest_estimated_relative_error", "<f8"), ("panels", "<u4"), ("reserved", "<u4")])
assert FOLDED_DTYPE.itemsize == 320

# name: (lattice args for ref_drop_harness vertices: radius sphere n_int kx ky kz grid [wavelength [c0..c7]],
#        query theta, query phi)
CASES = {
    "sphere_0.5mm_700nm_25_q90x180": (["0.5", "1", "1.3317", "0.9396926", "-0.3420201", "0", "25"], 90, 180),
    "table1_1.5mm_550nm_33_q60x120": (["1.5", "0", "1.3335", "1", "-0.3", "0.1", "33", "550"], 60, 120),
    "oblate_1.5mm_650nm_41_q72x144": (["1.5", "0", "1.3319", "0.9396926", "-0.3420201", "0", "41", "650",
                                       "0", "-0.08", "-0.02", "0.005", "0", "0", "0", "0"], 72, 144),
}


def run(cmd):
    subprocess.run([str(c) for c in cmd], check=True)


def chain_input(td: Path, args, nt, np_):
    from oracle import oracle as O
    lat = td / "lattice.bin"
    run([REF_BIN / "ref_drop_harness", "vertices", *args[:7], lat, *args[7:]])
    raw = lat.read_bytes()
    w, h = (int(x) for x in np.frombuffer(raw[:8], "<u4"))
    frame = np.frombuffer(raw[8:36], "<f4")
    n = 4 * w * h
    v = np.frombuffer(raw[36:36 + 68 * n], OC.VERTEX_DTYPE).copy()
    second = np.frombuffer(raw[36 + 68 * n:], "<f4").reshape(-1, 4).copy()
    e = float(frame[0])
    src, dst = td / "pa.in", td / "pa.out"
    src.write_bytes(OC.serialize_lattice(v, (w, h, e)))
    run([REF_BIN / "ref_patch_harness", src, dst])
    pr = dst.read_bytes()
    cells = 4 * (w - 1) * (h - 1)
    count = int(np.frombuffer(pr[4 * cells:4 * cells + 4], "<u4")[0])
    off = 4 * cells + 36
    patches = np.frombuffer(pr[off:off + 32 * count], OC.PATCH_DTYPE).copy()
    aabbs = np.frombuffer(pr[off + 32 * count:off + 56 * count], OC.AABB_DTYPE).copy()
    k, e0 = frame[1:4].copy(), frame[4:7].copy()
    dirs = O.ref_query_directions(nt, np_, k, e0, td)
    offsets, summaries, hits = O.patch_query(v, patches, aabbs, dirs)
    return OC.OpticsInput(v, patches, dirs, offsets, summaries, hits, second, k, e0, 1, (w, h, e, (0, 0, 0, 0)))


OPTICAL_COUNTERS = ("hit_count", "evaluated_hits", "rejected_hits", "refinement_hits", "boundary_hits",
                    "singular_hits", "flags", "query_flags", "first_problem_patch_id", "folded_hits")
FOCAL_COUNTERS = ("family_hits", "corrected_hits", "extra_quarter_turn_hits", "flags", "first_problem_patch_id")


def counters_digest(optical, focal) -> str:
    """SHA-256 over every direction's optical and focal counters and flags (exact integers)."""
    h = hashlib.sha256()
    for k in OPTICAL_COUNTERS:
        h.update(np.ascontiguousarray(optical[k]).tobytes())
    for k in FOCAL_COUNTERS:
        h.update(np.ascontiguousarray(focal[k]).tobytes())
    return h.hexdigest()


def main() -> None:
    subprocess.run([str(ROOT / "oracle" / "build_ref.sh"), str(REF)], check=True)
    out = {}
    with tempfile.TemporaryDirectory() as t:
        td = Path(t)
        for name, (args, nt, np_) in CASES.items():
            c = chain_input(td, args, nt, np_)
            src, dst = td / "op.in", td / "op.out"
            src.write_bytes(OC.serialize(c))
            run([REF_BIN / "ref_optics_harness", src, dst, "folded"])
            raw = dst.read_bytes()
            n = c.count
            fs = RC.FOCAL_DTYPE.itemsize
            optical = np.frombuffer(raw[:136 * n], OC.OPTICAL_DTYPE)
            focal = np.frombuffer(raw[136 * n:136 * n + fs * n], RC.FOCAL_DTYPE)
            pos = 136 * n + fs * n
            rc = int(np.frombuffer(raw[pos:pos + 4], "<u4")[0])
            pc = len(c.patches)
            indices = np.frombuffer(raw[pos + 4:pos + 4 + 4 * pc], "<u4").copy()
            records = np.frombuffer(raw[pos + 4 + 4 * pc:], FOLDED_DTYPE).copy()
            assert len(records) == rc
            refined = np.flatnonzero(c.summaries["refinement_hits"] > 0).astype(np.uint32)
            out[f"{name}.args"] = np.array(" ".join(args))
            out[f"{name}.query"] = np.array([nt, np_], np.uint32)
            out[f"{name}.digest"] = np.array(OC.digest(c))
            out[f"{name}.record_indices"] = indices
            out[f"{name}.records"] = records
            out[f"{name}.refined"] = refined
            out[f"{name}.optical"] = optical[refined].copy()
            out[f"{name}.focal"] = focal[refined].copy()
            out[f"{name}.counters_sha256"] = np.array(counters_digest(optical, focal))
            print(name, "patches", pc, "records", rc, "ready", int((records["flags"] == 0).sum()), "refined", len(refined),
                  "folded hits", int(optical["folded_hits"].sum()),
                  "pending dirs", int(((optical["flags"] & (32 | 64 | 128)) != 0).sum()))
    np.savez_compressed(HERE / "folded_reference.npz", **out)


if __name__ == "__main__":
    main()
