"""Regenerates the golden fixtures in tests/golden/ from the REFERENCE implementation.

Runs the reference's own CPU code, compiled from its sources by oracle/build_ref.sh into
oracle/_ref/ (ice_generate_phase_cpu and the ref_hex_harness driver), and stores its
outputs as small .npz files.  Needs the reference checkout (default /root/reference);
the fixtures are committed so that tests never need it.

    python tests/golden/make_golden.py [REFERENCE_ROOT]
"""
from __future__ import annotations

import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REF = Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference")
REF_BIN = ROOT / "oracle" / "_ref"

# The reference's CLI test plan (hex_phase/configs/two_orientations.csv), reproduced as data:
# identity and an active +90 degree rotation about +z; 1024 and 2048 rays.
TWO_ORIENTATIONS = ("qw,qx,qy,qz,weight,samples,seed\n"
                    "1,0,0,0,0.5,1024,12345\n"
                    "0.7071067811865475244,0,0,0.7071067811865475244,0.5,2048,54321\n")
# Config-3 geometry: circumradius 0.05 mm, length 0.2 mm, n = 1.31, ki = (cos30, -sin30, 0).
CONFIG3_PLAN = "qw,qx,qy,qz,weight,samples,seed\n1,0,0,0,1,20000,12345\n"


def run(cmd):
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode:
        raise SystemExit(f"{cmd[0]} failed: {r.stderr}")
    return r


def masses(td: Path, R, L, ki, n, nt, np_, plan: str, max_hits=1024, tail=1e-12, batch=4096):
    csv = td / "plan.csv"
    csv.write_text(plan)
    out = td / "m.bin"
    run([REF_BIN / "ref_hex_harness", "masses", repr(R), repr(L), *map(repr, ki), repr(n), "1", nt, np_, max_hits,
         repr(tail), csv, batch, out])
    raw = out.read_bytes()
    k = nt * np_
    return (np.frombuffer(raw[:8 * k], "<f8").copy(), np.frombuffer(raw[8 * k:8 * k + 72], "<f8").copy(),
            np.frombuffer(raw[8 * k + 72:], "<u8").copy())


def main() -> None:
    subprocess.run([str(ROOT / "oracle" / "build_ref.sh"), str(REF)], check=True)
    with tempfile.TemporaryDirectory() as t:
        td = Path(t)
        # 1. the reference CLI test record (phase_cli_test.py:242-246) + its masses
        csv = td / "two.csv"
        csv.write_text(TWO_ORIENTATIONS)
        out = td / "rec"
        run([REF_BIN / "ice_generate_phase_cpu", "--orientations", csv, "--radius-mm", "0.1", "--length-mm", "0.2",
             "--ki", "1", "-0.4", "0.3", "--ior", "1.31", "--wavelength-nm", "550", "--theta", "72", "--phi", "144",
             "--cdf-theta", "36", "--cdf-phi", "72", "--out", out, "--batch-size", "512"])
        meta = json.loads((out / "metadata.json").read_text())
        m, d, u = masses(td, 0.1, 0.2, (1.0, -0.4, 0.3), 1.31, 72, 144, TWO_ORIENTATIONS, batch=512)
        np.savez_compressed(
            HERE / "hex_two_orientations.npz", masses=m, stats=d, counts=u,
            phi=np.load(out / "phi_cdf.npy"), theta=np.load(out / "theta_given_phi_cdf.npy"),
            u=np.load(out / "u_edges.npy"),
            meta=np.array([meta["hg"]["g"], meta["quality"]["cdf_l1_mass_error"],
                           meta["storage_processing"]["coarsening_tv"], meta["transport_audit"]["escaped_mm2"],
                           meta["transport_audit"]["unresolved_mm2"], meta["geometry"]["projected_area_mm2"],
                           meta["histogram"]["mass_mm2"], meta["histogram"]["g_rays"]]),
            sampling_frame_columns=np.array(meta["sampling_frame_columns"]))
        # 2. config-3 geometry at 512x1024, 20k rays, 12 hits (sparse: the masses are a few hundred deltas)
        ki = (0.8660254037844387, -0.5, 0.0)
        m, d, u = masses(td, 0.05, 0.2, ki, 1.31, 512, 1024, CONFIG3_PLAN, max_hits=12)
        nz = np.flatnonzero(m)
        np.savez_compressed(HERE / "hex_config3_20k.npz", index=nz, value=m[nz], stats=d, counts=u)
        # 3. per-ray reference audits and exits for 48 rays of the config-3 node
        out = td / "t.bin"
        run([REF_BIN / "ref_hex_harness", "trace", "0.05", "0.2", *map(repr, ki), "1.31", "1", 12345, 20000, 1024,
             repr(1e-12), 100, 48, out])
        raw = np.frombuffer(out.read_bytes(), "<f8")
        info = raw[:48 * 6].reshape(48, 6)
        exits = raw[48 * 6:].reshape(-1, 4)
        np.savez_compressed(HERE / "hex_rays.npz", info=info, exits=exits)
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
