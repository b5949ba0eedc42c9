"""Writes small records with this repository's command-line drop-ins into tests/golden/records/.

Needs a CUDA device (the CLIs run the sm_100a kernels); run from the repository root after the
build:

    python tests/golden/make_record_fixtures.py [out_dir]

The records (hex column through ice_generate_phase, water drops through rainbow_generate -- the
ray model and the reference's default patch-model diffraction stage -- at small grids so that
they stay a few tens of KB) are the inputs of tests/test_record_reader_cpu.py,
which checks them with the reference's own record reader where the reference checkout is present.
"""
from __future__ import annotations

import shutil
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
BIN = ROOT / "ice_crystal_phase_b200" / "bin"
PLAN = ("qw,qx,qy,qz,weight,samples,seed\n"
        "1,0,0,0,0.5,1024,12345\n"
        "0.7071067811865475244,0,0,0.7071067811865475244,0.5,2048,54321\n")

RECORDS = {
    # the reference CLI test's plan and grids (hex_phase/tests/phase_cli_test.py:34-110)
    "hex_two_orientations_72x144_36x72": ["ice_generate_phase", "--radius-mm", "0.1", "--length-mm", "0.2", "--ki", "1",
                                          "-0.4", "0.3", "--ior", "1.31", "--wavelength-nm", "550", "--theta", "72",
                                          "--phi", "144", "--cdf-theta", "36", "--cdf-phi", "72"],
    # the benchmark drop's shape at a small grid, with the analytic diffraction stage
    "drop_oblate_1.5mm_650nm_90x180": ["rainbow_generate", "--wavelength-nm", "650", "--radius-mm", "1.5",
                                       "--shape-coefficients", "0,-0.08,-0.02,0.005", "--inclination-deg", "20",
                                       "--query-theta", "90", "--query-phi", "180", "--stage", "incoherent",
                                       "--rays", "200000",
                                       "--max-internal-hits", "10", "--max-unresolved-fraction", "1e-3",
                                       "--diffraction", "analytic"],
    # a Table-I drop, stored coarser than traced
    "drop_table1_0.5mm_550nm_72x144_36x72": ["rainbow_generate", "--wavelength-nm", "550", "--radius-mm", "0.5",
                                             "--query-theta", "72", "--query-phi", "144", "--cdf-theta", "36",
                                             "--cdf-phi", "72", "--stage", "incoherent", "--rays", "100000"],
    # the reference's default stage: the patch model with Table-II diffraction, lattice 129 x 129
    "drop_diffraction_0.5mm_650nm_grid129_90x180": ["rainbow_generate", "--wavelength-nm", "650", "--radius-mm",
                                                    "0.5", "--grid", "129", "--query-theta", "90", "--query-phi",
                                                    "180", "--allow-underresolved"],
}


def main(out_dir: Path) -> int:
    out_dir.mkdir(parents=True, exist_ok=True)
    plan = out_dir / "two_orientations.csv"
    plan.write_text(PLAN)
    for name, (exe, *args) in RECORDS.items():
        target = out_dir / name
        if target.exists():
            shutil.rmtree(target)
        extra = ["--orientations", str(plan)] if exe == "ice_generate_phase" else []
        r = subprocess.run([str(BIN / exe), *extra, *args, "--out", str(target)], capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            return r.returncode
        print(name, "written")
    plan.unlink()
    return 0


if __name__ == "__main__":
    sys.exit(main(Path(sys.argv[1]) if len(sys.argv) > 1 else ROOT / "tests" / "golden" / "records"))
