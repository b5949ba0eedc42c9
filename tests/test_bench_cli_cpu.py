"""bench.py's command line: it imports and parses without a GPU, and offers the flags of the
benchmark contract (GPU count, steps, warm-up, implementation arm, workload) and of its legs."""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_bench_help_lists_the_contract_flags():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--help"], capture_output=True, text=True,
                         timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    for flag in ("--gpus", "--steps", "--warmup", "--impl", "--workload", "--rays", "--batch-records",
                 "--surrogate-records", "--surrogate-batch", "--atlas-incidents", "--rainbow-steps", "--wave-steps",
                 "--no-cpu-baseline", "--parity-rays"):
        assert flag in out.stdout, flag
