"""Test configuration: the `gpu` marker and shared fixtures.

`-m "not gpu"` runs on any host (oracle pins, host logic, ABI surface, gloo ranks);
`-m gpu` needs a B200 and exercises the CUDA path through the C ABI.
"""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def icp():
    import ice_crystal_phase_b200 as I
    return I


@pytest.fixture(scope="session")
def ctx(icp):
    c = icp.Context(0)
    yield c
    c.close()


TWO_ORIENTATIONS = ("qw,qx,qy,qz,weight,samples,seed\n"
                    "1,0,0,0,0.5,1024,12345\n"
                    "0.7071067811865475244,0,0,0.7071067811865475244,0.5,2048,54321\n")
