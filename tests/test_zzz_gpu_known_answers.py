"""Known answers of the reference's own tracer tests on the device path (sorts after the
record-path GPU suites)."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


def test_long_tir_known_answer_fp64(ctx, icp, oracle):
    """The reference's long total-internal-reflection ray (hex_trace/tests/hex_trace_tests.cpp:282-300)
    through the FP64 trace kernel: stopped at the 256-interaction cap with more than 98 % of its
    power unresolved, resolved at 1024 interactions."""
    from test_oracle_pinned import _long_tir_case

    k, length = _long_tir_case(oracle)
    for hits in (256, 1024):
        acc = icp.PhaseMassAccumulatorCuda(ctx, icp.make_phase_grid(36, 72, k))
        s = acc.add_hex_node((1.0, length), (1.0, 0.0, 0.0, 0.0), 1.0, 100, 857, 1.31, max_internal_hits=hits,
                             precision=icp.ICP_FP64, first=93, count=1)
        assert s.rays == 1
        if hits == 256:
            assert s.status_counts[2] == 1 and s.encounters == 256 and s.unresolved > 0.98
        else:
            assert s.status_counts[0] + s.status_counts[1] == 1 and s.encounters > 256
            assert s.unresolved < 1e-12 and abs(s.escaped + s.unresolved - 1) < 1e-10


def test_direction_aspect_sweep_fp64(ctx, icp, oracle):
    """The reference's direction/aspect sweep on the FP64 trace kernel: every ray accepted, balance
    below 1e-10, TIR exercised, and each condition's escaped power equal to the oracle's
    (hex_trace/tests/hex_trace_tests.cpp:253-281)."""
    from test_oracle_pinned import _sweep_case

    encounters = 0
    for condition in range(300):
        k, length = _sweep_case(oracle, condition)
        acc = icp.PhaseMassAccumulatorCuda(ctx, icp.make_phase_grid(18, 36, k))
        s = acc.add_hex_node((1.0, length), (1.0, 0.0, 0.0, 0.0), 1.0, 100, condition + 700, 1.31,
                             precision=icp.ICP_FP64)
        assert s.rays == 100 and s.status_counts[0] + s.status_counts[1] == 100 and s.rejected_rays == 0
        assert s.max_ray_balance < 1e-10
        info, _ = oracle.hex_trace_rays(1.0, length, k, 1.31, 1.0, condition + 700, 100, 1024, 1e-12, 0, 100)
        assert s.escaped == pytest.approx(info[:, 2].sum(), rel=1e-11)  # 2^-44 fixed point per exit
        assert s.outputs == int(info[:, 1].sum())
        encounters += s.encounters
    assert encounters > 300 * 100 * 3


def test_scale_invariance_fp64(ctx, icp):
    """Scaling the prism by 1e-6 and 1e6 scales every cell mass by the area factor and changes
    nothing else (hex_trace/tests/hex_trace_tests.cpp:241-251)."""
    import numpy as np

    masses = []
    for scale in (1.0, 1e-6, 1e6):
        acc = icp.PhaseMassAccumulatorCuda(ctx, icp.make_phase_grid(36, 72, (1, -0.4, 0.3)))
        acc.add_hex_node((0.1 * scale, 0.2 * scale), (1.0, 0.0, 0.0, 0.0), 1.0, 4096, 43, 1.31,
                         precision=icp.ICP_FP64)
        masses.append(acc.masses() / scale ** 2)
    for m in masses[1:]:
        assert np.array_equal(m > 0, masses[0] > 0)
        assert np.abs(m - masses[0]).sum() / masses[0].sum() < 1e-12
