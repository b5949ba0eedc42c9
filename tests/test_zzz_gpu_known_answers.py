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
