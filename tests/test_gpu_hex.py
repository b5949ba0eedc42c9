"""Fused hex trace+bin kernel on the GPU vs the pinned CPU oracle, same seeds.

FP64 path: cell masses within the reference's own GPU-vs-CPU histogram tolerance
(2e-11 relative, hex_phase/tests/phase_cuda_tests.cpp:70-107), identical ray and exit
counts and status histograms, energy balance to 1e-12.
FP32 path (the fast path): total-variation distance of normalised cell mass
<= 1e-3 against the same-seed FP64 oracle; power is carried in exact fixed point, so the
energy balance holds to binary64 rounding (1e-12) as in the reference's CLI test.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, TWO_ORIENTATIONS

pytestmark = pytest.mark.gpu
COLUMN_KI = (0.8660254037844387, -0.5, 0.0)


def _tv(a, b):
    return 0.5 * np.abs(a / a.sum() - b / b.sum()).sum()


def _accumulate(ctx, icp, plan, R, L, ki, n, nt, np_, precision, hits=1024, tail=1e-12, tuning=None):
    grid = icp.make_phase_grid(nt, np_, ki)
    acc = icp.PhaseMassAccumulatorCuda(ctx, grid)
    for node in plan.nodes:
        acc.add_hex_node((R, L), node.quaternion, node.weight, node.samples, node.seed, n, max_internal_hits=hits,
                         tail_tolerance=tail, precision=precision, tuning=tuning)
    return acc


def test_fp64_matches_reference_masses(ctx, icp):
    g = np.load(GOLDEN / "hex_two_orientations.npz")
    plan = icp.parse_orientation_plan(TWO_ORIENTATIONS)
    acc = _accumulate(ctx, icp, plan, 0.1, 0.2, (1, -0.4, 0.3), 1.31, 72, 144, icp.ICP_FP64)
    m = acc.masses()
    ref = g["masses"]
    assert np.abs(m - ref).sum() / ref.sum() <= 2e-11
    assert np.array_equal(m > 0, ref > 0)
    s = acc.stats
    c = g["counts"]
    assert s.rays == c[3] and s.outputs == c[2]
    assert [s.status_counts[i] for i in range(8)] == [int(x) for x in c[4:12]]
    d = g["stats"]
    assert abs(acc.escaped_area / d[5] - 1) <= 1e-12
    assert abs(acc.unresolved_area - d[6]) <= 1e-12 * d[4]
    assert abs(acc.forward - d[2]) <= 1e-12 * d[4]


def test_fp64_hex_column_sparse(ctx, icp):
    g = np.load(GOLDEN / "hex_column_20k.npz")
    plan = icp.parse_orientation_plan("qw,qx,qy,qz,weight,samples,seed\n1,0,0,0,1,20000,12345\n")
    acc = _accumulate(ctx, icp, plan, 0.05, 0.2, COLUMN_KI, 1.31, 512, 1024, icp.ICP_FP64, hits=12)
    m = acc.masses()
    ref = np.zeros_like(m)
    ref[g["index"]] = g["value"]
    assert np.abs(m - ref).sum() / ref.sum() <= 2e-11
    assert abs(acc.escaped_area / g["stats"][5] - 1) <= 1e-12
    assert abs(acc.unresolved_area / g["stats"][6] - 1) <= 1e-10


@pytest.mark.parametrize("hash_slots", [0, 1, 64])
def test_fp32_tv_against_oracle(ctx, icp, oracle, hash_slots):
    # the hex column (circumradius 0.05 mm, length 0.2 mm), 2e5 rays, 12 interactions (unresolved residual reported, not dropped)
    n = 200_000
    text = f"qw,qx,qy,qz,weight,samples,seed\n1,0,0,0,1,{n},12345\n"
    plan = icp.parse_orientation_plan(text)
    tuning = icp.Tuning(0, 0, hash_slots, 0)
    acc = _accumulate(ctx, icp, plan, 0.05, 0.2, COLUMN_KI, 1.31, 512, 1024, icp.ICP_FP32, hits=12, tuning=tuning)
    rec = oracle.hex_record(0.05, 0.2, COLUMN_KI, 1.31, 1.0, 512, 1024, oracle.parse_plan(text), max_hits=12)
    tv = _tv(acc.masses(), rec.masses)
    assert tv <= 1e-3, tv
    area = rec.expected_area
    # binary32 physics, exact fixed-point power bookkeeping: energy balance to binary64 rounding
    assert abs((acc.escaped_area + acc.unresolved_area) / area - 1) <= 1e-12
    assert acc.stats.max_ray_balance == 0.0
    assert abs(acc.escaped_area / rec.escaped_area - 1) <= 1e-5
    assert acc.stats.rays == n


def test_fp32_two_orientations(ctx, icp, oracle):
    plan = icp.parse_orientation_plan(TWO_ORIENTATIONS)
    acc = _accumulate(ctx, icp, plan, 0.1, 0.2, (1, -0.4, 0.3), 1.31, 72, 144, icp.ICP_FP32)
    g = np.load(GOLDEN / "hex_two_orientations.npz")
    assert _tv(acc.masses(), g["masses"]) <= 1e-3
    assert abs((acc.escaped_area + acc.unresolved_area) / g["stats"][4] - 1) <= 1e-12


def test_record_entry_fp64_matches_oracle_record(ctx, icp, oracle):
    plan = icp.parse_orientation_plan(TWO_ORIENTATIONS)
    out = icp.generate_hex_record(ctx, 0.1, 0.2, (1, -0.4, 0.3), 1.31, 72, 144, plan, 36, 72, precision=icp.ICP_FP64,
                                  batch_size=512)
    g = np.load(GOLDEN / "hex_two_orientations.npz")
    p_gpu = np.diff(out.phi)[:, None] * np.diff(out.theta, axis=1)
    p_ref = np.diff(g["phi"])[:, None] * np.diff(g["theta"], axis=1)
    assert np.abs(p_gpu - p_ref).sum() <= 2e-10
    assert np.array_equal(out.u_edges, g["u"])
    rep = out.report
    assert abs(rep.cdf.g_stored - g["meta"][0]) <= 2e-11
    assert abs((rep.escaped_area_mm2 + rep.unresolved_area_mm2) / rep.expected_area_mm2 - 1) <= 1e-12
    assert rep.histogram_relative_error <= 1e-10
    assert rep.expected_area_mm2 == g["meta"][5]


def test_batch_partition_invariance(ctx, icp):
    plan = icp.parse_orientation_plan(TWO_ORIENTATIONS)
    a = icp.generate_hex_record(ctx, 0.1, 0.2, (1, -0.4, 0.3), 1.31, 72, 144, plan, 36, 72, batch_size=512)
    b = icp.generate_hex_record(ctx, 0.1, 0.2, (1, -0.4, 0.3), 1.31, 72, 144, plan, 36, 72, batch_size=31)
    pa = np.diff(a.phi)[:, None] * np.diff(a.theta, axis=1)
    pb = np.diff(b.phi)[:, None] * np.diff(b.theta, axis=1)
    assert np.abs(pa - pb).sum() < 1e-10


def test_capacity_and_truncation_gates(ctx, icp):
    plan = icp.parse_orientation_plan(TWO_ORIENTATIONS)
    with pytest.raises(icp.CapacityError):
        icp.generate_hex_record(ctx, 0.1, 0.2, (1, -0.4, 0.3), 1.31, 72, 144, plan, 36, 72, max_output_records=1)
    # one interaction: large unresolved residual is reported, never renormalised away
    r = icp.generate_hex_record(ctx, 0.1, 0.2, (1, -0.4, 0.3), 1.31, 72, 144, plan, 36, 72, max_internal_hits=1)
    assert r.report.unresolved_area_mm2 / r.report.expected_area_mm2 > 1e-3
    assert r.report.trace.status_counts[2] > 0


def test_transparent_limit_forward_cap(ctx, icp):
    text = ("qw,qx,qy,qz,weight,samples,seed\n1,0,0,0,0.5,1700,11\n"
            "0.7071067811865476,0,0,0.7071067811865476,0.5,5500,22\n")
    for prec in (icp.ICP_FP64, icp.ICP_FP32):
        out = icp.generate_hex_record(ctx, 0.1, 0.2, (1, -0.4, 0.3), 1.0, 72, 144, icp.parse_orientation_plan(text),
                                      36, 72, tail_tolerance=0.0, precision=prec)
        p = np.diff(out.phi)[:, None] * np.diff(out.theta, axis=1)
        assert np.abs(p[:, 0] - 1 / 72).max() < 1e-13
        assert np.abs(p[:, 1:]).max() == 0
        assert abs(out.report.cdf.g_stored - (1 - out.u_edges[1])) < 1e-12


def test_fp32_full_size_energy(ctx, icp):
    # 1e7 rays of the 1e8-ray config (512 x 1024, 12 interactions): size-independent properties
    plan = icp.parse_orientation_plan("qw,qx,qy,qz,weight,samples,seed\n1,0,0,0,1,10000000,12345\n")
    out = icp.generate_hex_record(ctx, 0.05, 0.2, COLUMN_KI, 1.31, 512, 1024, plan, max_internal_hits=12)
    rep = out.report
    assert abs((rep.escaped_area_mm2 + rep.unresolved_area_mm2) / rep.expected_area_mm2 - 1) <= 1e-12
    assert rep.histogram_relative_error <= 1e-10
    assert rep.trace.rays == 10_000_000 and rep.trace.invalid == 0
    assert np.all(np.diff(out.theta, axis=1) >= 0) and abs(rep.cdf.cdf_mass - 1) <= 1e-10
