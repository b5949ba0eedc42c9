"""The CPU oracle is pinned to the reference before it is trusted as a checker.

Fixtures in tests/golden/ were produced by the reference's own code compiled from its
sources (tests/golden/make_golden.py); where oracle/_ref is built on this host the oracle is
also compared with freshly run reference binaries.  Known-answer cases follow the
reference's hex_phase/tests/phase_tests.cpp and phase_cli_test.py.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import GOLDEN, TWO_ORIENTATIONS

COLUMN_KI = (0.8660254037844387, -0.5, 0.0)


def test_rng_midpoints(oracle):
    # 52-bit midpoints strictly inside (0,1) (hex_trace/include/ice_crystal/math.hpp:142-146)
    u = [oracle.sample_uniform(12345, i, d) for i in range(200) for d in range(3)]
    assert all(0 < x < 1 for x in u)
    assert all((x * 2.0**52 - 0.5) == int(x * 2.0**52 - 0.5) for x in u)


def test_two_orientation_masses_bit_exact(oracle):
    g = np.load(GOLDEN / "hex_two_orientations.npz")
    rec = oracle.hex_record(0.1, 0.2, [1, -0.4, 0.3], 1.31, 1.0, 72, 144, oracle.parse_plan(TWO_ORIENTATIONS),
                            batch=512)
    assert np.array_equal(rec.masses, g["masses"])
    d = g["stats"]
    assert (rec.point_mass, rec.point_axial, rec.forward, rec.backward) == tuple(d[:4])
    assert (rec.expected_area, rec.escaped_area, rec.unresolved_area) == tuple(d[4:7])
    c = g["counts"]
    assert rec.counts["outputs"] == c[2] and rec.counts["rays"] == c[3]
    assert [rec.counts[f"status{i}"] for i in range(8)] == list(c[4:12])


def test_two_orientation_cdf_bit_exact(oracle):
    g = np.load(GOLDEN / "hex_two_orientations.npz")
    cdf = oracle.build_cdf(g["masses"], 72, 144, 36, 72)
    assert cdf.report["status"] == 0
    assert np.array_equal(cdf.phi, g["phi"])
    assert np.array_equal(cdf.theta, g["theta"])
    assert np.array_equal(cdf.edges, g["u"])
    meta = g["meta"]
    assert cdf.report["g_stored"] == meta[0]
    assert cdf.report["l1_error"] == meta[1]
    assert cdf.report["coarsening_tv"] == meta[2]


def test_hex_column_masses_bit_exact(oracle):
    g = np.load(GOLDEN / "hex_column_20k.npz")
    nodes = oracle.parse_plan("qw,qx,qy,qz,weight,samples,seed\n1,0,0,0,1,20000,12345\n")
    rec = oracle.hex_record(0.05, 0.2, COLUMN_KI, 1.31, 1.0, 512, 1024, nodes, max_hits=12)
    nz = np.flatnonzero(rec.masses)
    assert np.array_equal(nz, g["index"])
    assert np.array_equal(rec.masses[nz], g["value"])
    assert rec.escaped_area == g["stats"][5] and rec.unresolved_area == g["stats"][6]


def test_per_ray_trace_bit_exact(oracle):
    g = np.load(GOLDEN / "hex_rays.npz")
    info, exits = oracle.hex_trace_rays(0.05, 0.2, COLUMN_KI, 1.31, 1.0, 12345, 20000, 1024, 1e-12, 100, 48)
    assert np.array_equal(info[:, :4], g["info"][:, :4])
    assert np.array_equal(info[:, 4], g["info"][:, 4])
    flat = np.concatenate([exits[i, :int(info[i, 1])] for i in range(48)])
    assert np.array_equal(flat, g["exits"])


def test_uniform_measure_contract(oracle):
    # phase_tests.cpp:57-70: per-solid-angle uniform masses -> u-edge conditionals, g = 0
    nt, np_ = 64, 128
    e = oracle.u_edges(nt)
    m = np.repeat((4 * math.pi / np_) * np.diff(e), np_)
    c = oracle.build_cdf(m, nt, np_)
    assert abs(c.report["g_stored"]) <= 1e-15
    assert np.abs(c.phi - np.arange(np_ + 1) / np_).max() <= 1e-14
    assert np.abs(c.theta - e[None, :]).max() <= 2e-15


def test_sparse_coarsening_and_zero_columns(oracle):
    # phase_tests.cpp:105-127
    nt, np_ = 48, 96
    i, j = np.meshgrid(np.arange(nt), np.arange(np_), indexing="ij")
    m = np.where(j % 7 == 0, 10.0 ** (-12.0 * ((17 * i + 13 * j) % 97) / 96), 0.0).reshape(-1)
    c = oracle.build_cdf(m, nt, np_, 24, 48)
    assert c.report["status"] == 0 and abs(c.report["cdf_mass"] - 1) <= 2e-15 and c.report["l1_error"] < 2e-14
    full = oracle.build_cdf(m, nt, np_)
    e = oracle.u_edges(nt)
    for col in range(np_):
        if col % 7:
            assert np.array_equal(full.theta[col], e)
    assert oracle.build_cdf(m, nt, np_, 24, 48, max_tv=0).report["status"] != 0
    assert oracle.build_cdf(np.zeros(nt * np_), nt, np_).report["status"] != 0
    bad = m.copy()
    bad[0] = -1
    assert oracle.build_cdf(bad, nt, np_).report["status"] != 0
    # lost mass is detected, never repaired
    assert oracle.build_cdf(np.array([1, 1e-20, 1e-20, 1e-20]), 2, 2, max_lost=0).report["status"] != 0


def test_pole_caps(oracle):
    # phase_tests.cpp:71-77: forward mass 3, backward 1 spread over the end rows
    nt, np_ = 8, 16
    m = np.zeros(nt * np_)
    m[:np_] += 3 / np_
    m[-np_:] += 1 / np_
    c = oracle.build_cdf(m, nt, np_)
    e = oracle.u_edges(nt)
    assert abs(c.report["g_stored"] - 0.5 * (1 - e[1])) <= 5e-16
    assert np.abs(c.phi - np.arange(np_ + 1) / np_).max() <= 1e-15


def test_transparent_limit(oracle):
    # n = 1: all light in the forward cap (phase_tests.cpp:172-182)
    nodes = oracle.parse_plan("qw,qx,qy,qz,weight,samples,seed\n1,0,0,0,0.5,17,11\n"
                              "0.7071067811865476,0,0,0.7071067811865476,0.5,55,22\n")
    rec = oracle.hex_record(1, 2, [0, -1, 0], 1.0, 1.0, 16, 32, nodes, tail=0)
    assert abs(rec.expected_area - 0.5 * ((3 * math.sqrt(3) / 2) + 4)) <= 2e-15
    assert abs(rec.escaped_area - rec.expected_area) <= 4e-15
    assert abs(rec.forward - rec.expected_area) <= 4e-15


@pytest.mark.skipif(not (GOLDEN.parents[1] / "oracle" / "_ref" / "ref_hex_harness").exists(),
                    reason="reference binaries not built on this host")
@pytest.mark.parametrize("ki,R,L,n,hits", [((1, -0.4, 0.3), 0.1, 0.2, 1.31, 1024), ((0.2, 0.9, -0.1), 0.07, 0.05, 1.5, 40),
                                           ((-1, 0, 0), 0.1, 0.3, 1.33, 1024)])
def test_oracle_matches_reference_binary(oracle, tmp_path, ki, R, L, n, hits):
    plan = "qw,qx,qy,qz,weight,samples,seed\n1,0,0,0,0.3,700,7\n0.5,0.5,0.5,0.5,0.7,900,99\n"
    (tmp_path / "p.csv").write_text(plan)
    m, d, _ = oracle.ref_masses(R, L, ki, n, 1.0, 24, 48, tmp_path / "p.csv", max_hits=hits, batch=333,
                                workdir=tmp_path)
    rec = oracle.hex_record(R, L, ki, n, 1.0, 24, 48, oracle.parse_plan(plan), max_hits=hits, batch=333)
    assert np.array_equal(m, rec.masses)
    assert rec.escaped_area == d[5] and rec.unresolved_area == d[6]


def _measure(oracle, edges, mass):
    out = np.zeros(2)
    nt, np_ = mass.shape
    e = np.ascontiguousarray(edges, dtype=np.float64)
    m = np.ascontiguousarray(mass, dtype=np.float64)
    assert oracle.lib().icpo_measure_mass(oracle._p(e), nt, np_, oracle._p(m), oracle._p(out)) == 0
    return out


def test_cell_moment_known_answers(oracle):
    """The saved-CDF first moment (tests/test_phase_storage_cpu.cpp:98-120): the mean cosine of a
    u band is 1 - (u_lo + u_hi); a uniform sphere has g = 0 to 5e-16 on every saved grid, and the
    two-column CDF of the reference's test has g = -0.40125 to 2e-16."""
    for nt in (1, 2, 17, 900, 1800):
        e = oracle.u_edges(nt)
        total, axial = _measure(oracle, e, np.diff(e)[:, None] * np.ones((1, 3)) / 3)
        assert abs(total - 1) < 4e-16 and abs(axial / total) < 5e-16
    phi = [0, .25, 1]
    c = [[0, .1, .5, 1], [0, 0, .25, 1]]
    e = np.array([0, .1, .7, 1])
    mass = np.array([[(phi[j + 1] - phi[j]) * (c[j][i + 1] - c[j][i]) for j in range(2)] for i in range(3)])
    total, axial = _measure(oracle, e, mass)
    assert abs(total - 1) < 2e-16 and abs(axial / total - (-0.40125)) < 2e-16


def _long_tir_case(oracle):
    """The reference's long total-internal-reflection ray: condition 157 of its direction/aspect
    sweep, sample 93 (hex_trace/tests/hex_trace_tests.cpp:282-300)."""
    k = [2 * oracle.sample_uniform(119, 157, d) - 1 for d in range(3)]
    length = 0.2 + 5 * oracle.sample_uniform(127, 157, 0)
    return k, length


def test_long_tir_known_answer(oracle):
    """At 256 interactions the ray stops at the cap with more than 98 % of its power unresolved;
    at 1024 it resolves (residual < 1e-12, balance 1e-10)."""
    k, length = _long_tir_case(oracle)
    info, _ = oracle.hex_trace_rays(1.0, length, k, 1.31, 1.0, 857, 100, 256, 1e-12, 93, 1)
    status, outputs, escaped, unresolved, hits, _ = info[0]
    assert status == 2 and hits == 256 and unresolved > 0.98
    info, _ = oracle.hex_trace_rays(1.0, length, k, 1.31, 1.0, 857, 100, 1024, 1e-12, 93, 1)
    status, outputs, escaped, unresolved, hits, _ = info[0]
    assert status in (0, 1) and hits > 256 and unresolved < 1e-12 and abs(escaped + unresolved - 1) < 1e-10


def _sweep_case(oracle, condition):
    k = [2 * oracle.sample_uniform(119, condition, d) - 1 for d in range(3)]
    return k, 0.2 + 5 * oracle.sample_uniform(127, condition, 0)


def test_direction_aspect_sweep(oracle):
    """300 random directions and aspect ratios, 100 rays each, every ray accepted with balance
    below 1e-10 and total internal reflection exercised (hex_trace/tests/hex_trace_tests.cpp:253-281)."""
    worst, tir_rays = 0.0, 0
    for condition in range(300):
        k, length = _sweep_case(oracle, condition)
        info, _ = oracle.hex_trace_rays(1.0, length, k, 1.31, 1.0, condition + 700, 100, 1024, 1e-12, 0, 100)
        assert np.all((info[:, 0] == 0) | (info[:, 0] == 1)), condition
        bal = np.abs(info[:, 2] + info[:, 3] - 1)
        worst = max(worst, float(bal.max()))
        tir_rays += int((info[:, 4] > 3).sum())
    assert worst < 1e-10 and tir_rays > 0


def test_scale_invariance(oracle):
    """Scaling the prism leaves every exit's direction and power unchanged
    (hex_trace/tests/hex_trace_tests.cpp:241-251)."""
    k = [1, -0.4, 0.3]
    base, ex0 = oracle.hex_trace_rays(0.1, 0.2, k, 1.31, 1.0, 43, 100, 1024, 1e-12, 0, 100)
    for scale in (1e-6, 1e6):
        info, ex = oracle.hex_trace_rays(0.1 * scale, 0.2 * scale, k, 1.31, 1.0, 43, 100, 1024, 1e-12, 0, 100)
        assert np.array_equal(info[:, 1], base[:, 1])
        assert np.allclose(ex, ex0, rtol=0, atol=1e-12)
