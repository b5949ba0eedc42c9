"""Fused drop trace+bin kernel on the GPU vs the CPU oracle (the FP64 restatement pinned to the
reference's four-family tracer in test_oracle_drop.py), same seeds and sampling disk.

FP64 path: cell masses within 2e-11 relative L1 (the reference's own GPU-vs-CPU histogram bar,
hex_phase/tests/phase_cuda_tests.cpp:70-107), identical ray / miss / exit counts and status
histograms, energy to 1e-12 -- for chains of up to 30 interactions.  A non-spherical drop is a
chaotic billiard: rays trapped by total internal reflection for hundreds of bounces amplify
ulp-level differences between two correct root finders exponentially, so at the 1024-interaction
default those few rays (~1e-3 of them) exit in different cells and the full chain is compared
statistically (same counts up to the trapped rays, TV bounded by their power).
FP32 path: total variation <= 1e-3 against the same-seed FP64 oracle; power in exact fixed
point, so escaped + residual equals the incident hit area to binary64 rounding (1e-12).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_WATER_700 = 1.3318  # an interior index near water's at 700 nm


def _tv(a, b):
    return 0.5 * np.abs(a / a.sum() - b / b.sum()).sum()


def _shape(icp, radius, sphere=False):
    return icp.RaindropShape.make(radius, sphere).coefficients


def _gpu(ctx, icp, coeff, radius, n, nt, np_, rays, seed, prec, incl=20.0, hits=1024, tail=1e-12, tuning=None,
         pieces=1):
    grid = icp.make_drop_grid(nt, np_, incl)
    acc = icp.PhaseMassAccumulatorCuda(ctx, grid)
    step = (rays + pieces - 1) // pieces
    for first in range(0, rays, step):
        acc.add_drop(coeff, radius, n, rays, seed, incl, max_internal_hits=hits, tail_tolerance=tail, precision=prec,
                     first=first, count=min(step, rays - first), tuning=tuning)
    return acc


def _oracle(oracle, icp, coeff, radius, n, nt, np_, rays, seed, incl=20.0, hits=1024, tail=1e-12):
    geo = oracle.drop_geometry(coeff, radius)
    frame = np.array(icp.drop_frame(incl))
    return oracle.drop_record(geo, frame, n, nt, np_, rays, seed, max_hits=hits, tail=tail)


@pytest.mark.parametrize("radius,sphere,hits", [(0.3, False, 1024), (1.5, True, 1024), (1.5, False, 30),
                                               (3.0, False, 30), (2.2, False, 3)])
def test_fp64_matches_oracle(ctx, icp, oracle, radius, sphere, hits):
    coeff = _shape(icp, radius, sphere)
    acc = _gpu(ctx, icp, coeff, radius, N_WATER_700, 72, 144, 20000, 4242, icp.ICP_FP64, hits=hits)
    rec = _oracle(oracle, icp, coeff, radius, N_WATER_700, 72, 144, 20000, 4242, hits=hits)
    m = acc.masses()
    assert np.abs(m - rec.masses).sum() / rec.masses.sum() <= 2e-11
    assert np.array_equal(m > 0, rec.masses > 0)
    s = acc.stats
    assert s.rays == rec.counts["rays"] and s.missed == rec.counts["missed"]
    assert s.outputs == rec.counts["outputs"] and s.encounters == rec.counts["encounters"]
    assert [s.status_counts[i] for i in range(8)] == [rec.counts[f"status{i}"] for i in range(8)]
    assert abs(acc.escaped_area / rec.escaped_area - 1) <= 1e-12
    assert abs(acc.unresolved_area - rec.unresolved_area) <= 1e-12 * rec.incident_area
    assert abs(acc.incident_area - rec.incident_area) <= 1e-15 * rec.incident_area
    assert abs((acc.escaped_area + acc.unresolved_area) / acc.incident_area - 1) <= 1e-12


@pytest.mark.parametrize("radius", [1.5, 3.0])
def test_fp64_full_chain_statistics(ctx, icp, oracle, radius):
    coeff = _shape(icp, radius)
    acc = _gpu(ctx, icp, coeff, radius, N_WATER_700, 72, 144, 20000, 4242, icp.ICP_FP64)
    rec = _oracle(oracle, icp, coeff, radius, N_WATER_700, 72, 144, 20000, 4242)
    s = acc.stats
    trapped = rec.counts["status2"]  # rays that reach the interaction limit
    assert 0 < trapped < 1e-3 * 20000
    assert s.missed == rec.counts["missed"] and s.rays == rec.counts["rays"]
    assert abs(int(s.status_counts[2]) - trapped) <= trapped and abs(int(s.outputs) - rec.counts["outputs"]) <= 64
    assert _tv(acc.masses(), rec.masses) <= 5e-3
    assert abs((acc.escaped_area + acc.unresolved_area) / acc.incident_area - 1) <= 1e-12


@pytest.mark.parametrize("hash_slots", [0, 1])
def test_fp32_tv_against_oracle(ctx, icp, oracle, hash_slots):
    # the 1.5 mm Table-I drop at 180 x 360 cells, 2e5 rays, 10 internal reflections
    coeff = _shape(icp, 1.5)
    n = 200_000
    acc = _gpu(ctx, icp, coeff, 1.5, N_WATER_700, 180, 360, n, 12345, icp.ICP_FP32, hits=10,
               tuning=icp.Tuning(0, 0, hash_slots, 0))
    rec = _oracle(oracle, icp, coeff, 1.5, N_WATER_700, 180, 360, n, 12345, hits=10)
    tv = _tv(acc.masses(), rec.masses)
    assert tv <= 1e-3, tv
    assert abs((acc.escaped_area + acc.unresolved_area) / acc.incident_area - 1) <= 1e-12
    assert acc.stats.max_ray_balance == 0.0
    assert abs(acc.escaped_area / rec.escaped_area - 1) <= 1e-5
    assert abs(acc.stats.missed - rec.counts["missed"]) <= 5
    assert acc.stats.rays == n


def test_ray_range_partition_invariance(ctx, icp):
    coeff = _shape(icp, 2.0)
    a = _gpu(ctx, icp, coeff, 2.0, N_WATER_700, 72, 144, 30000, 9, icp.ICP_FP64)
    b = _gpu(ctx, icp, coeff, 2.0, N_WATER_700, 72, 144, 30000, 9, icp.ICP_FP64, pieces=7)
    ma, mb = a.masses(), b.masses()
    assert np.abs(ma - mb).sum() <= 1e-13 * ma.sum()
    assert a.stats.outputs == b.stats.outputs and a.stats.missed == b.stats.missed


def test_transparent_limit_all_forward(ctx, icp):
    for prec in (icp.ICP_FP64, icp.ICP_FP32):
        acc = _gpu(ctx, icp, _shape(icp, 1.0), 1.0, 1.0, 36, 72, 5000, 3, prec, tail=0.0)
        assert abs(acc.forward / acc.incident_area - 1) <= 1e-12
        assert np.abs(acc.cell_mass()).max() == 0


def test_record_entry_fp64_matches_oracle_cdf(ctx, icp, oracle):
    coeff = _shape(icp, 1.5)
    out = icp.generate_drop_record(ctx, coeff, 1.5, N_WATER_700, 72, 144, 20000, seed=4242, ct=36, cp=72,
                                   precision=icp.ICP_FP64, max_internal_hits=30)
    rec = _oracle(oracle, icp, coeff, 1.5, N_WATER_700, 72, 144, 20000, 4242, hits=30)
    cdf = oracle.build_cdf(rec.masses, 72, 144, 36, 72)
    p_gpu = np.diff(out.phi)[:, None] * np.diff(out.theta, axis=1)
    p_ref = np.diff(cdf.phi)[:, None] * np.diff(cdf.theta, axis=1)
    assert np.abs(p_gpu - p_ref).sum() <= 2e-10
    assert np.array_equal(out.u_edges, cdf.edges)
    rep = out.report
    assert abs(rep.cdf.g_stored - cdf.report["g_stored"]) <= 2e-11
    assert abs((rep.escaped_area_mm2 + rep.unresolved_area_mm2) / rep.incident_area_mm2 - 1) <= 1e-12
    assert rep.histogram_relative_error <= 1e-10
    assert list(rep.ki) == out.grid.ki and list(rep.e1) == out.grid.e1
    # the sampled hit fraction estimates the CPU projected area
    pr = rep.projected_area_mm2 / rep.sampled_area_mm2
    assert abs(rep.incident_area_mm2 - rep.projected_area_mm2) <= 5 * rep.sampled_area_mm2 * math.sqrt(
        pr * (1 - pr) / 20000)


def test_diffraction_stage(ctx, icp, oracle):
    """Analytic Fraunhofer stage: rows of the circle of equal traced area added to the histogram;
    the stored CDF equals the oracle's CDF of (oracle masses + the same rows)."""
    coeff = _shape(icp, 0.2)
    out = icp.generate_drop_record(ctx, coeff, 0.2, N_WATER_700, 90, 180, 20000, seed=77, precision=icp.ICP_FP64,
                                   wavelength_nm=700.0, diffraction=True)
    rep = out.report
    assert abs(rep.diffraction_area_mm2 / rep.incident_area_mm2 - 1) <= 1e-12
    assert abs(rep.histogram_mass_mm2 / (rep.escaped_area_mm2 + rep.diffraction_area_mm2) - 1) <= 1e-10
    rec = _oracle(oracle, icp, coeff, 0.2, N_WATER_700, 90, 180, 20000, 77)
    rows = icp.diffraction_rows(icp.u_edges(90), rec.incident_area, 700.0)
    m = rec.masses.reshape(90, 180) + rows[:, None] / 180
    cdf = oracle.build_cdf(m.reshape(-1), 90, 180)
    p_gpu = np.diff(out.phi)[:, None] * np.diff(out.theta, axis=1)
    p_ref = np.diff(cdf.phi)[:, None] * np.diff(cdf.theta, axis=1)
    assert np.abs(p_gpu - p_ref).sum() <= 2e-10
    assert rep.cdf.g_stored > cdf.report["g_stored"] - 1e-10 > 0


def test_fp32_full_size_energy(ctx, icp):
    # 1e7 rays of the 1.5 mm drop at 900 x 1800, 10 internal reflections: size-independent properties
    out = icp.generate_drop_record(ctx, _shape(icp, 1.5), 1.5, N_WATER_700, 900, 1800, 10_000_000, seed=2024,
                                   max_internal_hits=10)
    rep = out.report
    assert abs((rep.escaped_area_mm2 + rep.unresolved_area_mm2) / rep.incident_area_mm2 - 1) <= 1e-12
    assert rep.histogram_relative_error <= 1e-10
    assert rep.trace.rays == 10_000_000 and rep.trace.invalid == 0
    assert np.all(np.diff(out.theta, axis=1) >= 0) and abs(rep.cdf.cdf_mass - 1) <= 1e-10
    pr = rep.projected_area_mm2 / rep.sampled_area_mm2
    assert abs(rep.incident_area_mm2 - rep.projected_area_mm2) <= 5 * rep.sampled_area_mm2 * math.sqrt(
        pr * (1 - pr) / 1e7)


def test_invalid_drop_inputs_rejected(ctx, icp):
    with pytest.raises(icp.InvalidArgument):  # nonconvex shape
        icp.generate_drop_record(ctx, [0, 0, 0.5], 1.0, 1.33, 8, 16, 100)
    with pytest.raises(icp.InvalidArgument):  # CDF dims must divide the query dims
        icp.generate_drop_record(ctx, [0.0] * 8, 1.0, 1.33, 9, 16, 100, ct=4)
    with pytest.raises(icp.InvalidArgument):  # diffraction needs a wavelength
        icp.generate_drop_record(ctx, [0.0] * 8, 1.0, 1.33, 8, 16, 100, diffraction=True)


# The record the headline measurement times: an oblate drop of equal-volume radius 1.5 mm with
# r/a = 1 - 0.08 cos(chi) - 0.02 cos(2 chi) + 0.005 cos(3 chi), 650 nm with the water index at
# 20 C held in binary32, inclination 20 deg, at most 10 internal interactions, 900 x 1800 cells,
# seed 12345, 1e8 rays in the record.  Its first ray ids are traced here, exactly the rays the
# timed record starts with (the counter RNG depends only on seed and ray id).
BENCH_COEFF = (0.0, -0.08, -0.02, 0.005, 0.0, 0.0, 0.0, 0.0)
BENCH_RAYS, BENCH_SEED, BENCH_HITS = 100_000_000, 12345, 10


def _bench_index(icp):
    return float(np.float32(icp.evaluate_water_optics(650.0).refractive_index))


def test_benchmark_record_slice_parity(ctx, icp, oracle):
    """FP32 device trace of the benchmark record's first 1e6 ray ids against the FP64 oracle on
    the same ray ids: TV of cell mass <= 1e-3, |g - g_oracle| <= 1e-4, energy balance <= 1e-6 --
    the tolerances the headline metric is quoted at."""
    from oracle import parity

    n_int, count = _bench_index(icp), 1_000_000
    acc = icp.PhaseMassAccumulatorCuda(ctx, icp.make_drop_grid(900, 1800, 20.0))
    acc.add_drop(BENCH_COEFF, 1.5, n_int, BENCH_RAYS, BENCH_SEED, 20.0, max_internal_hits=BENCH_HITS,
                 precision=icp.ICP_FP32, first=0, count=count)
    cfg = {"coefficients": list(BENCH_COEFF), "radius_mm": 1.5, "interior_index": n_int, "inclination_deg": 20.0,
           "nt": 900, "np": 1800, "rays": BENCH_RAYS, "seed": BENCH_SEED, "max_internal_hits": BENCH_HITS, "first": 0,
           "count": count}
    audit = {"escaped": acc.escaped_area, "unresolved": acc.unresolved_area, "incident": acc.incident_area,
             "missed": acc.stats.missed}
    r = parity.drop_parity(acc.masses(), cfg, audit)
    assert acc.stats.rays == count
    assert r["tv"] <= 1e-3, r
    assert r["g_abs_error"] <= 1e-4, r
    assert r["energy_residual_device"] <= 1e-6, r
    assert abs(r["missed_device"] - r["missed_oracle"]) <= 5, r


def test_benchmark_record_stored_cdf_parity(ctx, icp, oracle):
    """The benchmark record's whole pipeline at 1e6 rays (trace, analytic diffraction rows, stored
    CDF) through the host-buffer entry against the oracle's record of the same rays plus the same
    rows through the oracle's CDF build: TV of the stored cell probabilities <= 1e-3 and stored g
    within 1e-4."""
    n_int, rays = _bench_index(icp), 1_000_000
    out = icp.generate_drop_record(ctx, BENCH_COEFF, 1.5, n_int, 900, 1800, rays, seed=BENCH_SEED,
                                   max_internal_hits=BENCH_HITS, wavelength_nm=650.0, diffraction=True)
    rep = out.report
    geo = oracle.drop_geometry(BENCH_COEFF, 1.5)
    rec = oracle.drop_record_sharded(geo, np.array(icp.drop_frame(20.0)), n_int, 900, 1800, rays, BENCH_SEED,
                                     max_hits=BENCH_HITS)
    rows = icp.diffraction_rows(icp.u_edges(900), rec.incident_area, 650.0)
    cdf = oracle.build_cdf((rec.masses.reshape(900, 1800) + rows[:, None] / 1800).reshape(-1), 900, 1800)
    p_gpu = np.diff(out.phi)[:, None] * np.diff(out.theta, axis=1)
    p_ref = np.diff(cdf.phi)[:, None] * np.diff(cdf.theta, axis=1)
    assert 0.5 * np.abs(p_gpu - p_ref).sum() <= 1e-3
    assert abs(rep.cdf.g_stored - cdf.report["g_stored"]) <= 1e-4
    assert abs((rep.escaped_area_mm2 + rep.unresolved_area_mm2) / rep.incident_area_mm2 - 1) <= 1e-6
    assert abs(rep.diffraction_area_mm2 / rep.incident_area_mm2 - 1) <= 1e-12
    assert rep.trace.rays == rays and rep.cdf.status == 0
