"""Batched drop records (one persistent launch over a device work queue, optionally a captured
CUDA graph) against the single-record entry: every record keeps its seed and ray ids, so the
FP64 batch reproduces the single-record records up to the order of FP64 histogram additions,
with graph and direct launches identical."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _specs(icp):
    rng = np.random.default_rng(20260101)
    out = []
    for i, (radius, sphere) in enumerate([(0.3, False), (1.5, False), (2.6, False), (1.0, True), (0.8, False)]):
        shape = icp.RaindropShape.make(radius, sphere).coefficients
        lam = float(rng.uniform(400, 700))
        n = float(np.float32(icp.evaluate_water_optics(lam).refractive_index))
        out.append(icp.DropSpec(shape, radius, n, rays=int(rng.integers(20_000, 120_000)), seed=1000 + i,
                                inclination_deg=float(rng.uniform(-90, 90)), wavelength_nm=lam,
                                diffraction=bool(i % 2)))
    return out


def _p(phi, theta):
    return np.diff(phi)[:, None] * np.diff(theta, axis=1)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_equals_single_records(ctx, icp, precision):
    prec = icp.ICP_FP64 if precision == "fp64" else icp.ICP_FP32
    specs = _specs(icp)
    s = icp.batch_settings(72, 144, 36, 72, precision=prec, chunk_rays=4096, use_graph=False)
    out = icp.generate_drop_batch(ctx, specs, s)
    for r, sp in enumerate(specs):
        one = icp.generate_drop_record(ctx, sp.coefficients, sp.radius_mm, sp.interior_index, 72, 144, sp.rays,
                                       seed=sp.seed, inclination_deg=sp.inclination_deg, ct=36, cp=72, precision=prec,
                                       wavelength_nm=sp.wavelength_nm, diffraction=sp.diffraction)
        rep, ref = out.reports[r], one.report
        assert rep.trace.rays == ref.trace.rays
        assert rep.projected_area_mm2 == ref.projected_area_mm2
        assert list(rep.ki) == list(ref.ki)
        d = np.abs(_p(out.phi[r], out.theta[r]) - _p(one.phi, one.theta)).sum()
        if prec == icp.ICP_FP64:
            # the same per-ray arithmetic: identical counts, FP64 summation order only
            assert rep.trace.missed == ref.trace.missed and rep.trace.outputs == ref.trace.outputs
            assert [rep.trace.status_counts[i] for i in range(8)] == [ref.trace.status_counts[i] for i in range(8)]
            assert rep.incident_area_mm2 == ref.incident_area_mm2
            assert abs(rep.escaped_area_mm2 / ref.escaped_area_mm2 - 1) <= 1e-13
            assert abs(rep.diffraction_area_mm2 - ref.diffraction_area_mm2) <= 1e-13 * ref.incident_area_mm2
            assert d <= 1e-11, (r, d)
            assert abs(rep.cdf.g_stored - ref.cdf.g_stored) <= 1e-12
        else:
            # two kernels may contract binary32 products differently
            assert abs(int(rep.trace.missed) - int(ref.trace.missed)) <= 2
            assert 0.5 * d <= 1e-3, (r, d)
            assert abs(rep.cdf.g_stored - ref.cdf.g_stored) <= 1e-4
        assert abs((rep.escaped_area_mm2 + rep.unresolved_area_mm2) / rep.incident_area_mm2 - 1) <= 1e-12
    assert np.array_equal(out.u_edges, icp.u_edges(72)[::2])


def test_graph_replay_matches_direct_launch(ctx, icp):
    specs = _specs(icp)
    direct = icp.generate_drop_batch(ctx, specs, icp.batch_settings(90, 180, precision=icp.ICP_FP64, use_graph=False))
    first = icp.generate_drop_batch(ctx, specs, icp.batch_settings(90, 180, precision=icp.ICP_FP64, use_graph=True))
    again = icp.generate_drop_batch(ctx, specs, icp.batch_settings(90, 180, precision=icp.ICP_FP64, use_graph=True))
    for r in range(len(specs)):
        pd = _p(direct.phi[r], direct.theta[r])
        for other in (first, again):
            assert np.abs(_p(other.phi[r], other.theta[r]) - pd).sum() <= 1e-12
            assert other.reports[r].trace.outputs == direct.reports[r].trace.outputs


def test_uneven_chunks_and_autotune(ctx, icp):
    specs = _specs(icp)
    specs[0].rays, specs[1].rays = 33, 1  # records smaller than one chunk
    s = icp.batch_settings(36, 72, precision=icp.ICP_FP64, chunk_rays=32, use_graph=False)
    a = icp.generate_drop_batch(ctx, specs, s)
    b = icp.generate_drop_batch(ctx, specs, icp.batch_settings(36, 72, precision=icp.ICP_FP64, chunk_rays=1 << 16,
                                                               use_graph=False))
    for r in range(len(specs)):
        assert a.reports[r].trace.rays == specs[r].rays
        assert np.abs(_p(a.phi[r], a.theta[r]) - _p(b.phi[r], b.theta[r])).sum() <= 1e-12
    t = icp.batch_settings(36, 72)
    rate = icp.autotune_drop_batch(ctx, specs, t)
    assert rate > 0 and t.block_threads in (128, 256) and t.chunk_rays in (2048, 8192, 32768)


def test_batch_rejects_invalid_records(ctx, icp):
    specs = _specs(icp)
    specs[2].coefficients = [0, 0, 0.5]
    with pytest.raises(icp.InvalidArgument):
        icp.generate_drop_batch(ctx, specs, icp.batch_settings(36, 72))
    with pytest.raises(icp.InvalidArgument):
        icp.generate_drop_batch(ctx, _specs(icp), icp.batch_settings(36, 72, ct=10))
