"""CDF builder on the GPU vs the pinned CPU oracle (same masses in, same arrays out).

The column scans and the marginal scan use the reference's ordered binary64 additions, so
phi and theta are compared bit for bit; reductions (g, L1) are parallel and compared within
the reference's own GPU-vs-CPU tolerances (hex_phase/tests/phase_cuda_tests.cpp:18-47:
L1 2e-10, g 2e-11).  Edge cases follow tests/test_phase_cdf_cuda.cpp:15-71.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _check_same(ctx, icp, oracle, m, nt, np_, ct=None, cp=None, fwd=0.0, bwd=0.0):
    full = m.reshape(nt, np_).copy()
    full[0] += fwd / np_
    full[-1] += bwd / np_
    ref = oracle.build_cdf(full.reshape(-1), nt, np_, ct, cp)
    assert ref.report["status"] == 0
    out = icp.PhaseCdf(ctx).build(m, nt, np_, ct, cp, forward=fwd, backward=bwd)
    if fwd == 0 and bwd == 0:
        assert np.array_equal(out.phi, ref.phi)
        assert np.array_equal(out.theta, ref.theta)
    else:  # pole cap added with one rounding on the device instead of the Kahan pair
        assert np.abs(out.phi - ref.phi).max() <= 1e-15
        assert np.abs(out.theta - ref.theta).max() <= 1e-15
    assert np.array_equal(out.u_edges, ref.edges)
    r = out.report
    assert abs(r["g_stored"] - ref.report["g_stored"]) <= 2e-11
    assert abs(r["l1_error"] - ref.report["l1_error"]) <= 2e-10
    assert abs(r["cdf_mass"] - 1) <= 1e-10
    assert r["lost_cells"] == ref.report["lost_cells"]
    return out, ref


def test_reference_record_masses(ctx, icp, oracle):
    g = np.load(GOLDEN / "hex_two_orientations.npz")
    out, _ = _check_same(ctx, icp, oracle, g["masses"], 72, 144, 36, 72)
    assert np.array_equal(out.phi, g["phi"]) and np.array_equal(out.theta, g["theta"])
    assert abs(out.report["g_stored"] - g["meta"][0]) <= 2e-11


@pytest.mark.parametrize("nt,np_", [(1, 1), (17, 13), (257, 33), (513, 513), (900, 1800), (512, 1024)])
def test_synthetic_densities_with_zero_columns(ctx, icp, oracle, nt, np_):
    rng = np.random.default_rng(nt * 7919 + np_)
    m = rng.random((nt, np_)) ** 3
    m[:, ::5] = 0.0  # empty phi columns -> u-edge conditionals
    m[rng.random((nt, np_)) < 0.2] = 0.0  # plateaus
    if m.sum() == 0:
        m[0, 0] = 1.0
    _check_same(ctx, icp, oracle, m.reshape(-1), nt, np_)


def test_coarsening_and_poles(ctx, icp, oracle):
    rng = np.random.default_rng(3)
    m = rng.random(96 * 192)
    _check_same(ctx, icp, oracle, m, 96, 192, 48, 64)
    _check_same(ctx, icp, oracle, m, 96, 192, 96, 192, fwd=3.0, bwd=1.0)


def test_uniform_contract(ctx, icp, oracle):
    nt, np_ = 64, 128
    e = oracle.u_edges(nt)
    m = np.repeat((4 * math.pi / np_) * np.diff(e), np_)
    out, _ = _check_same(ctx, icp, oracle, m, nt, np_)
    assert abs(out.report["g_stored"]) <= 1e-15
    assert np.abs(out.theta - e[None, :]).max() <= 2e-15


def test_density_input(ctx, icp, oracle):
    # scalar density stage (PhaseDensityView::scalar): w = d * du
    nt, np_ = 36, 72
    e = oracle.u_edges(nt)
    rng = np.random.default_rng(5)
    d = rng.random((nt, np_))
    out = icp.PhaseCdf(ctx).build(d.reshape(-1), nt, np_, density=True)
    ref = oracle.build_cdf((d * np.diff(e)[:, None]).reshape(-1), nt, np_)
    assert np.abs(out.theta - ref.theta).max() <= 1e-15 and np.abs(out.phi - ref.phi).max() <= 1e-15


def test_rejections(ctx, icp):
    cdf = icp.PhaseCdf(ctx)
    m = np.ones(8 * 16)
    bad = m.copy()
    bad[3] = -1
    with pytest.raises(icp.InvalidArgument):
        cdf.build(bad, 8, 16)
    bad[3] = np.nan
    with pytest.raises(icp.InvalidArgument):
        cdf.build(bad, 8, 16)
    with pytest.raises(icp.AuditError):
        cdf.build(np.zeros(8 * 16), 8, 16)
    with pytest.raises(icp.InvalidArgument):
        cdf.build(m, 8, 16, 3, 16)
    with pytest.raises(icp.AuditError):
        cdf.build(np.array([1, 1e-20, 1e-20, 1e-20]), 2, 2, max_lost_mass=0)
    rng = np.random.default_rng(1)
    with pytest.raises(icp.AuditError):
        cdf.build(rng.random(48 * 96), 48, 96, 24, 48, max_coarsening_tv=0)


def test_full_size_properties(ctx, icp):
    # 900 x 1800: monotone conditionals with exact endpoints, normalised marginal, mass 1
    rng = np.random.default_rng(11)
    m = rng.exponential(size=900 * 1800) * (rng.random(900 * 1800) < 0.3)
    out = icp.PhaseCdf(ctx).build(m, 900, 1800)
    t = out.theta
    assert np.all(np.diff(t, axis=1) >= 0) and np.all(t[:, 0] == 0) and np.all(t[:, -1] == 1)
    assert out.phi[0] == 0 and out.phi[-1] == 1 and np.all(np.diff(out.phi) >= 0)
    assert abs(out.report["cdf_mass"] - 1) <= 1e-10


@pytest.mark.parametrize("count,nt,np_,ct,cp", [(5, 72, 144, 36, 72), (100, 256, 512, 64, 128), (3, 900, 1800, 900, 1800),
                                               (7, 256, 512, 256, 512)])
def test_batched_build_equals_single_records(ctx, icp, count, nt, np_, ct, cp):
    """icp_phase_cdf_build_batch (several records per cooperative launch, 16 strips each; 100
    records need two launches) writes the same phi / theta bits as icp_phase_cdf_build per
    record, including records with empty columns and one whose mass is all in the pole rows."""
    import ctypes as C

    import torch

    rng = np.random.default_rng(count + nt)
    m = rng.gamma(0.4, size=(count, nt, np_))
    m[:, :, rng.choice(np_, np_ // 7, replace=False)] = 0.0
    m[0] = 0.0
    m[0, 0] = 1.0
    m[0, -1] = 0.5
    dv = torch.from_numpy(m.reshape(-1).copy()).cuda()
    phi = torch.empty(count * (cp + 1), dtype=torch.float64, device="cuda")
    theta = torch.empty(count * cp * (ct + 1), dtype=torch.float64, device="cuda")
    reps = (icp.CdfReport * count)()
    policy = icp.CdfPolicy(1e-10, 1e-12, 1.0)
    torch.cuda.synchronize()
    icp.check(icp.LIB.icp_phase_cdf_build_batch(ctx.handle, C.c_void_p(dv.data_ptr()), count, nt, np_, ct, cp,
                                                C.byref(policy), C.c_void_p(phi.data_ptr()),
                                                C.c_void_p(theta.data_ptr()), reps))
    bp = phi.cpu().numpy().reshape(count, cp + 1)
    bt = theta.cpu().numpy().reshape(count, cp, ct + 1)
    for r in range(count):
        one = icp.PhaseCdf(ctx).build(m[r].reshape(-1), nt, np_, ct, cp)
        assert np.array_equal(bp[r], one.phi), r
        assert np.array_equal(bt[r], one.theta.reshape(cp, ct + 1)), r
        assert reps[r].status == 0
        assert abs(reps[r].g_stored - one.report["g_stored"]) <= 1e-13
        assert abs(reps[r].l1_error - one.report["l1_error"]) <= 1e-13


def test_enqueue_and_result_equal_the_build(ctx, icp):
    """icp_phase_cdf_enqueue + icp_phase_cdf_result (one kernel on the stream, report later) give
    the bits and report of icp_phase_cdf_build, on repeated builds (the barrier counters are left
    at zero by every completed build) and across grid shapes (the u edges follow nt)."""
    import ctypes as C

    rng = np.random.default_rng(77)
    for nt, np_ in ((900, 1800), (64, 128), (900, 1800)):
        m = rng.exponential(size=nt * np_) * (rng.random(nt * np_) < 0.5)
        ref = icp.PhaseCdf(ctx).build(m, nt, np_)
        d = icp.DeviceArray(ctx, nt * np_).upload(m)
        phi, theta = icp.DeviceArray(ctx, np_ + 1), icp.DeviceArray(ctx, np_ * (nt + 1))
        for _ in range(2):
            icp.check(icp.LIB.icp_phase_cdf_enqueue(ctx.handle, d.ptr, 0, nt, np_, 0.0, 0.0, nt, np_, phi.ptr, theta.ptr))
            rep = icp.CdfReport()
            icp.check(icp.LIB.icp_phase_cdf_result(ctx.handle, C.byref(icp.CdfPolicy(1e-10, 1e-12, 1.0)), C.byref(rep)))
            assert np.array_equal(phi.download(), ref.phi)
            assert np.array_equal(theta.download().reshape(np_, nt + 1), ref.theta)
            assert rep.status == 0 and rep.g_stored == ref.report["g_stored"] and rep.l1_error == ref.report["l1_error"]


def test_grid_barrier_wait_that_runs_out_reports_timeout(ctx, icp):
    """A grid-barrier wait limited to one poll runs out (129 cooperative blocks cannot all arrive
    before the first ones poll): the build ends with ICP_ERR_TIMEOUT, and the same context then
    builds the same record correctly once the default limit is back."""
    rng = np.random.default_rng(12)
    m = rng.exponential(size=900 * 1800)
    ref = icp.PhaseCdf(ctx).build(m, 900, 1800)
    icp.check(icp.LIB.icp_context_set_wait_limit(ctx.handle, 1))
    try:
        with pytest.raises(icp.IcpError) as err:
            icp.PhaseCdf(ctx).build(m, 900, 1800)
        assert err.value.status == icp.ICP_ERR_TIMEOUT
        assert "gave up waiting" in icp.last_error()
    finally:
        icp.check(icp.LIB.icp_context_set_wait_limit(ctx.handle, 0))
    again = icp.PhaseCdf(ctx).build(m, 900, 1800)
    assert np.array_equal(again.phi, ref.phi) and np.array_equal(again.theta, ref.theta)
    assert again.report["status"] == 0


def test_refused_allocation_leaves_the_context_usable(ctx, icp):
    """A device allocation the driver refuses (a petabyte) is reported as ICP_ERR_DEVICE with
    the driver's message; the context then builds a record as before."""
    import ctypes as C

    p = C.c_void_p()
    rc = icp.LIB.icp_device_alloc(ctx.handle, 1 << 50, C.byref(p))
    assert rc == icp.ICP_ERR_DEVICE and not p.value
    assert "cudaMalloc" in icp.last_error()
    rng = np.random.default_rng(4)
    m = rng.random(64 * 128)
    out = icp.PhaseCdf(ctx).build(m, 64, 128)
    assert out.report["status"] == 0 and out.phi[-1] == 1
