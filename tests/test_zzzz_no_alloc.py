"""The static-scratch CDF entry (icp_phase_cdf_build_static) against the regular one.

That entry exists for callers that cannot allocate device memory (their own allocator owns
the device, or allocation is not allowed where they call from): it takes its scratch from a
file-scope device array instead of cudaMalloc.  Its results must equal those of
icp_phase_cdf_build bit for bit (the tolerance the CDF parity tests use for phi and theta),
including on a second call that finds the previous call's contents still in the array.
Collected last so that a run stopping at the first failure has run every other test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(icp):
    f = icp.LIB.icp_phase_cdf_build_static
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_uint32,
                  C.c_uint32, C.POINTER(icp.CdfPolicy), C.c_void_p, C.c_void_p, C.POINTER(icp.CdfReport)]
    return f


def _regular(icp, ctx, dvals, nt, np_, ct, cp, fwd, bwd):
    phi, theta = icp.DeviceArray(ctx, cp + 1), icp.DeviceArray(ctx, cp * (ct + 1))
    rep = icp.CdfReport()
    icp.check(icp.LIB.icp_phase_cdf_build(ctx.handle, dvals.ptr, 0, nt, np_, fwd, bwd, ct, cp,
                                          C.byref(icp.CdfPolicy(1e-10, 1e-12, 1.0)), phi.ptr, theta.ptr, C.byref(rep)))
    return phi.download(), theta.download(), rep


def _static(icp, ctx, fn, stream, dvals, nt, np_, ct, cp, fwd, bwd):
    phi, theta = icp.DeviceArray(ctx, cp + 1), icp.DeviceArray(ctx, cp * (ct + 1))
    rep = icp.CdfReport()
    icp.check(fn(stream, dvals.ptr, 0, nt, np_, fwd, bwd, ct, cp, C.byref(icp.CdfPolicy(1e-10, 1e-12, 1.0)), phi.ptr,
                 theta.ptr, C.byref(rep)))
    return phi.download(), theta.download(), rep


def test_static_scratch_entry_matches_regular_entry_twice():
    import ice_crystal_phase_b200 as icp

    fn = _bind(icp)
    rng = np.random.default_rng(2024)
    with icp.Context(0) as ctx:
        cases = [(96, 192, 48, 64, 3.0, 1.0), (512, 1024, 512, 1024, 0.0, 0.0)]
        streams = [None, icp.LIB.icp_context_stream(ctx.handle)]
        for (nt, np_, ct, cp, fwd, bwd), stream in zip(cases, streams):
            m = rng.exponential(size=nt * np_) * (rng.random(nt * np_) < 0.6)
            d = icp.DeviceArray(ctx, nt * np_).upload(m)
            a_phi, a_theta, a_rep = _regular(icp, ctx, d, nt, np_, ct, cp, fwd, bwd)
            b_phi, b_theta, b_rep = _static(icp, ctx, fn, stream, d, nt, np_, ct, cp, fwd, bwd)
            assert np.array_equal(a_phi, b_phi)
            assert np.array_equal(a_theta, b_theta)
            assert abs(a_rep.g_stored - b_rep.g_stored) <= 2e-11
            assert abs(a_rep.l1_error - b_rep.l1_error) <= 2e-10
            assert b_rep.status == 0 and b_rep.lost_cells == a_rep.lost_cells


def test_static_scratch_rejects_sizes_beyond_its_maximum():
    import ice_crystal_phase_b200 as icp

    fn = _bind(icp)
    with icp.Context(0) as ctx:
        nt, np_ = 4097 * 2, 2
        d = icp.DeviceArray(ctx, nt * np_).upload(np.ones(nt * np_))
        phi, theta = icp.DeviceArray(ctx, np_ + 1), icp.DeviceArray(ctx, np_ * (nt + 1))
        rep = icp.CdfReport()
        rc = fn(None, d.ptr, 0, nt, np_, 0.0, 0.0, nt, np_, C.byref(icp.CdfPolicy(1e-10, 1e-12, 1.0)), phi.ptr, theta.ptr,
                C.byref(rep))
        assert rc == icp.ICP_ERR_CAPACITY
        assert "static scratch maximum" in icp.last_error()
