"""The static-scratch CDF entry (icp_phase_cdf_build_static) against the regular one.

That entry exists for callers that cannot allocate device memory (their own allocator owns
the device, or allocation is not allowed where they call from): it takes its scratch from a
file-scope device array instead of cudaMalloc.  Its results must equal those of
icp_phase_cdf_build bit for bit (the tolerance the CDF parity tests use for phi and theta),
including on a second call that finds the previous call's contents still in the array, for
mass and density input, and with the same status, message and report when an audit gate
rejects the record.  Collected last so that a run stopping at the first failure has run every
other test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REPORT_FIELDS = ["g_source", "g_stored", "coarsening_tv", "cdf_mass", "l1_error", "lost_mass", "maximum_cell_error",
                 "aggregation_relative_error", "fine_mass", "fine_axial", "lost_cells", "malformed", "status"]


def _bind(icp):
    f = icp.LIB.icp_phase_cdf_build_static
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_uint32,
                  C.c_uint32, C.POINTER(icp.CdfPolicy), C.c_void_p, C.c_void_p, C.POINTER(icp.CdfReport)]
    return f


def _regular(icp, ctx, dvals, kind, nt, np_, ct, cp, fwd, bwd, policy):
    phi, theta = icp.DeviceArray(ctx, cp + 1), icp.DeviceArray(ctx, cp * (ct + 1))
    rep = icp.CdfReport()
    rc = icp.LIB.icp_phase_cdf_build(ctx.handle, dvals.ptr, kind, nt, np_, fwd, bwd, ct, cp, C.byref(policy), phi.ptr,
                                     theta.ptr, C.byref(rep))
    return rc, icp.last_error(), phi.download(), theta.download(), rep


def _static(icp, ctx, fn, stream, dvals, kind, nt, np_, ct, cp, fwd, bwd, policy):
    phi, theta = icp.DeviceArray(ctx, cp + 1), icp.DeviceArray(ctx, cp * (ct + 1))
    rep = icp.CdfReport()
    rc = fn(stream, dvals.ptr, kind, nt, np_, fwd, bwd, ct, cp, C.byref(policy), phi.ptr, theta.ptr, C.byref(rep))
    return rc, icp.last_error(), phi.download(), theta.download(), rep


def _same_report(a, b):
    for k in REPORT_FIELDS:
        assert getattr(a, k) == getattr(b, k), (k, getattr(a, k), getattr(b, k))


def test_static_scratch_entry_matches_regular_entry_twice():
    import ice_crystal_phase_b200 as icp

    fn = _bind(icp)
    rng = np.random.default_rng(2024)
    policy = icp.CdfPolicy(1e-10, 1e-12, 1.0)
    with icp.Context(0) as ctx:
        stream = icp.LIB.icp_context_stream(ctx.handle)
        # (kind, nt, np, ct, cp, fwd, bwd): mass with coarsening and poles, mass at full size,
        # density input -- each built twice in a row through the static entry
        cases = [(0, 96, 192, 48, 64, 3.0, 1.0), (0, 512, 1024, 512, 1024, 0.0, 0.0), (1, 180, 360, 90, 120, 0.0, 0.0)]
        for kind, nt, np_, ct, cp, fwd, bwd in cases:
            m = rng.exponential(size=nt * np_) * (rng.random(nt * np_) < 0.6)
            d = icp.DeviceArray(ctx, nt * np_).upload(m)
            rc_a, _, a_phi, a_theta, a_rep = _regular(icp, ctx, d, kind, nt, np_, ct, cp, fwd, bwd, policy)
            assert rc_a == 0
            for s in (None, stream):
                rc_b, _, b_phi, b_theta, b_rep = _static(icp, ctx, fn, s, d, kind, nt, np_, ct, cp, fwd, bwd, policy)
                assert rc_b == 0
                assert np.array_equal(a_phi, b_phi)
                assert np.array_equal(a_theta, b_theta)
                _same_report(a_rep, b_rep)


def test_static_scratch_entry_rejects_like_regular_entry():
    """A record that an audit gate rejects (an L1 bar below the CDF's own rounding) returns the
    same status, message and report from both entries; the next call through the static entry,
    which finds the rejected call's contents in the array, succeeds again."""
    import ice_crystal_phase_b200 as icp

    fn = _bind(icp)
    rng = np.random.default_rng(7)
    with icp.Context(0) as ctx:
        nt, np_ = 128, 256
        d = icp.DeviceArray(ctx, nt * np_).upload(rng.exponential(size=nt * np_))
        tight = icp.CdfPolicy(1e-30, 1e-12, 1.0)
        rc_a, msg_a, _, _, a_rep = _regular(icp, ctx, d, 0, nt, np_, nt, np_, 0.0, 0.0, tight)
        rc_b, msg_b, _, _, b_rep = _static(icp, ctx, fn, None, d, 0, nt, np_, nt, np_, 0.0, 0.0, tight)
        assert rc_a == rc_b == icp.ICP_ERR_AUDIT
        assert msg_a == msg_b
        _same_report(a_rep, b_rep)
        ok = icp.CdfPolicy(1e-10, 1e-12, 1.0)
        rc_c, _, c_phi, c_theta, _ = _static(icp, ctx, fn, None, d, 0, nt, np_, nt, np_, 0.0, 0.0, ok)
        rc_d, _, d_phi, d_theta, _ = _regular(icp, ctx, d, 0, nt, np_, nt, np_, 0.0, 0.0, ok)
        assert rc_c == rc_d == 0
        assert np.array_equal(c_phi, d_phi) and np.array_equal(c_theta, d_theta)


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
