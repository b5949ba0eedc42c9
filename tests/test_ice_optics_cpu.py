"""Ice Ih refractive index (Warren & Brandt 2008), host material service (no GPU).

Pinned two ways: bit for bit against the reference's evaluate_ice_wb2008
(hex_atlas/src/ice_optics.cpp), run over knots, geometric midpoints, seeded random wavelengths
and domain edges (tests/golden/ice_wb2008.npz, made by tests/golden/make_golden.py), and against
the known answers of the reference's own test (hex_atlas/tests/ice_optics_tests.cpp:14-26).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import GOLDEN


def test_matches_reference_bit_for_bit(icp):
    z = np.load(GOLDEN / "ice_wb2008.npz")
    assert (z["status"] == 0).sum() > 500
    for nm, st, v in zip(z["wavelength_nm"], z["status"], z["values"]):
        if st == 0:
            s = icp.evaluate_ice_optics(float(nm))
            got = (s.n, s.kappa, s.lower_nm, s.upper_nm, s.log_wavelength_fraction)
            assert got == tuple(float(x) for x in v), nm
            assert s.wavelength_nm == float(nm)
        else:  # the reference raised std::invalid_argument
            assert st == 1
            with pytest.raises(icp.InvalidArgument):
                icp.evaluate_ice_optics(float(nm))


def test_reference_known_answers(icp):
    ev = icp.evaluate_ice_optics
    assert ev(450).n == 1.3157 and ev(550).n == 1.3110 and ev(650).n == 1.3080 and ev(1100).n == 1.2998
    s = ev(math.sqrt(550.0 * 560.0))
    assert abs(s.n - (1.3110 + 1.3106) / 2) < 4e-16
    assert abs(s.kappa / math.sqrt(2.289e-9 * 2.839e-9) - 1) < 5e-15
    assert ev(200).lower_nm == 199
    for x in (199.0, 1101.0, 0.0, math.inf, math.nan, -5.0):
        with pytest.raises(icp.InvalidArgument):
            ev(x)
    last = ev(200).n
    for w in range(201, 1101):
        n = ev(w).n
        assert n < last, w
        last = n


def test_interpolation_is_linear_in_log_wavelength(icp):
    """Between two table rows, n is linear and log kappa is linear in log wavelength; the
    fraction reported is the position of log(nm) between the rows."""
    ev = icp.evaluate_ice_optics
    for nm in (203.7, 333.3, 612.5, 1045.0):
        s = ev(nm)
        a, b = ev(s.lower_nm), ev(s.upper_nm)
        f = math.log(nm / s.lower_nm) / math.log(s.upper_nm / s.lower_nm)
        assert 0 < s.log_wavelength_fraction < 1 and abs(s.log_wavelength_fraction - f) < 1e-14
        assert abs(s.n - (a.n + f * (b.n - a.n))) < 1e-15
        assert abs(math.log(s.kappa) - (math.log(a.kappa) + f * (math.log(b.kappa) - math.log(a.kappa)))) < 1e-12
