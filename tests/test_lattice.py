"""The drop's outgoing-ray lattice: the trace configuration (host) and the device trace against the
REFERENCE's own CPU lattice trace (tests/golden/drop_lattice_cases.npz, written by
tests/golden/make_lattice_fixtures.py from RaindropPathTracer::trace_vertex_unpolarized,
include/rainbow/raindrop_paths.hpp:27-107, compiled from the reference's sources).

The device records must equal the reference's bit for bit: every case compares SHA-256 digests of
the whole vertex and second-column buffers, and the lattice's middle row record by record.
"""
from __future__ import annotations

import ctypes as C
import hashlib
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = np.load(GOLDEN / "drop_lattice_cases.npz")
NAMES = [k[:-len(".args")] for k in CASES.files if k.endswith(".args")]


def _config(icp, name):
    a = str(CASES[f"{name}.args"]).split()
    radius, sphere, n_int = float(a[0]), a[1] == "1", float(a[2])
    k = tuple(float(x) for x in a[3:6])
    grid, wavelength = int(a[6]), float(a[7])
    coef = [float(x) for x in a[8:16]] if len(a) > 8 else None
    return icp.raindrop_config(radius, wavelength, n_int, k, grid, sphere=sphere, coefficients=coef)


def _bytes(struct) -> bytes:
    return bytes(C.string_at(C.addressof(struct), C.sizeof(struct)))


@pytest.mark.parametrize("name", NAMES)
def test_config_equals_reference_make_config(icp, name):
    """icp_raindrop_config_make is RaindropSettings::make_config byte for byte (shape, normalised
    direction, transverse basis, half extent, reference distances)."""
    assert C.sizeof(icp.RaindropConfig) == 116 and C.sizeof(icp.LatticeStats) == 288
    assert _bytes(_config(icp, name)) == bytes(CASES[f"{name}.config"])


def test_config_rejects_like_reference(icp):
    bad = [dict(radius_mm=3.5), dict(wavelength_nm=300.0), dict(interior_index=2.5), dict(grid=1),
           dict(incident_direction=(0.0, 0.0, 0.0)), dict(incident_direction=(float("nan"), 0.0, 1.0))]
    base = dict(radius_mm=1.0, wavelength_nm=550.0, interior_index=1.333, incident_direction=(1.0, 0.0, 0.0), grid=9)
    for b in bad:
        with pytest.raises(icp.InvalidArgument):
            icp.raindrop_config(**{**base, **b})
    with pytest.raises(icp.InvalidArgument, match="radius_mm must be in"):
        icp.raindrop_config(**{**base, "radius_mm": 0.0})


def _first_difference(v, second, name, width, height):
    idx = CASES[f"{name}.row_index"]
    want_v, want_s = CASES[f"{name}.row_vertices"], CASES[f"{name}.row_second"]
    got_v = v[idx]
    for i in range(len(idx)):
        if got_v[i].tobytes() != want_v[i].tobytes() or (second is not None and
                                                          second[idx[i]].tobytes() != want_s[i].tobytes()):
            return f"record {idx[i]}: device {got_v[i]} reference {want_v[i]}"
    return "middle row equal; difference elsewhere"


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_device_lattice_equals_reference_trace(icp, name):
    cfg = _config(icp, name)
    with icp.Context(0) as ctx:
        lat = icp.lattice_trace(ctx, cfg)
        v = lat.vertices.download()
        s = lat.second.download().reshape(-1, 4)
    vb, sb = v.tobytes(), s.tobytes()
    same = (hashlib.sha256(vb).hexdigest() == str(CASES[f"{name}.vertices_sha256"]) and
            hashlib.sha256(sb).hexdigest() == str(CASES[f"{name}.second_sha256"]))
    assert same, _first_difference(v, s, name, cfg.grid_width, cfg.grid_height)
    assert np.array_equal(lat.stats.histogram(), CASES[f"{name}.histogram"])
    assert lat.stats.incomplete == int(CASES[f"{name}.incomplete"])
    assert lat.stats.first_problem == int(CASES[f"{name}.first_problem"])
    fb = int(((v["diagnostics"] & 1) != 0).sum())
    assert lat.stats.intersection_fallbacks == fb
    assert lat.stats.snell_fallbacks == int(((v["diagnostics"] & 2) != 0).sum())


@pytest.mark.gpu
def test_device_lattice_reproduces_reference_lattice_fixture(icp):
    """The 25 x 25 lattice of a 0.5 mm sphere that feeds the patch / query / optics fixtures,
    record for record."""
    z = np.load(GOLDEN / "drop_lattice_reference.npz")
    w, h = (int(x) for x in z["shape"])
    f = z["frame"]
    cfg = icp.raindrop_config(0.5, 700.0, 1.3317, (0.9396926, -0.3420201, 0.0), w, sphere=True)
    assert np.float32(cfg.grid_half_extent) == f[0]
    with icp.Context(0) as ctx:
        lat = icp.lattice_trace(ctx, cfg)
        v = lat.vertices.download()
        s = lat.second.download().reshape(-1, 4)
    assert v.tobytes() == z["vertices"].tobytes()
    assert s.tobytes() == z["second"].tobytes()


@pytest.mark.gpu
def test_single_input_trace_is_one_column_of_the_unpolarised_trace(icp):
    """RaindropTracer::trace (one input field) and trace_unpolarized share every step; the
    response is linear, column by column: the single-input trace of the unit states gives the
    unpolarised trace's first and second columns exactly."""
    name = "table1_1.5mm_550nm_33"
    cfg = _config(icp, name)
    with icp.Context(0) as ctx:
        both = icp.lattice_trace(ctx, cfg)
        v2, s2 = both.vertices.download(), both.second.download().reshape(-1, 4)
        cfg.incident_field.x_real, cfg.incident_field.x_imag = 1.0, 0.0
        cfg.incident_field.y_real, cfg.incident_field.y_imag = 0.0, 0.0
        one = icp.lattice_trace(ctx, cfg, unpolarized=False)
        assert one.second is None
        v1 = one.vertices.download()
        cfg.incident_field.x_real, cfg.incident_field.y_real = 0.0, 1.0
        other = icp.lattice_trace(ctx, cfg, unpolarized=False).vertices.download()
    assert v1.tobytes() == v2.tobytes()
    valid = other["status"] == 1
    assert np.array_equal(other["field"][valid], s2[valid])
    rest = [k for k in icp.VERTEX_DTYPE.names if k != "field"]
    for k in rest:
        assert np.array_equal(other[k], v2[k]), k


@pytest.mark.gpu
def test_lattice_rejects_bad_configuration(icp):
    cfg = _config(icp, "sphere_0.5mm_700nm_25")
    with icp.Context(0) as ctx:
        bad = icp.RaindropConfig.from_buffer_copy(cfg)
        bad.grid_width = 1
        with pytest.raises(icp.InvalidArgument):
            icp.lattice_trace(ctx, bad)
        bad = icp.RaindropConfig.from_buffer_copy(cfg)
        bad.wavelength_nm = float("inf")
        with pytest.raises(icp.InvalidArgument):
            icp.lattice_trace(ctx, bad)
