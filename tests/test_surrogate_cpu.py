"""Learned surrogate, host side (no GPU): the library's feature rows equal the oracle's bit for
bit, the oracle's analytic gradient matches central finite differences, its BF16 emulation only
rounds, and the library rejects invalid configurations."""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import surrogate_oracle as SO


def _specs(icp, n, seed=5):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        r = float(np.float32(math.exp(rng.uniform(math.log(0.1), math.log(3.0)))))
        lam = float(rng.uniform(400, 700))
        out.append(icp.DropSpec(icp.RaindropShape.make(r).coefficients, r,
                                float(np.float32(icp.evaluate_water_optics(lam).refractive_index)), rays=1000,
                                seed=1, inclination_deg=float(rng.uniform(-90, 90)), wavelength_nm=lam))
    return out


@pytest.mark.parametrize("over", [{}, {"nt": 32, "np": 64, "input_width": 64, "theta_frequencies": 14,
                                       "phi_frequencies": 4, "axis_harmonics": 8}])
def test_feature_rows_match_oracle(icp, over):
    cfg = icp.surrogate_config(**over)
    oc = SO.Config.of(cfg)
    cells = icp.surrogate_cell_features(cfg)
    assert cells.shape == (cfg.nt * cfg.np, cfg.input_width - 16)
    assert np.array_equal(cells, SO.bf16_bits(SO.cell_features(oc)))
    specs = _specs(icp, 9)
    rec = icp.surrogate_record_features(cfg, specs)
    want = np.stack([SO.bf16_bits(SO.record_features(oc, s.radius_mm, s.wavelength_nm, s.inclination_deg,
                                                      s.interior_index, s.coefficients)) for s in specs])
    assert np.array_equal(rec, want)
    # every feature stays O(1) over the batched-record ranges
    assert np.abs(SO.from_bits(rec)).max() <= 4.0 and np.abs(SO.from_bits(cells)).max() <= 1.0


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, 1.0 + 2 ** -9, -2.5, 3e38, 1e-40])
    got = SO.bf16(x)
    assert got[0] == 1.0
    assert got[1] == 1.0                       # tie: to even (mantissa 0)
    assert got[3] == 1.0                       # below the tie
    assert got[2] == 1.0 + 2 ** -7             # above the tie
    assert got[4] == -2.5
    assert np.all(np.abs(SO.bf16(got) - got) == 0)  # idempotent
    r = np.random.default_rng(0).normal(size=10000)
    assert np.all(np.abs(SO.bf16(r) - r) <= np.abs(r) * 2 ** -8)


def test_oracle_gradient_matches_finite_differences():
    cfg = SO.Config(nt=4, np=8, hidden=8, input_width=64, theta_frequencies=10, phi_frequencies=3, axis_harmonics=8)
    rng = np.random.default_rng(1)
    R = 2
    rec = rng.uniform(-1, 1, (R, 16))
    X = SO.inputs(cfg, rec, SO.cell_features(cfg), [20.0, -63.0])
    p = SO.init_parameters(cfg, 3).astype(np.float64)
    target = rng.dirichlet(np.ones(cfg.nt * cfg.np), size=R)
    target[0, :5] = 0.0
    target[0] /= target[0].sum()
    loss, g = SO.gradient(cfg, p, X, target, R, emulate=False)
    assert loss > 0
    idx = rng.choice(p.size - 1, 60, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        lp, _ = SO.gradient(cfg, p + e, X, target, R, emulate=False)
        lm, _ = SO.gradient(cfg, p - e, X, target, R, emulate=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-8, (i, fd, g[i])
    # the head bias does not change the loss (softmax is shift-invariant)
    assert abs(g[-1]) == 0.0


def test_oracle_emulation_only_rounds():
    cfg = SO.Config(nt=8, np=16, hidden=16, input_width=64, theta_frequencies=10, phi_frequencies=3, axis_harmonics=8)
    rng = np.random.default_rng(2)
    X = SO.inputs(cfg, rng.uniform(-1, 1, (1, 16)), SO.cell_features(cfg), [35.0])
    p = SO.init_parameters(cfg, 4)
    target = rng.dirichlet(np.ones(cfg.nt * cfg.np), size=1)
    l0, g0 = SO.gradient(cfg, p, X, target, 1, emulate=False)
    l1, g1 = SO.gradient(cfg, p, X, target, 1, emulate=True)
    assert abs(l1 - l0) <= 2e-2 * abs(l0)
    assert np.linalg.norm(g1 - g0) <= 5e-2 * np.linalg.norm(g0)


def test_config_validation(icp):
    for bad in [{"hidden": 96}, {"input_width": 96}, {"theta_frequencies": 60}, {"nt": 3, "np": 5},
                {"axis_harmonics": 4}, {"axis_harmonics": 32},
                {"max_records": 0}, {"wavelength_nm": (700.0, 400.0)}, {"index_scale": 0.0},
                {"max_records": 256, "nt": 4096, "np": 4096}]:  # 2^32 rows in one call
        cfg = icp.surrogate_config(**bad)
        with pytest.raises(icp.InvalidArgument):
            icp.surrogate_parameter_count(cfg)
        with pytest.raises(icp.InvalidArgument):
            icp.surrogate_cell_features(cfg)
    cfg = icp.surrogate_config()
    assert icp.surrogate_parameter_count(cfg) == SO.parameter_count(SO.Config.of(cfg)) == 256 * 128 + 2 * 256 ** 2 + 4 * 256 + 1
    with pytest.raises(icp.InvalidArgument):
        icp.surrogate_record_features(cfg, [icp.DropSpec([0] * 8, -1.0, 1.33, rays=1, seed=1)])


def test_axis_harmonics_are_the_angle_to_the_drop_axis(icp):
    """cos psi of the axis harmonics is the cosine between a cell's direction (theta from ki,
    phi from e0 towards e1, the binning's azimuth in [-pi, pi)) and the drop's axis y, and is
    even about phi = pi/2 like every other feature."""
    cfg = SO.Config(nt=8, np=16, axis_harmonics=8)
    ct, sts = SO.cell_geometry(cfg)
    for a in (0.0, 20.0, -55.0, 89.0):
        k, e0, e1 = (np.array(v) for v in icp.drop_frame(a))
        T = SO.axis_features(cfg, [a], (ct, sts))
        x = T[:, 0]
        for i in range(cfg.nt):
            th = math.pi * (i + 0.5) / cfg.nt
            for j in range(cfg.np):
                ph = -math.pi + 2 * math.pi * (j + 0.5) / cfg.np
                w = math.cos(th) * k + math.sin(th) * (math.cos(ph) * e0 + math.sin(ph) * e1)
                assert abs(x[i * cfg.np + j] - w[1]) <= 1e-6  # the frame is held in binary32
        assert np.allclose(T[:, 2], 4 * x ** 3 - 3 * x, atol=1e-12)  # T_3
        # mirror phi -> pi - phi: column j -> np/2 - 1 - j (mod np) of the [-pi, pi) azimuths
        g = x.reshape(cfg.nt, cfg.np)
        assert np.allclose(g, g[:, [(cfg.np // 2 - 1 - j) % cfg.np for j in range(cfg.np)]], atol=1e-12)


def test_fallback_gate_rules(icp):
    """The gate trusts a checked record by its own verdict, any other record only when its k
    nearest checked records (normalised log radius, wavelength, inclination) all passed; it survives
    the round trip through the model file's JSON."""
    import json

    import ice_crystal_phase_b200.surrogate as S

    def spec(r, lam, inc):
        return icp.DropSpec([0.0] * 8, r, 1.33, 1, seed=1, inclination_deg=inc, wavelength_nm=lam)

    checked = [spec(0.2, 500, 0), spec(0.21, 505, 2), spec(0.19, 495, -2), spec(2.5, 600, 40), spec(2.6, 610, 45),
              spec(2.4, 590, 35)]
    gate = S.FallbackGate.of(checked, [True, True, True, True, False, True], k=3)
    assert gate.trusted(checked[0]) and not gate.trusted(checked[4])
    assert gate.trusted(spec(0.2, 501, 1))          # all three neighbours passed
    assert not gate.trusted(spec(2.5, 601, 41))     # a failed neighbour among the three
    back = S.FallbackGate.from_dict(json.loads(json.dumps(gate.as_dict())))
    assert back.k == 3 and np.array_equal(back.passed, gate.passed) and np.allclose(back.keys, gate.keys)


def test_learning_rate_schedule():
    import ice_crystal_phase_b200.surrogate as S

    s = S.TrainSettings(lr=2e-3, lr_final=2e-5, warmup_steps=10)
    lrs = [S._lr(s, k, 110) for k in range(110)]
    assert abs(lrs[0] - 2e-4) < 1e-12 and abs(lrs[9] - 2e-3) < 1e-12      # linear warm-up
    assert abs(lrs[10] - 2e-3) < 1e-9 and abs(S._lr(s, 110, 110) - 2e-5) < 1e-12  # cosine to lr_final
    assert all(a >= b for a, b in zip(lrs[10:], lrs[11:]))


def test_storage_grid_sums_and_tv():
    import torch

    import ice_crystal_phase_b200.surrogate as S

    rng = np.random.default_rng(3)
    p = rng.dirichlet(np.ones(16 * 32), size=2)
    q = rng.dirichlet(np.ones(16 * 32), size=2)
    pt, qt = torch.from_numpy(p), torch.from_numpy(q)
    c = S.coarse(pt, 16, 32, 4, 8).numpy()
    want = p.reshape(2, 4, 4, 8, 4).sum(axis=(2, 4)).reshape(2, -1)
    assert np.allclose(c, want, atol=1e-15)
    assert np.allclose(S.tv(pt, qt).numpy(), 0.5 * np.abs(p - q).sum(axis=1))
    # aggregation never raises the total variation
    assert np.all(S.tv(S.coarse(pt, 16, 32, 4, 8), S.coarse(qt, 16, 32, 4, 8)).numpy() <= S.tv(pt, qt).numpy() + 1e-15)


def test_tv_is_the_reference_record_metric():
    """On records of one grid the surrogate's TV judge equals the reference's record-vs-record TV
    (tools/phase_analysis.py compare_tables, golden from the reference tool), and the record g
    equals its g of the saved cells."""
    import torch

    import ice_crystal_phase_b200.surrogate as S
    from conftest import GOLDEN

    z = np.load(GOLDEN / "compare_reference.npz")
    cells = {k: np.diff(z[f"phi_{k}"])[:, None] * np.diff(z[f"theta_{k}"], axis=1) for k in "ab"}
    p = torch.from_numpy(cells["a"].reshape(1, -1))
    q = torch.from_numpy(cells["b"].reshape(1, -1))
    tv, l1, marginal_tv, _, _, ga, gb = z["metrics"]
    assert float(S.tv(p, q)[0]) == pytest.approx(tv, rel=1e-12)
    e = z["edges"]
    mu = 1.0 - (e[:-1] + e[1:])
    for c, g in ((cells["a"], ga), (cells["b"], gb)):
        assert float((c * mu[None, :]).sum() / c.sum()) == pytest.approx(g, abs=1e-15)
    # the theta marginal TV is the TV of the column sums
    assert 0.5 * np.abs(cells["a"].sum(axis=0) - cells["b"].sum(axis=0)).sum() == pytest.approx(marginal_tv, rel=1e-12)


def test_drop_items_carry_every_field(icp):
    """The C array of icp_drop_item that batch and surrogate calls pass is filled column by column;
    every field equals the record description's, short coefficient lists are zero-padded and more
    than eight are refused."""
    specs = icp.batched_record_specs(9, seed=3)
    specs[0].coefficients = [0.0, -0.05]
    specs[1].diffraction = False
    arr = icp._items(specs)
    for i, sp in enumerate(specs):
        c = [float(x) for x in sp.coefficients] + [0.0] * (8 - len(sp.coefficients))
        assert list(arr[i].coefficients) == c
        assert (arr[i].radius_mm, arr[i].inclination_deg, arr[i].interior_index, arr[i].wavelength_nm) == \
            (sp.radius_mm, sp.inclination_deg, sp.interior_index, sp.wavelength_nm)
        assert (arr[i].rays, arr[i].seed, arr[i].diffraction, arr[i].reserved) == \
            (sp.rays, sp.seed, int(bool(sp.diffraction)), 0)
    assert len(icp._items([])) == 0
    specs[2].coefficients = [0.0] * 9
    with pytest.raises(ValueError):
        icp._items(specs)
