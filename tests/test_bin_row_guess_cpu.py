"""The FP32 binning's row search (csrc/icp_bin.cuh, bin_f32): the row is guessed from Hastings'
acos approximation (Abramowitz & Stegun 4.4.45) of the scattering angle and then settled against
the stored u edges by stepping down or up.  Restated in binary32 here, the settled row equals a
binary search in the edges for every direction, and the search takes at most one step for grids
of up to 16384 rows (more for finer ones, where it still ends on the right row)."""
from __future__ import annotations

import numpy as np
import pytest

F = np.float32


def _edges(nt: int) -> np.ndarray:
    i = np.arange(nt + 1, dtype=np.float64)
    return np.sin(np.pi * i / (2 * nt)) ** 2


def _guess_and_settle(mu, u, edges32, nt):
    am = np.minimum(np.abs(mu), F(1))
    poly = ((F(-0.0187293) * am + F(0.0742610)) * am + F(-0.2121144)) * am + F(1.5707288)
    acos_am = (np.sqrt(F(1) - am) * poly).astype(F)
    theta = np.where(mu >= 0, acos_am, F(3.14159265) - acos_am).astype(F)
    i = np.floor(theta * F(nt / np.pi)).astype(np.int64)
    i = np.clip(i, 0, nt - 1)
    steps = np.zeros_like(i)
    while True:  # vectorised form of the two while loops
        down = (i > 0) & (u < edges32[i])
        up = ~down & (i < nt - 1) & (u >= edges32[np.minimum(i + 1, nt)])
        if not (down.any() or up.any()):
            return i, steps
        i = i - down + up
        steps += down | up


@pytest.mark.parametrize("nt", [90, 900, 4096, 16384, 100000])
def test_row_guess_settles_on_the_binary_search_row(nt):
    rng = np.random.default_rng(nt)
    mu = rng.uniform(-1, 1, 200000).astype(F)
    mu = np.concatenate([mu, F([-1, 1, 0]), np.nextafter(F(1), F(0), dtype=F)[None],
                         np.nextafter(F(-1), F(0), dtype=F)[None]]).astype(F)
    edges32 = _edges(nt).astype(F)
    u = ((F(1) - mu) * F(0.5)).astype(F)
    row, steps = _guess_and_settle(mu, u, edges32, nt)
    want = np.clip(np.searchsorted(edges32, u, side="right") - 1, 0, nt - 1)
    assert np.array_equal(row, want)
    if nt <= 16384:
        assert steps.max() <= 1, int(steps.max())
