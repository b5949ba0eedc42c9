"""The N-rank record of bench.py --gpus N on the CPU: world size 2 over gloo through the same
package function bench.py runs (ice_crystal_phase_b200.sharded.sharded_drop_record), with the
CPU oracle's trace and CDF build injected in place of the device's.  Each rank traces its own
contiguous ray-id shard of one drop record, the FP64 histograms and the pole / hit sums cross one
all-reduce each, and rank 0 adds the diffraction rows and builds the CDF.  The counter RNG makes
the result partition-invariant: it must equal the one-rank record up to FP64 summation order,
also for a ray count that does not divide by the world size."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

NT, NP = 36, 72


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _record_inputs():
    import ice_crystal_phase_b200 as icp
    from oracle import oracle

    coeff = icp.RaindropShape.make(1.5).coefficients
    geo = oracle.drop_geometry(coeff, 1.5)
    frame = np.array(icp.drop_frame(20.0))
    return icp, oracle, geo, frame


def _oracle_parts(total: int):
    """Trace / finish callables of sharded_drop_record with the oracle in place of the device."""
    icp, oracle, geo, frame = _record_inputs()

    def trace(first: int, count: int):
        from ice_crystal_phase_b200.sharded import ShardTrace

        rec = oracle.drop_record(geo, frame, 1.3317, NT, NP, total, 77, max_hits=10, first=first, count=count)
        w = geo.disk_area_mm2 / total  # the oracle's pole sums are in mm^2 already: back to ray units
        return ShardTrace(torch.from_numpy(rec.cells.copy()), rec.forward / w, rec.backward / w,
                          rec.counts["rays"] - rec.counts["missed"])

    def finish(mass, forward, backward, incident):
        rows = icp.diffraction_rows(icp.u_edges(NT), incident, 650.0)
        m = mass.numpy().reshape(NT, NP).copy() + rows[:, None] / NP
        m[0] += forward / NP
        m[-1] += backward / NP
        cdf = oracle.build_cdf(m.reshape(-1), NT, NP)
        return mass.numpy().copy(), np.array([forward, backward, incident]), cdf

    return trace, finish, geo


def _rank(rank: int, world: int, port: int, total: int, out: str) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from ice_crystal_phase_b200.sharded import shard_of, sharded_drop_record

        trace, finish, geo = _oracle_parts(total)
        shard = shard_of(total, rank, world, geo.disk_area_mm2)
        got = sharded_drop_record(shard, trace, dist.all_reduce, finish,
                                  lambda v: torch.tensor(v, dtype=torch.float64))
        if rank == 0:
            mass, sums, cdf = got
            np.savez(out, mass=mass, sums=sums, phi=cdf.phi, theta=cdf.theta, g=cdf.report["g_stored"])
        else:
            assert got is None
    finally:
        dist.destroy_process_group()


def test_shard_bounds_cover_the_record_once():
    from ice_crystal_phase_b200.sharded import shard_of

    for total, world in ((10, 3), (6001, 2), (100_000_000, 8), (7, 7)):
        shards = [shard_of(total, r, world, 1.0) for r in range(world)]
        assert shards[0].first == 0 and sum(s.count for s in shards) == total
        assert all(a.first + a.count == b.first for a, b in zip(shards, shards[1:]))
        assert max(s.count for s in shards) - min(s.count for s in shards) <= 1
        assert all(s.weight == 1.0 / total for s in shards)
    with pytest.raises(ValueError):
        shard_of(10, 2, 2, 1.0)
    with pytest.raises(ValueError):
        shard_of(1, 0, 2, 1.0)


@pytest.mark.parametrize("total", [6000, 6001])
def test_two_rank_shards_equal_one_rank_record(tmp_path, total):
    out = str(tmp_path / "r0.npz")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, total, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    got = np.load(out)
    icp, oracle, geo, frame = _record_inputs()
    one = oracle.drop_record(geo, frame, 1.3317, NT, NP, total, 77, max_hits=10)
    assert np.abs(got["mass"] - one.cells).sum() <= 1e-13 * one.cells.sum()
    assert abs(got["sums"][2] - one.incident_area) <= 1e-14 * one.incident_area
    assert abs(got["sums"][0] - one.forward) <= 1e-13 * max(one.forward, 1e-300)
    rows = icp.diffraction_rows(icp.u_edges(NT), one.incident_area, 650.0)
    cdf = oracle.build_cdf((one.masses.reshape(NT, NP) + rows[:, None] / NP).reshape(-1), NT, NP)
    p_one = np.diff(cdf.phi)[:, None] * np.diff(cdf.theta, axis=1)
    p_two = np.diff(got["phi"])[:, None] * np.diff(got["theta"], axis=1)
    assert np.abs(p_one - p_two).sum() <= 1e-12
    assert abs(float(got["g"]) - cdf.report["g_stored"]) <= 1e-13
