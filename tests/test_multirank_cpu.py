"""The N-rank record of bench.py --gpus N on the CPU: world size 2 over gloo, each rank traces
its own contiguous ray-id shard of one drop record (here with the CPU oracle), the FP64
histograms, pole sums and hit counts are summed with one all-reduce, and rank 0 adds the
diffraction rows and builds the CDF.  The counter RNG makes the result partition-invariant:
it must equal the one-rank record up to FP64 summation order."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

RAYS_PER_RANK = 3000
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


def _rank(rank: int, world: int, port: int, out: str) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        icp, oracle, geo, frame = _record_inputs()
        total = RAYS_PER_RANK * world
        rec = oracle.drop_record(geo, frame, 1.3317, NT, NP, total, 77, max_hits=10, first=rank * RAYS_PER_RANK,
                                 count=RAYS_PER_RANK)
        mass = torch.from_numpy(rec.masses.copy())
        sums = torch.tensor([rec.incident_area, rec.escaped_area, rec.unresolved_area], dtype=torch.float64)
        dist.all_reduce(mass)
        dist.all_reduce(sums)
        if rank == 0:
            rows = icp.diffraction_rows(icp.u_edges(NT), float(sums[0]), 650.0)
            m = mass.numpy().reshape(NT, NP) + rows[:, None] / NP
            cdf = oracle.build_cdf(m.reshape(-1), NT, NP)
            np.savez(out, mass=mass.numpy(), sums=sums.numpy(), phi=cdf.phi, theta=cdf.theta,
                     g=cdf.report["g_stored"])
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_equal_one_rank_record(tmp_path):
    out = str(tmp_path / "r0.npz")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    got = np.load(out)
    icp, oracle, geo, frame = _record_inputs()
    one = oracle.drop_record(geo, frame, 1.3317, NT, NP, 2 * RAYS_PER_RANK, 77, max_hits=10)
    assert np.abs(got["mass"] - one.masses).sum() <= 1e-13 * one.masses.sum()
    assert abs(got["sums"][0] - one.incident_area) <= 1e-14 * one.incident_area
    assert abs(got["sums"][1] / one.escaped_area - 1) <= 1e-13
    rows = icp.diffraction_rows(icp.u_edges(NT), one.incident_area, 650.0)
    cdf = oracle.build_cdf((one.masses.reshape(NT, NP) + rows[:, None] / NP).reshape(-1), NT, NP)
    p_one = np.diff(cdf.phi)[:, None] * np.diff(cdf.theta, axis=1)
    p_two = np.diff(got["phi"])[:, None] * np.diff(got["theta"], axis=1)
    assert np.abs(p_one - p_two).sum() <= 1e-12
    assert abs(float(got["g"]) - cdf.report["g_stored"]) <= 1e-13
