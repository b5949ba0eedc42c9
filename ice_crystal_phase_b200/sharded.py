"""One drop record traced by several ranks (one process per GPU), summed with one all-reduce.

The reference builds one record per process on one device (apps/generate_phase.cpp:395-453).
Rays are independent and the counter RNG makes every ray depend only on (seed, ray id)
(hex_trace/include/ice_crystal/math.hpp:136-146), so a record's ray ids can be cut into
contiguous shards, one per rank: each rank traces its shard into its own FP64 histogram, the
histograms and the record's pole / hit sums are added with one collective, and rank 0 adds the
diffraction rows and builds the stored CDF.  The result equals the one-rank record up to the
order of the FP64 sums.

Everything rank-specific is here (shard bounds, per-ray weight, the sums that cross the
collective, the finishing step); the trace, the collective and the CDF build are passed in, so
that `bench.py --gpus N` runs it with the device trace, NCCL and the device CDF, and the CPU tests
run it over gloo with the oracle's trace and CDF.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Callable


@dataclass(frozen=True)
class Shard:
    rank: int
    world: int
    first: int      # first ray id of this rank
    count: int      # rays of this rank
    total: int      # rays of the whole record
    weight: float   # mm^2 of incident power per traced ray: sampling-disk area / total rays


def shard_of(total_rays: int, rank: int, world: int, sampling_area_mm2: float) -> Shard:
    """Contiguous ray-id shard of `rank`: the first total % world ranks take one ray more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    if total_rays < world:
        raise ValueError("fewer rays than ranks")
    base, extra = divmod(int(total_rays), world)
    first = rank * base + min(rank, extra)
    count = base + (1 if rank < extra else 0)
    return Shard(rank, world, first, count, int(total_rays), float(sampling_area_mm2) / float(total_rays))


@dataclass
class ShardTrace:
    """What one rank's trace returns: its cell-mass histogram (theta-major, pole caps not yet
    spread; a tensor the collective can reduce) and its shard's pole powers and hit count in
    units of one ray's incident power."""
    mass: Any
    forward_pole: float
    backward_pole: float
    hits: int


def sharded_drop_record(shard: Shard, trace: Callable[[int, int], ShardTrace], all_reduce: Callable[[Any], None],
                        finish: Callable[[Any, float, float, float], Any], make_sums: Callable[[list], Any]):
    """Traces this rank's shard, sums histograms and [forward, backward, incident] (mm^2) over
    the ranks, and on rank 0 returns finish(mass, forward_mm2, backward_mm2, incident_mm2)
    (diffraction rows and the stored CDF); other ranks return None.  Every rank takes the same
    two collective steps in the same order.  make_sums turns the three floats into a tensor on
    the histogram's device for the collective."""
    t = trace(shard.first, shard.count)
    sums = make_sums([shard.weight * t.forward_pole, shard.weight * t.backward_pole, shard.weight * t.hits])
    all_reduce(t.mass)
    all_reduce(sums)
    if shard.rank != 0:
        return None
    forward, backward, incident = (float(x) for x in sums)
    return finish(t.mass, forward, backward, incident)


def device_record(ctx, rec, grid, edges, mass, stream_sync: Callable[[], None] | None = None):
    """Trace and finish callables of the device path for sharded_drop_record: `rec` the record's
    icp_drop_record (rays = the whole record), `grid` its make_drop_grid, `edges` / `mass` device
    tensors (u edges, FP64 histogram of nt * np cells).  finish adds the analytic diffraction rows
    of the record's incident area (when rec.diffraction) and builds the stored CDF on the device;
    it returns (phi, theta, report) device tensors and the CdfReport."""
    import ctypes as C

    import torch

    import ice_crystal_phase_b200 as I

    g = grid.abi()
    nt, np_ = grid.nt, grid.np
    disk = I.sampling_area(list(rec.coefficients), rec.radius_mm)

    def trace(first: int, count: int) -> ShardTrace:
        mass.zero_()
        s = I.TraceStats()
        I.check(I.LIB.icp_drop_trace_bin(ctx.handle, C.byref(rec), first, count, disk / float(rec.rays), C.byref(g),
                                         C.c_void_p(edges.data_ptr()), C.c_void_p(mass.data_ptr()), C.byref(s)))
        return ShardTrace(mass, s.forward_pole, s.backward_pole, s.rays - s.missed)

    def finish(m, forward: float, backward: float, incident: float):
        if rec.diffraction:
            rows = torch.from_numpy(I.diffraction_rows(grid.edges, incident, rec.wavelength_nm)).to(m.device)
            m.view(nt, np_).add_(rows[:, None] / np_)
        phi = torch.empty(rec.cp + 1, dtype=torch.float64, device=m.device)
        theta = torch.empty(rec.cp * (rec.ct + 1), dtype=torch.float64, device=m.device)
        rep = I.CdfReport()
        I.check(I.LIB.icp_phase_cdf_build(ctx.handle, C.c_void_p(m.data_ptr()), 0, nt, np_, forward, backward, rec.ct,
                                          rec.cp, C.byref(rec.policy), C.c_void_p(phi.data_ptr()),
                                          C.c_void_p(theta.data_ptr()), C.byref(rep)))
        return phi, theta, rep

    def make_sums(v: list):
        return torch.tensor(v, dtype=torch.float64, device=mass.device)

    return trace, finish, make_sums, disk
