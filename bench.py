"""Benchmark: rays/s of one phase-function record on B200 (and the reference CPU arm).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload drop|hex] [--rays R]

Default workload (drop, the configuration the headline metric is quoted on): an oblate water
drop of equal-volume radius 1.5 mm with r/a = 1 - 0.08 cos(chi) - 0.02 cos(2 chi) + 0.005 cos(3 chi),
650 nm, n = IAPWS R9-97 water at 20 C (binary32, as the solver holds it), inclination 20 deg,
1e8 rays sampled over the drop's bounding disk (seed 12345), at most 10 internal interactions
(the residual is reported), 900 x 1800 (u, phi) cells, analytic Fraunhofer diffraction stage,
FP32 trace, FP64 histogram flush and CDF.  A step is one record: projected area (CPU FP64),
trace + bin of all rays, diffraction rows and the stored CDF.
Workload hex (--workload hex): the hexagonal ice column (circumradius 0.05 mm, length 0.2 mm,
n = 1.31, 550 nm, ki = (cos30, -sin30, 0), 1e8 rays, 12 interactions, 512 x 1024 cells).

With N ranks (torchrun) every rank traces its own 1e8-ray shard of one record (weak scaling),
the FP64 histograms are summed with one NCCL all-reduce, and rank 0 finishes the record.

Two more measurements ride on the same line (N = 1):
* `batched`: 256 records of the batched distribution in one autotuned, graph-captured launch,
  against the same records one by one through the plain entry;
* `surrogate`: the committed learned surrogate on 256 fresh records (256 x 512 cells, stored at
  64 x 128), alone and with its tracer fallback, against the plain tracer on the same records,
  with a held-out sample checked by 1e8-ray tracer records and the forward pass against the BF16
  peak.

Timing: CUDA events on the library's stream, W untimed warm-up steps, K timed steps, each
bracketed by barrier + synchronize; an L2 flush (a 256 MiB write) separates timed steps;
max over ranks.  `value` keeps the outputs in HBM (icp_drop_generate_device); `e2e` goes
through the public host-buffer entry (icp_drop_generate / icp_hex_generate) with the
host<->device copies inside the timed region.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of the drop record's two
# kernels, from single-pass ncu captures of this workload: the 1e8-ray trace launch
# (profiles/drop_trace_bin_kernel_dram_oblate_1e8.md) and the 900 x 1800 CDF launch
# (profiles/cdf_build_kernel_900x1800.md)
DROP_TRACE_TRAFFIC = 14.249e6 + 2.328e6
DROP_CDF_TRAFFIC = 13.0885e6 + 0.0
CFG = dict(R=0.05, L=0.2, ki=(0.8660254037844387, -0.5, 0.0), n=1.31, nt=512, np=1024, hits=12, seed=12345)
DROP = dict(radius=1.5, coefficients=(0.0, -0.08, -0.02, 0.005, 0.0, 0.0, 0.0, 0.0), wavelength=650.0, incl=20.0,
            nt=900, np=1800, hits=10, seed=12345)
METRIC = "rays/s (one phase-function record: rays traced, binned and stored as a CDF)"
# Algorithmic FP32 work counted from the trace kernel source (flops per event; div/sqrt/rsqrt,
# sincospi and atan2 counted as one op each).  Prism: entry = geometry 20 + Fresnel/Stokes split
# 150 + binning 80; internal interaction = nearest-plane search 66 + split 150 + binning 80.
FLOP_ENTRY, FLOP_INTERACTION = 250.0, 296.0
# Drop: every sampled ray = disk point 20 + bounding-sphere roots 12; entry of a hit = normal 105
# + split 150 + binning 80; internal interaction = bounding-sphere roots 12 + normal 105 + split
# 150 + binning 80; each Newton evaluation of the surface gauge (Chebyshev R, dR/dmu) = 110.
FLOP_DROP_RAY, FLOP_DROP_ENTRY, FLOP_DROP_INTERACTION, FLOP_DROP_GAUGE = 32.0, 335.0, 347.0, 110.0


def _env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, device: int):
        self.device, self.rows, self.proc = device, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # the timed region starts once the sampler is running (nvidia-smi takes a moment)
            t0 = time.perf_counter()
            while not self.rows and time.perf_counter() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm = [float(r[0]) for r in self.rows if r and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) > 1 and r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 3 + i and r[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm)}


# ----------------------------------------------------------------------------- reference arm
def reference_sample(rays_per_proc: int, procs: int) -> dict:
    """Reference CPU path (oracle/_ref/ref_hex_harness, built from the reference sources),
    one process per core over disjoint ray-id slices of the same record."""
    exe = ROOT / "oracle" / "_ref" / "ref_hex_harness"
    if not exe.exists():
        raise FileNotFoundError(exe)
    c = CFG
    args = [str(exe), "time", repr(c["R"]), repr(c["L"]), *map(repr, c["ki"]), repr(c["n"]), "1", str(c["nt"]),
            str(c["np"]), str(c["hits"]), repr(1e-12), str(c["seed"])]
    t0 = time.perf_counter()
    ps = [subprocess.Popen(args + [str(i * rays_per_proc), str(rays_per_proc)], stdout=subprocess.PIPE, text=True)
          for i in range(procs)]
    outs = [json.loads(p.communicate()[0]) for p in ps]
    wall = time.perf_counter() - t0
    rays = sum(o["rays"] for o in outs)
    return {"rays": rays, "seconds": wall, "rays_per_s": rays / wall, "procs": procs}


def run_reference_hex(a) -> None:
    rank, world, _ = _env_rank()
    if rank != 0:
        return
    procs = os.cpu_count() or 1
    per = max(1000, 5 * int(a.ref_rays) // procs)
    for _ in range(a.warmup):
        reference_sample(max(1000, per // 10), procs)
    vals = [reference_sample(per, procs) for _ in range(a.steps)]
    v = sum(x["rays"] for x in vals) / sum(x["seconds"] for x in vals)
    line = {"metric": METRIC, "value": v, "unit": "rays/s", "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1e3 * sum(x["seconds"] for x in vals) / len(vals), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "hex_column_r0.05mm_1e8_rays_512x1024", **_cfg_public()}, "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "rays/s", "cores": procs, "kind": "reference",
                             "sample": f"{per} rays per process x {procs} processes per step (disjoint ray ids), "
                                       "reference ice_crystal hex trace + PhaseMassAccumulator"},
            "e2e": {"value": v, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _drop_reference_inputs() -> dict:
    """Interior index (the reference's water model at 650 nm, 20 C, as binary32, from its own
    evaluate_water_optics) and the incident direction the reference CLI builds."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np

    import oracle

    d = DROP
    n = float(np.float32(oracle.ref_drop_lines("water", ["650.0 20.0 101325.0"])[0][0]))
    a = math.radians(d["incl"])
    return {"n": n, "k": (float(np.float32(math.cos(a))), float(np.float32(-math.sin(a))), 0.0)}


def reference_drop_sample(rays_per_proc: int, procs: int, inputs: dict, first: int = 0) -> dict:
    """The record's work by the reference's own CPU code (oracle/_ref/ref_record_harness, built
    from its sources): the same sampled ray ids of this record, at most 10 internal interactions
    through its drop intersector and Fresnel split, every exit binned by its PhaseMassAccumulator,
    and the stored CDF of the histogram by its build_host_cdf.  One process per core over
    disjoint ray-id slices; the first process also builds the 900 x 1800 CDF (one record's CDF per
    step).  Rays/s = rays of all processes / wall time of the step."""
    exe = ROOT / "oracle" / "_ref" / "ref_record_harness"
    if not exe.exists():
        raise FileNotFoundError(exe)
    d = DROP
    base = [str(exe), "record", repr(d["radius"]), repr(inputs["n"]), *map(repr, inputs["k"]), str(d["nt"]),
            str(d["np"]), str(d["hits"]), str(d["seed"]), str(int(1e8))]
    t0 = time.perf_counter()
    ps = [subprocess.Popen(base + [str(first + i * rays_per_proc), str(rays_per_proc), *map(repr, d["coefficients"]),
                                   "1" if i == 0 else "0"], stdout=subprocess.PIPE, text=True) for i in range(procs)]
    outs = [p.communicate()[0].split() for p in ps]
    wall = time.perf_counter() - t0
    if any(p.returncode != 0 for p in ps):
        raise RuntimeError("reference record harness failed")
    rays = sum(int(o[0]) for o in outs)
    return {"rays": rays, "hits": sum(int(o[1]) for o in outs), "exits": sum(int(o[2]) for o in outs),
            "seconds": wall, "procs": procs, "rays_per_s": rays / wall, "cdf_seconds": float(outs[0][4]),
            "trace_seconds_per_proc": sum(float(o[3]) for o in outs) / procs}


def _drop_public() -> dict:
    d = DROP
    return {"radius_mm": d["radius"], "shape_coefficients": list(d["coefficients"]), "wavelength_nm": d["wavelength"],
            "inclination_deg": d["incl"], "cells": [d["nt"], d["np"]], "max_internal_hits": d["hits"],
            "seed": d["seed"], "diffraction": "analytic_fraunhofer", "material": "water_iapws_r9_97_20C"}


def run_reference_drop(a) -> None:
    rank, world, _ = _env_rank()
    if rank != 0:
        return
    procs = os.cpu_count() or 1
    inputs = _drop_reference_inputs()
    per = max(100, int(a.ref_rays) // procs)
    for _ in range(a.warmup):
        reference_drop_sample(max(100, per // 10), procs, inputs)
    vals = [reference_drop_sample(per, procs, inputs, first=i * per * procs) for i in range(a.steps)]
    v = sum(x["rays"] for x in vals) / sum(x["seconds"] for x in vals)
    sample = (f"{per} rays per process x {procs} processes per step (disjoint ray ids of this record), "
              "<= 10 internal interactions, every exit binned, one 900x1800 stored CDF per step; the reference's "
              "RaindropIntersector, DielectricInterface::split, PhaseMassAccumulator and build_host_cdf compiled from "
              "its sources (oracle/_ref/ref_record_harness)")
    line = {"metric": METRIC, "value": v, "unit": "rays/s", "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1e3 * sum(x["seconds"] for x in vals) / len(vals), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "oblate_drop_1.5mm_1e8_rays_900x1800", **_drop_public()}, "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "rays/s", "cores": procs, "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _cfg_public() -> dict:
    c = CFG
    return {"circumradius_mm": c["R"], "length_mm": c["L"], "ki": list(c["ki"]), "interior_index": c["n"],
            "wavelength_nm": 550, "cells": [c["nt"], c["np"]], "max_internal_hits": c["hits"], "seed": c["seed"]}


# ----------------------------------------------------------------------------- B200 arm
def run_b200_hex(a) -> None:
    import ctypes as C

    import numpy as np
    import torch

    import ice_crystal_phase_b200 as I

    rank, world, local = _env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    ctx = I.Context(local)
    stream = torch.cuda.ExternalStream(I.LIB.icp_context_stream(ctx.handle))
    torch.cuda.set_stream(stream)
    c = CFG
    rays = int(a.rays)
    grid = I.make_phase_grid(c["nt"], c["np"], c["ki"])
    g = grid.abi()
    edges = torch.from_numpy(grid.edges).cuda()
    mass = torch.zeros(c["nt"] * c["np"], dtype=torch.float64, device="cuda")
    phi = torch.empty(c["np"] + 1, dtype=torch.float64, device="cuda")
    theta = torch.empty(c["np"] * (c["nt"] + 1), dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    node = I.HexNode()
    node.circumradius_mm, node.length_mm = c["R"], c["L"]
    for i, v in enumerate(I.rotation_from_quaternion(1, 0, 0, 0)):
        node.rotation[i] = v
    node.exterior_index, node.interior_index = 1.0, c["n"]
    node.tail_tolerance, node.balance_tolerance = 1e-12, 1e-10
    node.seed, node.total_samples = c["seed"], rays * world
    node.first_sample, node.sample_count = rank * rays, rays
    node.max_internal_hits, node.batch_size, node.precision = c["hits"], 4096, I.ICP_FP32
    area = C.c_double()
    I.check(I.LIB.icp_hex_node_area(C.byref(node), C.byref(g), C.byref(area)))
    node.area_weight = area.value / float(rays * world)
    policy = I.CdfPolicy(1e-10, 1e-12, 1.0)
    pole = torch.zeros(2, dtype=torch.float64, device="cuda")

    def step() -> I.TraceStats:
        mass.zero_()
        s = I.TraceStats()
        I.check(I.LIB.icp_hex_trace_bin(ctx.handle, C.byref(node), C.byref(g), C.c_void_p(edges.data_ptr()),
                                        C.c_void_p(mass.data_ptr()), C.byref(s), None, None))
        if world > 1:
            pole[0], pole[1] = node.area_weight * s.forward_pole, node.area_weight * s.backward_pole
            dist.all_reduce(mass)
            dist.all_reduce(pole)
            fwd, bwd = float(pole[0]), float(pole[1])
        else:
            fwd, bwd = node.area_weight * s.forward_pole, node.area_weight * s.backward_pole
        if rank == 0:
            rep = I.CdfReport()
            I.check(I.LIB.icp_phase_cdf_build(ctx.handle, C.c_void_p(mass.data_ptr()), 0, c["nt"], c["np"], fwd, bwd,
                                              c["nt"], c["np"], C.byref(policy), C.c_void_p(phi.data_ptr()),
                                              C.c_void_p(theta.data_ptr()), C.byref(rep)))
        return s

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(a.warmup):
        stats = step()
    # timed region: K steps, device events per step, L2 flush between steps (not timed)
    launches0 = I.kernel_launches()
    times, stats_all = [], []
    with ClockSampler(local) as clocks:
        for _ in range(a.steps):
            flush.fill_(1.0)
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            stats_all.append(step())
            e1.record(stream)
            barrier()
            times.append(e0.elapsed_time(e1) / 1e3)
    launches = I.kernel_launches() - launches0
    t_local = torch.tensor([sum(times)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t_local, op=dist.ReduceOp.MAX)
    t_step = float(t_local) / a.steps
    value = rays * world / t_step

    # dominant kernel alone (trace+bin), for the roofline: events on the same stream
    s0 = stats_all[-1]
    mean_hits = s0.encounters / max(1, s0.rays)
    flops_per_ray = FLOP_ENTRY + FLOP_INTERACTION * mean_hits
    k_times = []
    for _ in range(2):
        flush.fill_(1.0)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        mass.zero_()
        s = I.TraceStats()
        e0.record(stream)
        I.check(I.LIB.icp_hex_trace_bin(ctx.handle, C.byref(node), C.byref(g), C.c_void_p(edges.data_ptr()),
                                        C.c_void_p(mass.data_ptr()), C.byref(s), None, None))
        e1.record(stream)
        barrier()
        k_times.append(e0.elapsed_time(e1) / 1e3)
    t_kernel = min(k_times)
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    clk = clocks.summary()
    mhz = clk["sm_mhz"] or 1965.0
    fp32_peak = sms * 128 * 2 * mhz * 1e6 / 1e12
    achieved = rays * flops_per_ray / t_kernel / 1e12

    # CDF kernel alone (HBM bound): read 8*C, write 8*np*(nt+1) + 8*(np+1)
    cdf_bytes = 8 * c["nt"] * c["np"] + 8 * c["np"] * (c["nt"] + 1) + 8 * (c["np"] + 1)
    cdf_t = cdf_kernel_times(I, ctx, stream, mass, c["nt"], c["np"], phi, theta, flush, policy) if rank == 0 else []
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)

    # e2e through the host-buffer public entry (N=1) or the sharded Python entry (N>1)
    e2e_times = []
    ph = torch.empty(c["np"] + 1, dtype=torch.float64).pin_memory()
    th = torch.empty(c["np"] * (c["nt"] + 1), dtype=torch.float64).pin_memory()
    uh = torch.empty(c["nt"] + 1, dtype=torch.float64).pin_memory()
    if world == 1:
        rec = I.HexRecordArgs()
        rec.circumradius_mm, rec.length_mm = c["R"], c["L"]
        for i in range(3):
            rec.ki[i] = c["ki"][i]
        rec.exterior_index, rec.interior_index = 1.0, c["n"]
        rec.tail_tolerance, rec.balance_tolerance = 1e-12, 1e-10
        rec.nt, rec.np, rec.ct, rec.cp = c["nt"], c["np"], c["nt"], c["np"]
        rec.max_internal_hits, rec.batch_size, rec.precision = c["hits"], 4096, I.ICP_FP32
        rec.policy = policy
        nodes = (I.Orientation * 1)()
        nodes[0].quaternion[0] = 1.0
        nodes[0].weight, nodes[0].samples, nodes[0].seed = 1.0, rays, c["seed"]
        for i in range(a.steps + 1):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            rr = I.RecordReport()
            e0.record(stream)
            I.check(I.LIB.icp_hex_generate(ctx.handle, C.byref(rec), nodes, 1,
                                           C.cast(C.c_void_p(ph.data_ptr()), I._D),
                                           C.cast(C.c_void_p(th.data_ptr()), I._D),
                                           C.cast(C.c_void_p(uh.data_ptr()), I._D), C.byref(rr)))
            e1.record(stream)
            torch.cuda.synchronize()
            if i:
                e2e_times.append(e0.elapsed_time(e1) / 1e3)
        e2e_value = rays / (sum(e2e_times) / len(e2e_times))
    else:
        e2e_value = None
    h2d = 8 * (c["nt"] + 1) + 168  # u edges + per-node record arguments
    d2h = 8 * (c["np"] + 1) + 8 * c["np"] * (c["nt"] + 1) + 200

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            procs = os.cpu_count() or 1
            rb = reference_sample(max(2000, 5 * int(a.ref_rays) // procs), procs)
            cpu = {"value": rb["rays_per_s"], "unit": "rays/s", "cores": procs, "kind": "reference",
                   "sample": f"{rb['rays']} rays of the same record (disjoint ray ids, {procs} processes), "
                             "reference hex tracer + PhaseMassAccumulator compiled from its sources"}
        except (OSError, ValueError) as e:
            cpu = {"value": None, "unit": "rays/s", "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}

    line = {
        "metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * t_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "hex_column_r0.05mm_1e8_rays_512x1024", **_cfg_public(), "rays_per_gpu": rays,
                   "l2": "flushed between timed steps (256 MiB write)", "trace_precision": "fp32",
                   "parallelism": f"ray shards x{world}, NCCL all-reduce of FP64 histogram" if world > 1 else "1 GPU"},
        "records_per_s": 1.0 / t_step,
        "e2e": {"value": e2e_value, "unit": "rays/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": {"kernel": "hex_trace_bin_kernel<float>", "bound": "fp32_simt", "achieved": achieved,
                     "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak, "traffic": None,
                     "peak_note": f"derived: {sms} SMs x 128 FP32 lanes x 2 x {mhz:.0f} MHz (median SM clock under load)",
                     "flops_per_ray": flops_per_ray, "kernel_ms": 1e3 * t_kernel,
                     "mean_interactions_per_ray": mean_hits},
        "roofline_cdf": ({"kernel": "cdf_build_kernel", "bound": "hbm", "achieved": cdf_bytes / statistics.mean(cdf_t) / 1e9,
                          "peak": hbm, "unit": "GB/s", "frac": cdf_bytes / statistics.mean(cdf_t) / 1e9 / hbm,
                          "traffic": None, "algorithmic_bytes": cdf_bytes, "kernel_us": 1e6 * statistics.mean(cdf_t), "kernel_us_min": 1e6 * min(cdf_t),
                          "peak_note": "MEASURED_PEAKS.json hbm_gbs (of measured)"} if cdf_t else None),
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": launches,
        "trace": {"outputs_per_ray": s0.outputs / max(1, s0.rays), "unresolved_fraction": s0.unresolved / max(1, s0.rays),
                  "fallback_adds": s0.fallback_adds, "near_edge": s0.near_edge},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_batched(I, ctx, stream, a, nt: int, np_: int) -> dict:
    """Batched records: one autotuned, graph-captured persistent launch per batch (device-resident
    outputs), timed with CUDA events on the library stream; then the same records through the
    single-record entry one after another (the plain path) for records/s at equal work."""
    import ctypes as C

    import torch

    specs = I.batched_record_specs(a.batch_records)
    rays = sum(sp.rays for sp in specs)
    s = I.batch_settings(nt, np_, max_internal_hits=DROP["hits"], precision=I.ICP_FP32, use_graph=True)
    tuned_rate = I.autotune_drop_batch(ctx, specs, s)
    n = len(specs)
    phi = torch.empty(n * (np_ + 1), dtype=torch.float64, device="cuda")
    theta = torch.empty(n * np_ * (nt + 1), dtype=torch.float64, device="cuda")
    items = I._items(specs)
    reps = (I.DropReport * n)()
    launches0 = I.kernel_launches()

    def one_batch():
        I.check(I.LIB.icp_drop_batch_generate_device(ctx.handle, items, n, C.byref(s), C.c_void_p(phi.data_ptr()),
                                                     C.c_void_p(theta.data_ptr()), reps))

    one_batch()  # warm-up (captures and instantiates the graph)
    times = []
    for _ in range(a.batch_steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        one_batch()
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    launches = (I.kernel_launches() - launches0) // (a.batch_steps + 1)
    t = sum(times) / len(times)
    tv_ok = all(r.cdf.status == 0 for r in reps)
    # plain: the same records one by one through the single-record device entry
    rec_phi = torch.empty(np_ + 1, dtype=torch.float64, device="cuda")
    rec_theta = torch.empty(np_ * (nt + 1), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for sp in specs:
        r = I._drop_args(sp.coefficients, sp.radius_mm, sp.inclination_deg, sp.interior_index, sp.rays, sp.seed, nt,
                         np_, nt, np_, 1.0, DROP["hits"], 1e-12, I.ICP_FP32, 1e-10, sp.wavelength_nm, True)
        rr = I.DropReport()
        I.check(I.LIB.icp_drop_generate_device(ctx.handle, C.byref(r), C.c_void_p(rec_phi.data_ptr()),
                                               C.c_void_p(rec_theta.data_ptr()), None, C.byref(rr)))
    e1.record(stream)
    torch.cuda.synchronize()
    t_plain = e0.elapsed_time(e1) / 1e3
    return {"workload": "batched_drop_records_256_900x1800", "records": n, "rays": rays, "seed": 20260101,
            "cells": [nt, np_], "max_internal_hits": DROP["hits"], "diffraction": "analytic_fraunhofer",
            "ms_per_batch": 1e3 * t, "rays_per_s": rays / t, "records_per_s": n / t,
            "plain_loop": {"seconds": t_plain, "rays_per_s": rays / t_plain, "records_per_s": n / t_plain},
            "speedup_vs_plain_loop": t_plain / t, "cuda_graph": True, "kernel_launches_per_batch": launches,
            "tuned": {"block_threads": s.block_threads, "chunk_rays": s.chunk_rays,
                      "sample_rays_per_s": tuned_rate}, "all_records_pass_cdf_audits": tv_ok}




def run_surrogate(I, ctx, stream, a) -> dict:
    """The learned surrogate on fresh records of the batched distribution (256 x 512 cells, stored
    at 64 x 128): records/s of serving (surrogate where the fallback gate trusts it, the batched
    tracer elsewhere) and of the surrogate alone, against the plain single-record tracer entry on
    the same records; held-out TV of a fresh sample against 1e8-ray tracer records; the forward
    pass against the measured BF16 tensor peak."""
    import ctypes as C

    import torch

    import ice_crystal_phase_b200.surrogate as S

    if not S.DEFAULT_MODEL.exists():
        return {"unavailable": f"{S.DEFAULT_MODEL.name} missing"}
    R = a.surrogate_batch  # records per surrogate call
    sur, extra = S.load(ctx, S.DEFAULT_MODEL, max_records=R)
    gate = S.FallbackGate.from_dict(extra["gate"])
    ct, cp = extra["storage"]
    nt, np_ = sur.cfg.nt, sur.cfg.np
    specs = I.batched_record_specs(a.surrogate_records, seed=20260102)
    n = len(specs)
    phi = torch.empty(n * (cp + 1), dtype=torch.float64, device="cuda")
    theta = torch.empty(n * cp * (ct + 1), dtype=torch.float64, device="cuda")

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3, out

    def surrogate_only():
        for i in range(0, n, R):
            sur.generate(specs[i:i + R], ct, cp, phi[i * (cp + 1):].data_ptr(), theta[i * cp * (ct + 1):].data_ptr(),
                         raise_on_audit=False)

    surrogate_only()  # warm-up
    t_sur = min(timed(surrogate_only)[0] for _ in range(3))
    launches0 = I.kernel_launches()
    S.serve(ctx, sur, specs, gate, ct, cp, phi, theta)  # warm-up
    t_serve, served = timed(lambda: S.serve(ctx, sur, specs, gate, ct, cp, phi, theta))
    launches = (I.kernel_launches() - launches0) // 2
    # the plain GPU tracer: the same records one by one through the single-record device entry
    rec_phi = torch.empty(cp + 1, dtype=torch.float64, device="cuda")
    rec_theta = torch.empty(cp * (ct + 1), dtype=torch.float64, device="cuda")

    def plain():
        for sp in specs:
            r = I._drop_args(sp.coefficients, sp.radius_mm, sp.inclination_deg, sp.interior_index, sp.rays, sp.seed,
                             nt, np_, ct, cp, 1.0, 10, 1e-12, I.ICP_FP32, 1e-10, sp.wavelength_nm, True)
            rr = I.DropReport()
            I.check(I.LIB.icp_drop_generate_device(ctx.handle, C.byref(r), C.c_void_p(rec_phi.data_ptr()),
                                                   C.c_void_p(rec_theta.data_ptr()), None, C.byref(rr)))

    t_plain, _ = timed(plain)
    # forward pass of R records on the tensor cores
    nf = min(R, n)  # records of the timed forward pass
    y = torch.empty(nf * sur.cells, dtype=torch.float32, device="cuda")
    sur.predict(specs[:nf], y.data_ptr())
    t_fwd = min(timed(lambda: sur.predict(specs[:nf], y.data_ptr()))[0] for _ in range(5))
    H, K0 = sur.cfg.hidden, sur.cfg.input_width
    flops = 2.0 * nf * sur.cells * (K0 * H + 2 * H * H + H)
    peaks = _peaks()
    bf16 = peaks.get("bf16_tflops", 1590.0)
    # fresh held-out sample checked by the tracer
    truth_specs = I.batched_record_specs(a.surrogate_checked, seed=20260103)
    st = S.TrainSettings(truth_rays=1e8, storage=(ct, cp))
    ev = S.evaluate(ctx, sur, truth_specs, st)
    sur.close()
    tv = ev["storage"]["tv"]
    # the fallback gate's decisions on the checked records: how many records it would serve by the
    # surrogate, and how many of those are out of tolerance against their 1e8-ray truth
    trusted = [gate.trusted(sp) for sp in truth_specs]
    served_tv = [t for ok, t in zip(trusted, tv) if ok]
    served_bad = sum(1 for t in served_tv if t > 5e-3)
    return {
        "workload": "learned_surrogate_256x512", "model": S.DEFAULT_MODEL.name, "records": n, "records_per_call": R,
        "cells": [nt, np_],
        "storage": [ct, cp], "network": {"hidden": H, "layers": 4, "input_width": K0, "dtype": "bf16 weights and "
                                         "activations, fp32 accumulation (tcgen05, TMEM)"},
        "surrogate_records_per_s": n / t_sur, "served_records_per_s": n / t_serve,
        "served_by_surrogate": served["surrogate"], "served_by_tracer": served["tracer"],
        "plain_tracer_records_per_s": n / t_plain,
        "speedup_served_vs_plain": t_plain / t_serve, "speedup_surrogate_only_vs_plain": t_plain / t_sur,
        "kernel_launches_per_serve": launches,
        "heldout": {"records": len(tv), "truth_rays": 1e8, "tv_storage_mean": ev["storage"]["tv_mean"],
                    "tv_storage_median": ev["storage"]["tv_median"], "truth_floor_storage": ev["storage"]["floor_mean"],
                    "tv_cells_mean": ev["cells"]["tv_mean"], "truth_floor_cells": ev["cells"]["floor_mean"],
                    "pass_fraction_tv_5e-3": ev["pass_fraction"],
                    "gate_serves_by_surrogate": len(served_tv),
                    "served_out_of_tolerance": served_bad,
                    "served_out_of_tolerance_fraction": served_bad / max(1, len(served_tv)),
                    "served_tv_storage_max": max(served_tv) if served_tv else None},
        "roofline_forward": {"kernel": "features_kernel + mlp_fused_kernel (forward pass: input rows, three layers and head in one kernel)", "bound": "tensor",
                             "achieved": flops / t_fwd / 1e12, "peak": bf16, "unit": "TFLOP/s",
                             "frac": flops / t_fwd / 1e12 / bf16, "records": nf, "ms": 1e3 * t_fwd,
                             "peak_note": "MEASURED_PEAKS.json bf16_tflops (of measured)"},
    }


def run_atlas(I, ctx, stream, a) -> dict:
    """Deterministic atlas composition at the record grid: a 28-node atlas of the hex column
    (6 x 3 incident intervals, 900 x 1800 cells, S = 2 area quadrature, n from the ice table at
    550 nm) traced on the device, then per incident inclination the coupling of the reference's
    horizontal_gaussian rule (16 x 8 x 12 nodes, two components), the cyclic composition and the
    stored CDF, device-resident; the composition kernel against the FP64 pipe; the NumPy
    composition of the oracle (the reference's algorithm) on the host as the CPU baseline."""
    import ctypes as C

    import numpy as np
    import torch

    from ice_crystal_phase_b200 import atlas as A

    nt, np_ = DROP["nt"], DROP["np"]
    s = A.settings(0.05, 0.2, I.evaluate_ice_optics(550.0).n, 6, 3, nt, np_, 2)
    nodes = (s.theta_intervals + 1) * (s.phi_intervals + 1)
    d_mass = torch.empty(nodes * nt * np_, dtype=torch.float64, device="cuda")
    area = np.empty(nodes)
    residual = np.empty(nodes)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for n in range(nodes):
        i, j = divmod(n, s.phi_intervals + 1)
        rep = I.AtlasNodeReport()
        I.check(I.LIB.icp_atlas_trace_node(ctx.handle, C.byref(s), i, j,
                                           C.c_void_p(d_mass.data_ptr() + 8 * n * nt * np_), C.byref(rep)))
        area[n], residual[n] = rep.projected_area_mm2, rep.unresolved_mm2
    t_atlas = time.perf_counter() - t0
    rule = {"quadrature": {"azimuth": 16, "tilt": 8, "spin": 12},
            "components": [{"kind": "horizontal_gaussian", "sigma_deg": 10, "fraction": 0.9},
                           {"kind": "isotropic", "fraction": 0.1}]}
    rot, w, _ = A.orientation_rule(rule)
    d_rot = torch.from_numpy(np.ascontiguousarray(rot.reshape(-1, 9))).cuda()
    d_w = torch.from_numpy(w).cuda()
    incl = [0.0, 15.0, 30.0, 45.0, 60.0, 75.0][: max(1, a.atlas_incidents)]
    coupling = torch.empty(nodes * 2 * np_, dtype=torch.float64, device="cuda")
    out = torch.empty(nt * np_, dtype=torch.float64, device="cuda")
    phi = torch.empty(np_ + 1, dtype=torch.float64, device="cuda")
    theta = torch.empty(np_ * (nt + 1), dtype=torch.float64, device="cuda")
    policy = I.CdfPolicy(1e-10, 1e-12, 1.0)
    areas = (C.c_double * nodes)(*area)
    nnz = []

    def record(alpha: float, keep: bool = False) -> None:
        k = (C.c_double * 3)(math.cos(math.radians(alpha)), -math.sin(math.radians(alpha)), 0.0)
        coupling.zero_()
        exp = C.c_double()
        I.check(I.LIB.icp_atlas_coupling(ctx.handle, s.theta_intervals, s.phi_intervals, np_, s.circumradius_mm,
                                         s.length_mm, areas, C.c_void_p(d_rot.data_ptr()), C.c_void_p(d_w.data_ptr()),
                                         len(w), k, 1.0, 0, C.c_void_p(coupling.data_ptr()), C.byref(exp)))
        if keep:
            nnz.append(int((coupling > 0).sum()))
        I.check(I.LIB.icp_atlas_compose(ctx.handle, nodes, nt, np_, C.c_void_p(d_mass.data_ptr()),
                                        C.c_void_p(coupling.data_ptr()), C.c_void_p(out.data_ptr())))
        crep = I.CdfReport()
        I.check(I.LIB.icp_phase_cdf_build(ctx.handle, C.c_void_p(out.data_ptr()), 0, nt, np_, 0.0, 0.0, nt, np_,
                                          C.byref(policy), C.c_void_p(phi.data_ptr()), C.c_void_p(theta.data_ptr()),
                                          C.byref(crep)))

    for alpha in incl:
        record(alpha, keep=True)  # warm-up, nonzero weights per incidence
    launches0 = I.kernel_launches()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for alpha in incl:
        record(alpha)
    e1.record(stream)
    torch.cuda.synchronize()
    t_rec = e0.elapsed_time(e1) / 1e3 / len(incl)
    launches = (I.kernel_launches() - launches0) // len(incl)
    # the composition kernel alone, on the last incidence's weights
    ck = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        I.check(I.LIB.icp_atlas_compose(ctx.handle, nodes, nt, np_, C.c_void_p(d_mass.data_ptr()),
                                        C.c_void_p(coupling.data_ptr()), C.c_void_p(out.data_ptr())))
        e1.record(stream)
        torch.cuda.synchronize()
        ck.append(e0.elapsed_time(e1) / 1e3)
    flops = 2.0 * nnz[-1] * nt * np_
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    fp64_peak = 40.0  # nominal B200 FP64 TFLOP/s (no measured FP64 figure)
    cpu = None
    if not a.no_cpu_baseline:
        try:
            # the reference's NumPy composition (the oracle's restatement, in a child process) on a
            # bounded sample of 64 nonzero weights over this atlas's shape; its cost per weight does
            # not depend on the values, so it is scaled to all the composition's weights
            r = _cpu_leg("atlas_compose", {"nodes": nodes, "nt": nt, "np": np_, "weights": 64})
            t_cpu = r["seconds"] * nnz[-1] / r["weights"]
            cpu = {"value": 1.0 / t_cpu, "unit": "compositions/s", "cores": 1, "kind": "port",
                   "sample": f"{r['weights']} of {nnz[-1]} nonzero weights of one composition ({nodes} nodes, "
                             f"{nt}x{np_}) as NumPy rolls in the reference's order, scaled to all weights"}
        except (RuntimeError, ValueError, OSError) as e:
            cpu = {"value": None, "unit": "compositions/s", "cores": 0, "kind": "port", "sample": f"unavailable: {e}"}
    # the reference's CPU precompute on a bounded sample: the 4 nodes of 1 x 1 intervals at the
    # same grid (--batch-rays 16 keeps its per-ray columns within its 512 MiB default)
    cpu_pre = None
    ref_exe = ROOT / "oracle" / "_ref" / "ice_precompute_atlas_cpu"
    if not a.no_cpu_baseline and ref_exe.exists():
        with tempfile.TemporaryDirectory() as td:
            t0 = time.perf_counter()
            r = subprocess.run([str(ref_exe), "--out", str(Path(td) / "a"), "--radius-mm", "0.05", "--length-mm", "0.2",
                                "--wavelength-nm", "550", "--incident-theta-intervals", "1",
                                "--incident-phi-intervals", "1", "--theta", str(nt), "--phi", str(np_),
                                "--area-subdivisions", "2", "--batch-rays", "16"], capture_output=True, text=True)
            t_ref = time.perf_counter() - t0
        if r.returncode == 0:
            cpu_pre = {"value": 4 / t_ref, "unit": "atlas nodes/s", "cores": 1, "kind": "reference",
                       "sample": "reference ice_precompute_atlas_cpu, 4 nodes (1 x 1 intervals), 900x1800, S = 2",
                       "gpu_nodes_per_s": nodes / t_atlas}
    return {"workload": "hex_column_atlas_28_nodes_900x1800_horizontal_gaussian", "nodes": nodes,
            "cells": [nt, np_], "rotations": len(w), "incidences": incl, "atlas_trace_s": t_atlas,
            "ms_per_record": 1e3 * t_rec, "records_per_s": 1.0 / t_rec, "kernel_launches_per_record": launches,
            "nonzero_weights": nnz,
            "roofline_compose": {"kernel": "atlas_compose_kernel", "bound": "fp64", "achieved": flops / min(ck) / 1e12,
                                 "peak": fp64_peak, "unit": "TFLOP/s", "frac": flops / min(ck) / 1e12 / fp64_peak,
                                 "kernel_ms": 1e3 * min(ck), "sms": sms,
                                 "peak_note": "nominal FP64 (separate mul and add; no measured FP64 peak)"},
            "cpu_baseline": cpu, "cpu_baseline_precompute": cpu_pre}


def run_rainbow(I, ctx, stream, a) -> dict:
    """Table-II rainbow diffraction on the drop records' 1800 x 3600 query grid (0.1 degree
    cells; a seeded synthetic focal grid with wobbling primary and secondary bows, radius
    0.5 mm -> sigma 0.22 / 0.44 degrees): both passes through the C ABI, device-resident, timed
    on the context's stream; the oracle's detect and a uniform sample of its filter as the CPU
    baseline."""
    import ctypes as C

    import numpy as np
    import torch

    sys.path.insert(0, str(ROOT / "tests"))
    import rainbow_cases as RC

    nt, np_ = 1800, 3600
    n = nt * np_
    focal = RC.bow_grid(nt, np_, 31, noise=0.2)
    cfg = I.diffraction_config(0.5)
    d_focal = I.DeviceArray(ctx, n, I.FOCAL_DTYPE).upload(focal)
    d_edges = I.DeviceArray(ctx, n, np.uint32)
    d_res = I.DeviceArray(ctx, n, I.DIFFRACTION_DTYPE)
    d_den = I.DeviceArray(ctx, n)
    stats = I.DiffractionStats()

    def once() -> None:
        I.check(I.LIB.icp_rainbow_diffraction(ctx.handle, d_focal.ptr, nt, np_, C.byref(cfg), d_edges.ptr, d_res.ptr,
                                              d_den.ptr, C.byref(stats)))

    for _ in range(3):
        once()
    launches0 = I.kernel_launches()
    times = []
    for _ in range(max(1, a.rainbow_steps)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        once()
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    launches = (I.kernel_launches() - launches0) // max(1, a.rainbow_steps)
    t = sorted(times)[len(times) // 2]
    # algorithmic bytes per direction: the focal fields read (s, p, flags, TRT / TRRT hits and
    # incoherent: 44 B), labels and packed samples written and read back (2 x 20 B), result and
    # density written (48 B)
    bytes_per_dir = 44 + 40 + 48
    hbm = _peaks().get("hbm_gbs") or 6650.0
    cpu = None
    if not a.no_cpu_baseline:
        try:
            c4 = [cfg.primary_sigma_rad, cfg.support_sigma, cfg.transition_contrast, cfg.inner_blend_sigma]
            r = _cpu_leg("rainbow", {"nt": nt, "np": np_, "config": c4, "picks": 20000})
            cpu = {"value": n / (r["detect_seconds"] + r["filter_seconds"] * n / r["picks"]), "unit": "directions/s",
                   "cores": 1, "kind": "port",
                   "sample": "oracle detect over the whole grid + its filter at 20000 uniform random directions, "
                             "scaled to the grid (child process)"}
        except (RuntimeError, ValueError, OSError) as e:
            cpu = {"value": None, "unit": "directions/s", "cores": 0, "kind": "port", "sample": f"unavailable: {e}"}
    return {"workload": "rainbow_table2_1800x3600_r0.5mm", "directions": n, "ms_per_pass": 1e3 * t,
            "directions_per_s": n / t, "kernel_launches_per_pass": launches, "stats": {
                k: getattr(stats, k) for k, _ in stats._fields_},
            "roofline": {"bound": "hbm", "achieved": bytes_per_dir * n / t / 1e9, "peak": hbm, "unit": "GB/s",
                         "frac": bytes_per_dir * n / t / 1e9 / hbm,
                         "note": "whole pass (detect + filter + counters) against the algorithmic bytes; the "
                                 "filtered band is FP64-bound (sin, asin, exp per neighbour)"},
            "cpu_baseline": cpu}


def run_wave(I, ctx, stream, a) -> dict:
    """One wave-stage record of a real drop at the reference CLI's defaults (1.0 mm Table-I drop,
    650 nm water, inclination 20 deg, 513 x 513 lattice, 360 x 720 query grid, diffraction
    stage): lattice trace, patch build, all-hit query (sizing and fill passes), folded-patch
    records, patch optics with the focal stage, Table-II diffraction, stage density and the stored
    CDF, every stage timed with CUDA events on the context's stream."""
    import ctypes as C

    import numpy as np
    import torch

    w = h = 513
    nt, np_ = 360, 720
    n_int = float(np.float32(I.evaluate_water_optics(650.0).refractive_index))
    alpha = math.radians(20.0)
    cfg = I.raindrop_config(1.0, 650.0, n_int, (math.cos(alpha), -math.sin(alpha), 0.0), w)
    e = cfg.grid_half_extent
    k = np.array([cfg.incident_direction.x, cfg.incident_direction.y, cfg.incident_direction.z], np.float32)
    e0 = np.array([cfg.incident_basis_x.x, cfg.incident_basis_x.y, cfg.incident_basis_x.z], np.float32)
    dirs = I.query_directions(nt, np_, k, e0)
    nv, n, cells = 4 * w * h, nt * np_, 4 * (w - 1) * (h - 1)
    dv, d2 = I.DeviceArray(ctx, nv, I.VERTEX_DTYPE), I.DeviceArray(ctx, 4 * nv, np.float32)
    dp, db = I.DeviceArray(ctx, cells, I.PATCH_DTYPE), I.DeviceArray(ctx, cells, I.AABB_DTYPE)
    dd = I.DeviceArray(ctx, 3 * n, np.float32).upload(dirs.reshape(-1))
    do, ds = I.DeviceArray(ctx, n + 1, np.uint64), I.DeviceArray(ctx, n, I.SUMMARY_DTYPE)
    dr, df = I.DeviceArray(ctx, n, I.OPTICAL_DTYPE), I.DeviceArray(ctx, n, I.FOCAL_DTYPE)
    dt, dres, dden = I.DeviceArray(ctx, n, np.uint32), I.DeviceArray(ctx, n, I.DIFFRACTION_DTYPE), I.DeviceArray(ctx, n)
    dphi, dth = I.DeviceArray(ctx, np_ + 1), I.DeviceArray(ctx, np_ * (nt + 1))
    di = I.DeviceArray(ctx, cells, np.uint32)
    npatch, hits, nrec = C.c_uint32(0), C.c_uint64(0), C.c_uint32(0)
    hist = (C.c_uint64 * 8)()
    dcfg = I.diffraction_config(1.0)
    fc = I.FocalConfig(w, h, e, 0, (C.c_uint32 * 4)(0, 0, 0, 0))
    lstats, fstats, dstats = I.LatticeStats(), I.FoldedStats(), I.DiffractionStats()
    drep, crep = I.DensityReport(), I.CdfReport()
    pol = I.CdfPolicy(1e-10, 1e-12, 1.0)
    kin = (C.c_float * 3)(*map(float, k))
    state = {}

    def trace():
        I.check(I.LIB.icp_lattice_trace(ctx.handle, C.byref(cfg), dv.ptr, d2.ptr, C.byref(lstats)))

    def build():
        I.check(I.LIB.icp_patch_build(ctx.handle, dv.ptr, w, h, e, dp.ptr, db.ptr, None, C.byref(npatch), hist))

    def query():
        # one call counts and fills when the hits fit (four per direction to start with)
        args = (ctx.handle, dv.ptr, nv, dp.ptr, db.ptr, npatch.value, dd.ptr, n, do.ptr)
        if "dh" not in state:
            state["dh"] = I.DeviceArray(ctx, 4 * n, I.HIT_DTYPE)
        st = I.LIB.icp_patch_query(*args, ds.ptr, state["dh"].ptr, state["dh"].count, C.byref(hits))
        if st == I.ICP_ERR_CAPACITY:
            state["dh"] = I.DeviceArray(ctx, hits.value, I.HIT_DTYPE)
            st = I.LIB.icp_patch_query(*args, ds.ptr, state["dh"].ptr, state["dh"].count, C.byref(hits))
        I.check(st)

    def folded():
        args = (ctx.handle, dv.ptr, nv, dp.ptr, npatch.value, kin, C.byref(fc), None, di.ptr)
        if "dfr" not in state:
            I.LIB.icp_folded_prepare(*args, None, 0, C.byref(nrec), C.byref(fstats))
            state["dfr"] = I.DeviceArray(ctx, max(1, nrec.value), I.FOLDED_DTYPE)
        I.check(I.LIB.icp_folded_prepare(*args, state["dfr"].ptr, state["dfr"].count, C.byref(nrec), C.byref(fstats)))

    def optics():
        inp = I.OpticsInput(dv.ptr, dp.ptr, dd.ptr, do.ptr, ds.ptr, state["dh"].ptr, d2.ptr, hits.value, nv,
                            npatch.value, n, nv, I.Vec3f(*map(float, k)), I.Vec3f(*map(float, e0)), 1, 0)
        view = I.FoldedView(di.ptr, state["dfr"].ptr, npatch.value, nrec.value)
        I.check(I.LIB.icp_patch_optics_folded(ctx.handle, C.byref(inp), dr.ptr, C.byref(fc), df.ptr,
                                              C.byref(view) if nrec.value else None))

    def diffraction():
        I.check(I.LIB.icp_rainbow_diffraction(ctx.handle, df.ptr, nt, np_, C.byref(dcfg), dt.ptr, dres.ptr, None,
                                              C.byref(dstats)))

    def density():
        I.check(I.LIB.icp_stage_density(ctx.handle, I.WAVE_STAGES["diffraction"], dr.ptr, df.ptr, dres.ptr, n,
                                        dden.ptr, C.byref(drep)))

    def cdf():
        I.check(I.LIB.icp_phase_cdf_build(ctx.handle, dden.ptr, 1, nt, np_, 0.0, 0.0, nt, np_, C.byref(pol), dphi.ptr,
                                          dth.ptr, C.byref(crep)))

    stages = {"lattice_trace": trace, "patch_build": build, "patch_query": query, "folded_prepare": folded,
              "patch_optics": optics, "rainbow_diffraction": diffraction, "stage_density": density, "cdf_build": cdf}
    for _ in range(3):
        for f in stages.values():
            f()
    ms = {}
    for name, f in stages.items():
        times = []
        for _ in range(max(1, a.wave_steps)):
            e0v, e1v = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0v.record(stream)
            f()
            e1v.record(stream)
            torch.cuda.synchronize()
            times.append(e0v.elapsed_time(e1v))
        ms[name] = sorted(times)[len(times) // 2]
    total = sum(ms.values())
    # the reference's CDF input gate; the 1.0 mm drop's Table-II width (0.15 deg) is below twice the
    # 0.5 deg cell, so its bow directions are underresolved and the record is the one written
    # with --allow-underresolved
    gate = drep.invalid_values == 0 and drep.incomplete == 0 and drep.maximum > 0
    out = {"workload": "drop_diffraction_record_1.0mm_650nm_lattice_513x513_query_360x720", "lattice": [w, h],
           "query": [nt, np_], "patches": npatch.value, "patch_status_histogram": list(hist), "hits": hits.value,
           "folded_records": nrec.value, "folded": fstats.as_dict(), "trace_incomplete": lstats.incomplete,
           "density_gate_passed_allowing_underresolved": bool(gate), "incomplete_directions": drep.incomplete,
           "underresolved_directions": drep.underresolved,
           "cdf_g": crep.g_stored, "cdf_l1": crep.l1_error,
           "ms_per_stage": ms, "ms_per_record": total, "records_per_s": 1e3 / total,
           "filtered_directions": dstats.filtered_directions}
    # the reference's own CPU lattice trace (RaindropPathTracer, its only CPU stage of this chain)
    # on a few rows of the same lattice, one process per core, beside the device trace
    if not a.no_cpu_baseline and (ROOT / "oracle" / "_ref" / "ref_drop_harness").exists():
        try:
            out["cpu_baseline_lattice_trace"] = reference_lattice_rows(w, n_int)
            out["cpu_baseline_lattice_trace"]["device_vertices_per_s"] = w * h / (ms["lattice_trace"] / 1e3)
        except (OSError, ValueError, subprocess.SubprocessError) as ex:
            out["cpu_baseline_lattice_trace"] = {"unavailable": f"{type(ex).__name__}: {ex}"}
    return out


def reference_lattice_rows(grid: int, n_int: float, rows_per_proc: int = 2) -> dict:
    """The reference's CPU lattice trace (oracle/_ref/ref_drop_harness time: RaindropPathTracer::
    trace_vertex_unpolarized with its RaindropIntersector) of `rows_per_proc` rows per process from
    the middle of the same 1.0 mm drop's lattice, one process per core: vertices per second."""
    import numpy as np

    procs = os.cpu_count() or 1
    alpha = math.radians(20.0)
    k = (repr(float(np.float32(math.cos(alpha)))), repr(float(np.float32(-math.sin(alpha)))), "0")
    base = grid // 2 - (procs * rows_per_proc) // 2
    cmds = [[str(ROOT / "oracle" / "_ref" / "ref_drop_harness"), "time", "1.0", "0", repr(n_int), *k, str(grid),
             str(max(0, base + p * rows_per_proc)), str(rows_per_proc)] for p in range(procs)]
    t0 = time.perf_counter()
    ps = [subprocess.Popen(c, stdout=subprocess.PIPE, text=True) for c in cmds]
    outs = [p.communicate()[0].split() for p in ps]
    wall = time.perf_counter() - t0
    verts = sum(int(o[0]) for o in outs)
    per_proc = [int(o[0]) / float(o[2]) for o in outs]
    return {"value": verts / wall, "unit": "lattice vertices/s", "cores": procs, "kind": "reference",
            "one_core": sum(per_proc) / len(per_proc),
            "sample": f"{verts} vertices ({rows_per_proc} lattice rows per process, {procs} processes) of the "
                      "513 x 513 lattice through the reference's RaindropPathTracer compiled from its sources"}


def _cpu_leg(kind: str, payload: dict) -> dict:
    """Runs one CPU-side leg (the reference CPU baseline sample or the oracle parity check) in a
    child process, so that the oracle library never loads into the process that measures the
    device; returns its JSON result."""
    r = subprocess.run([sys.executable, str(Path(__file__).resolve()), "--cpu-leg", kind, "--cpu-leg-args",
                        json.dumps(payload)], capture_output=True, text=True, cwd=str(ROOT))
    if r.returncode != 0:
        raise RuntimeError(f"{kind} leg failed: {(r.stderr or r.stdout).strip().splitlines()[-1:]}")
    return json.loads(r.stdout.strip().splitlines()[-1])


def run_cpu_leg(kind: str, payload: dict) -> None:
    """Child side of _cpu_leg: the oracle and the reference binaries are used here only."""
    if kind == "drop_reference":
        inputs = _drop_reference_inputs()
        out = reference_drop_sample(int(payload["rays_per_proc"]), int(payload["procs"]), inputs)
    elif kind == "drop_parity":
        import numpy as np

        from oracle import parity

        z = np.load(payload["npz"], allow_pickle=False)
        out = parity.drop_parity(z["masses"], json.loads(str(z["cfg"])), json.loads(str(z["audit"])))
    elif kind == "atlas_compose":
        import numpy as np

        from oracle import atlas_oracle as AO

        rng = np.random.default_rng(5)
        nodes, nt, np_ = int(payload["nodes"]), int(payload["nt"]), int(payload["np"])
        mass = rng.random((nodes, nt, np_))
        w = np.zeros((nodes, 2, np_))
        w.flat[rng.choice(w.size, int(payload["weights"]), replace=False)] = rng.random(int(payload["weights"]))
        t0 = time.perf_counter()
        AO.compose(mass, w)
        out = {"seconds": time.perf_counter() - t0, "weights": int(payload["weights"])}
    elif kind == "rainbow":
        import numpy as np

        sys.path.insert(0, str(ROOT / "tests"))
        import rainbow_cases as RC

        from oracle import oracle as O

        nt, np_ = int(payload["nt"]), int(payload["np"])
        focal = RC.bow_grid(nt, np_, 31, noise=0.2)
        c4 = tuple(payload["config"])
        t0 = time.perf_counter()
        edges = O.rainbow_detect(focal, nt, np_, c4)
        t_det = time.perf_counter() - t0
        pick = np.random.default_rng(9).integers(0, nt * np_, int(payload["picks"]))
        t0 = time.perf_counter()
        O.rainbow_filter_at(focal, edges, nt, np_, c4, pick)
        out = {"detect_seconds": t_det, "filter_seconds": time.perf_counter() - t0, "picks": int(pick.size)}
    else:
        raise ValueError(kind)
    print(json.dumps(out), flush=True)


def drop_parity_leg(I, ctx, rec, g, edges, mass, weight: float, count: int) -> dict:
    """Same-seed parity of the timed record: the first `count` ray ids of the record traced again
    by the FP32 kernel (outside the timed region) and checked against the FP64 oracle on the same
    ray ids in a child process (TV of cell mass, g, energy, Monte Carlo noise floor)."""
    import ctypes as C

    import numpy as np

    d = DROP
    nt, np_ = d["nt"], d["np"]
    mass.zero_()
    s = I.TraceStats()
    I.check(I.LIB.icp_drop_trace_bin(ctx.handle, C.byref(rec), 0, count, weight, C.byref(g),
                                     C.c_void_p(edges.data_ptr()), C.c_void_p(mass.data_ptr()), C.byref(s)))
    m = mass.cpu().numpy().reshape(nt, np_).copy()
    m[0] += weight * s.forward_pole / np_
    m[-1] += weight * s.backward_pole / np_
    cfg = {"coefficients": list(d["coefficients"]), "radius_mm": d["radius"], "interior_index": rec.interior_index,
           "inclination_deg": d["incl"], "nt": nt, "np": np_, "rays": int(rec.rays), "seed": d["seed"],
           "max_internal_hits": d["hits"], "first": 0, "count": count}
    audit = {"escaped": weight * s.escaped, "unresolved": weight * s.unresolved,
             "incident": weight * (s.rays - s.missed), "missed": s.missed}
    with tempfile.TemporaryDirectory() as td:
        path = str(Path(td) / "slice.npz")
        np.savez(path, masses=m.reshape(-1), cfg=json.dumps(cfg), audit=json.dumps(audit))
        return _cpu_leg("drop_parity", {"npz": path})


def cdf_kernel_times(I, ctx, stream, values, nt: int, np_: int, phi, theta, flush, policy, launches: int = 5) -> list:
    """Device time of the CDF kernel alone: icp_phase_cdf_enqueue puts one cooperative kernel on
    the library's stream (the grid's u edges are already on the device after the first build, and
    the barrier counters are left at zero by every build), bracketed by CUDA events on that
    stream; the L2 is flushed before each launch.  A short spin kernel ahead of the first event
    keeps the stream busy while the host enqueues, so the events bracket the kernel and not the
    host's launch latency.  The report is then checked through icp_phase_cdf_result."""
    import ctypes as C

    import torch

    args = (ctx.handle, C.c_void_p(values.data_ptr()), 0, nt, np_, 0.0, 0.0, nt, np_, C.c_void_p(phi.data_ptr()),
            C.c_void_p(theta.data_ptr()))
    rep = I.CdfReport()
    I.check(I.LIB.icp_phase_cdf_build(*args[:9], C.byref(policy), *args[9:], C.byref(rep)))
    times = []
    for _ in range(launches):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            torch.cuda._sleep(200_000)  # about 0.1 ms of device time
        e0.record(stream)
        I.check(I.LIB.icp_phase_cdf_enqueue(*args))
        e1.record(stream)
        I.check(I.LIB.icp_phase_cdf_result(ctx.handle, C.byref(policy), C.byref(rep)))
        times.append(e0.elapsed_time(e1) / 1e3)
    return times


def _peaks() -> dict:
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        return {}


def run_b200_drop(a) -> None:
    import ctypes as C

    import numpy as np
    import torch

    import ice_crystal_phase_b200 as I

    rank, world, local = _env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    ctx = I.Context(local)
    stream = torch.cuda.ExternalStream(I.LIB.icp_context_stream(ctx.handle))
    torch.cuda.set_stream(stream)
    d = DROP
    nt, np_ = d["nt"], d["np"]
    rays = int(a.rays)
    n_int = float(np.float32(I.evaluate_water_optics(d["wavelength"]).refractive_index))
    tuning = I.Tuning(a.block_threads, 0, a.hash_slots, 0)
    rec = I._drop_args(d["coefficients"], d["radius"], d["incl"], n_int, rays * world, d["seed"], nt, np_, nt, np_,
                       1.0, d["hits"], 1e-12, I.ICP_FP32, 1e-10, d["wavelength"], True, tuning=tuning)
    grid = I.make_drop_grid(nt, np_, d["incl"])
    g = grid.abi()
    edges = torch.from_numpy(grid.edges).cuda()
    mass = torch.zeros(nt * np_, dtype=torch.float64, device="cuda")
    phi = torch.empty(np_ + 1, dtype=torch.float64, device="cuda")
    theta = torch.empty(np_ * (nt + 1), dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    weight = I.sampling_area(d["coefficients"], d["radius"]) / float(rays * world)
    policy = rec.policy
    from ice_crystal_phase_b200 import sharded

    shard_trace, shard_finish, shard_sums, disk = sharded.device_record(ctx, rec, grid, edges, mass)
    shard = sharded.shard_of(rays * world, rank, world, disk)
    last_trace = {}

    def traced(first: int, count: int):
        t = shard_trace(first, count)
        last_trace["t"] = t
        return t

    def step():
        """One record; returns (trace summary of this rank, record report or None)."""
        if world == 1:
            rep = I.DropReport()
            I.check(I.LIB.icp_drop_generate_device(ctx.handle, C.byref(rec), C.c_void_p(phi.data_ptr()),
                                                   C.c_void_p(theta.data_ptr()), None, C.byref(rep)))
            return rep.trace, rep
        sharded.sharded_drop_record(shard, traced, dist.all_reduce, shard_finish, shard_sums)
        return last_trace["t"], None

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(a.warmup):
        step()
    launches0 = I.kernel_launches()
    times, stats_all, reps = [], [], []
    with ClockSampler(local) as clocks:
        for _ in range(a.steps):
            flush.fill_(1.0)
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st, rp = step()
            e1.record(stream)
            barrier()
            times.append(e0.elapsed_time(e1) / 1e3)
            stats_all.append(st)
            reps.append(rp)
    launches = I.kernel_launches() - launches0
    t_local = torch.tensor([sum(times)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t_local, op=dist.ReduceOp.MAX)
    t_step = float(t_local) / a.steps
    value = rays * world / t_step

    # dominant kernel alone (drop trace+bin, FP32) on the same stream, for the roofline
    k_times, ks = [], None
    for _ in range(2):
        flush.fill_(1.0)
        barrier()
        mass.zero_()
        ks = I.TraceStats()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        I.check(I.LIB.icp_drop_trace_bin(ctx.handle, C.byref(rec), rank * rays, rays, weight, C.byref(g),
                                         C.c_void_p(edges.data_ptr()), C.c_void_p(mass.data_ptr()), C.byref(ks)))
        e1.record(stream)
        barrier()
        k_times.append(e0.elapsed_time(e1) / 1e3)
    t_kernel = min(k_times)
    hits = ks.rays - ks.missed
    flops = (FLOP_DROP_RAY * ks.rays + FLOP_DROP_ENTRY * hits + FLOP_DROP_INTERACTION * ks.encounters
             + FLOP_DROP_GAUGE * ks.gauge_evals)
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    clk = clocks.summary()
    mhz = clk["sm_mhz"] or 1965.0
    fp32_peak = sms * 128 * 2 * mhz * 1e6 / 1e12
    achieved = flops / t_kernel / 1e12

    cdf_bytes = 8 * nt * np_ + 8 * np_ * (nt + 1) + 8 * (np_ + 1)
    cdf_t = cdf_kernel_times(I, ctx, stream, mass, nt, np_, phi, theta, flush, policy) if rank == 0 else []
    hbm = _peaks().get("hbm_gbs", 6650.0)

    # e2e through the public host-buffer entry (one whole record per step, N=1)
    e2e_value = None
    ph = torch.empty(np_ + 1, dtype=torch.float64).pin_memory()
    th = torch.empty(np_ * (nt + 1), dtype=torch.float64).pin_memory()
    uh = torch.empty(nt + 1, dtype=torch.float64).pin_memory()
    if world == 1:
        e2e_times = []
        for i in range(a.steps + 1):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            rr = I.DropReport()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            I.check(I.LIB.icp_drop_generate(ctx.handle, C.byref(rec), C.cast(C.c_void_p(ph.data_ptr()), I._D),
                                            C.cast(C.c_void_p(th.data_ptr()), I._D),
                                            C.cast(C.c_void_p(uh.data_ptr()), I._D), C.byref(rr)))
            e1.record(stream)
            torch.cuda.synchronize()
            if i:
                e2e_times.append(e0.elapsed_time(e1) / 1e3)
        e2e_value = rays / (sum(e2e_times) / len(e2e_times))
    h2d = 8 * (nt + 1) + 8 * nt  # u edges + diffraction rows
    d2h = 8 * (np_ + 1) + 8 * np_ * (nt + 1) + 256 + 128  # CDF + trace counters + CDF report

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            procs = os.cpu_count() or 1
            per = max(100, int(a.ref_rays) // procs)
            rb = _cpu_leg("drop_reference", {"rays_per_proc": per, "procs": procs})
            r1 = _cpu_leg("drop_reference", {"rays_per_proc": per, "procs": 1})
            cpu = {"value": rb["rays_per_s"], "unit": "rays/s", "cores": rb["procs"], "kind": "reference",
                   "one_core": r1["rays_per_s"],
                   "sample": f"{rb['rays']} rays of this record ({per} per process, {procs} processes, "
                             f"{rb['seconds']:.1f} s; one core: {r1['rays']} rays in {r1['seconds']:.1f} s), <= 10 "
                             "internal interactions, every exit binned, one 900x1800 stored CDF per sample; the "
                             "reference's RaindropIntersector, DielectricInterface::split, PhaseMassAccumulator and "
                             "build_host_cdf compiled from its sources"}
        except (OSError, ValueError, IndexError, RuntimeError) as e:
            cpu = {"value": None, "unit": "rays/s", "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}

    batched = None
    if world == 1 and a.batch_records > 0:
        batched = run_batched(I, ctx, stream, a, nt, np_)
    surrogate = None
    if world == 1 and a.surrogate_records > 0:
        surrogate = run_surrogate(I, ctx, stream, a)
    atlas = None
    if world == 1 and a.atlas_incidents > 0:
        try:
            atlas = run_atlas(I, ctx, stream, a)
        except (I.IcpError, RuntimeError, ValueError, OSError) as e:  # reported on the line, not fatal to it
            atlas = {"error": f"{type(e).__name__}: {e}"}

    rainbow = None
    if world == 1 and a.rainbow_steps > 0:
        try:
            rainbow = run_rainbow(I, ctx, stream, a)
        except (I.IcpError, RuntimeError, ValueError, OSError) as e:  # reported on the line, not fatal to it
            rainbow = {"error": f"{type(e).__name__}: {e}"}

    wave = None
    if world == 1 and a.wave_steps > 0:
        try:
            wave = run_wave(I, ctx, stream, a)
        except (I.IcpError, RuntimeError, ValueError, OSError) as e:  # reported on the line, not fatal to it
            wave = {"error": f"{type(e).__name__}: {e}"}

    parity = None
    if rank == 0 and world == 1 and a.parity_rays > 0:
        try:
            parity = drop_parity_leg(I, ctx, rec, g, edges, mass, weight, int(a.parity_rays))
        except (I.IcpError, RuntimeError, ValueError, OSError) as e:  # reported on the line, not fatal to it
            parity = {"error": f"{type(e).__name__}: {e}"}

    s0 = stats_all[-1] if world == 1 else ks
    r0 = reps[-1]
    line = {
        "metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * t_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "oblate_drop_1.5mm_1e8_rays_900x1800", **_drop_public(), "interior_index": n_int,
                   "rays_per_gpu": rays, "l2": "flushed between timed steps (256 MiB write)", "trace_precision": "fp32",
                   "parallelism": f"ray shards x{world}, NCCL all-reduce of FP64 histogram" if world > 1 else "1 GPU"},
        "records_per_s": 1.0 / t_step,
        "e2e": {"value": e2e_value, "unit": "rays/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": {"kernel": "trace_bin_kernel<float, DropGeo<float>>", "bound": "fp32_simt", "achieved": achieved,
                     "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                     "traffic": DROP_TRACE_TRAFFIC if rays == 1e8 else None,
                     "traffic_note": "DRAM bytes of one 1e8-ray launch (ncu, one pass): 14.2 MB read, 2.3 MB "
                                     "written, against 13.0 MB algorithmic (the FP64 histogram)",
                     "peak_note": f"derived: {sms} SMs x 128 FP32 lanes x 2 x {mhz:.0f} MHz (median SM clock under load)",
                     "flops_per_ray": flops / max(1, ks.rays), "kernel_ms": 1e3 * t_kernel,
                     "interactions_per_hit": ks.encounters / max(1, hits),
                     "gauge_evaluations_per_hit": ks.gauge_evals / max(1, hits)},
        "roofline_cdf": ({"kernel": "cdf_build_kernel", "bound": "hbm", "achieved": cdf_bytes / statistics.mean(cdf_t) / 1e9,
                          "peak": hbm, "unit": "GB/s", "frac": cdf_bytes / statistics.mean(cdf_t) / 1e9 / hbm,
                          "traffic": DROP_CDF_TRAFFIC if (nt, np_) == (900, 1800) else None,
                          "traffic_note": "DRAM bytes of one launch (ncu): the 13.1 MB histogram read; the "
                                          "13 MB of a / T output stay in L2 during the launch",
                          "algorithmic_bytes": cdf_bytes, "kernel_us": 1e6 * statistics.mean(cdf_t), "kernel_us_min": 1e6 * min(cdf_t),
                          "peak_note": "MEASURED_PEAKS.json hbm_gbs (of measured)"} if cdf_t else None),
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": launches,
        "trace": {"outputs_per_ray": s0.outputs / max(1, s0.rays), "missed_fraction": s0.missed / max(1, s0.rays),
                  "unresolved_fraction": s0.unresolved / max(1, s0.rays - s0.missed),
                  "fallback_adds": s0.fallback_adds},
    }
    if batched is not None:
        line["batched"] = batched
    if surrogate is not None:
        line["surrogate"] = surrogate
    if atlas is not None:
        line["atlas"] = atlas
    if rainbow is not None:
        line["rainbow_diffraction"] = rainbow
    if wave is not None:
        line["wave_stages"] = wave
    if parity is not None:
        line["parity"] = parity
    if r0 is not None:
        line["record"] = {"g": r0.cdf.g_stored, "projected_area_mm2": r0.projected_area_mm2,
                          "incident_area_mm2": r0.incident_area_mm2, "diffraction_mm2": r0.diffraction_area_mm2,
                          "histogram_relative_error": r0.histogram_relative_error, "cdf_l1": r0.cdf.l1_error,
                          "trace_s": r0.seconds_trace, "cdf_s": r0.seconds_cdf}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--workload", choices=["drop", "hex"], default="drop")
    p.add_argument("--block-threads", type=int, default=0, help="trace block size (0 = library default)")
    p.add_argument("--batch-records", type=int, default=256, help="records of the batched measurement (0 = skip)")
    p.add_argument("--batch-steps", type=int, default=3)
    p.add_argument("--surrogate-records", type=int, default=256, help="records of the surrogate measurement (0 = skip)")
    p.add_argument("--surrogate-checked", type=int, default=64, help="fresh records checked by 1e8-ray tracer records")
    p.add_argument("--surrogate-batch", type=int, default=256,
                   help="records per surrogate call (records/s grows with it up to ~128 and flattens)")
    p.add_argument("--hash-slots", type=int, default=0, help="shared histogram slots (0 = default, 1 = none)")
    p.add_argument("--atlas-incidents", type=int, default=3,
                   help="incidences of the deterministic atlas composition measurement (0 = skip)")
    p.add_argument("--rainbow-steps", type=int, default=5,
                   help="timed passes of the Table-II rainbow diffraction measurement (0 = skip)")
    p.add_argument("--wave-steps", type=int, default=5,
                   help="timed passes of each stage of a wave-stage (diffraction) record: lattice trace, patch build, "
                        "query, folded records, optics, Table-II diffraction, density, CDF (0 = skip)")
    p.add_argument("--rays", type=float, default=1e8)
    p.add_argument("--ref-rays", type=float, default=3.2e5,
                   help="reference rays per step (all processes; the hex workload traces five times more)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--parity-rays", type=float, default=4e6,
                   help="first ray ids of the timed record checked against the FP64 oracle (0 = skip)")
    p.add_argument("--cpu-leg", default=None, help=argparse.SUPPRESS)
    p.add_argument("--cpu-leg-args", default="{}", help=argparse.SUPPRESS)
    a = p.parse_args()
    if a.cpu_leg:
        run_cpu_leg(a.cpu_leg, json.loads(a.cpu_leg_args))
        return
    if a.warmup < 3:
        a.warmup = 3
    if a.impl == "reference":
        (run_reference_drop if a.workload == "drop" else run_reference_hex)(a)
    else:
        (run_b200_drop if a.workload == "drop" else run_b200_hex)(a)


if __name__ == "__main__":
    main()
