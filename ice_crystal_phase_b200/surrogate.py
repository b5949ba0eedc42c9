"""Training and serving of the learned surrogate (no reference counterpart: the reference makes
every record with the tracer, one process per record).

    python -m ice_crystal_phase_b200.surrogate train --out DIR [--records 2000 --heldout 200 ...]

1. Training set: records drawn from the batched-record distribution (radius log-uniform
   0.1-3 mm, wavelength 400-700 nm, inclination -90..90 deg, rays proportional to the projected
   area) traced by the batched tracer at the network's cell grid without the diffraction stage;
   the targets are their cell probabilities (icp_surrogate_targets).  The network learns the
   geometric-optics part only: a record with diffraction gets the analytic Fraunhofer rows of
   its projected area added by icp_surrogate_generate, with as much power as the geometric part.
2. Training: Adam with a cosine learning rate over whole records (the loss is the per-record KL
   divergence, which needs every cell of a record), all on the device
   (icp_surrogate_train_step).
3. Held-out truth: every held-out record is traced twice at half the truth's ray count with
   independent seeds; the truth is their mean (a record of the full ray count) and half their
   total-variation distance estimates the truth's own Monte-Carlo noise.  The surrogate's TV
   against the truth is reported on the cell grid and on a coarser storage grid.
4. Fallback: a record is served by the surrogate only when its k nearest checked held-out
   records (normalised log radius, wavelength, inclination) all passed the TV threshold;
   otherwise, and for every held-out record that failed, the tracer makes it.

Device buffers are torch tensors (memory only); every computation runs in libicp_b200.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import sys
import time
from dataclasses import asdict, dataclass
from pathlib import Path

import numpy as np

import ice_crystal_phase_b200 as I

# The trained network for the batched-record distribution (parameters, configuration, fallback
# gate), written by `train` and read by bench.py and the tests.
DEFAULT_MODEL = Path(__file__).resolve().parent / "surrogate_drop.npz"


@dataclass
class TrainSettings:
    records: int = 2000
    heldout: int = 200
    epochs: int = 100
    batch: int = 16
    lr: float = 2e-3
    lr_final: float = 2e-5
    warmup_steps: int = 100
    weight_decay: float = 0.0
    seed: int = 7
    max_internal_hits: int = 10
    rays_max: float = 6e7
    rays_min: float = 1e6
    truth_rays: float = 1e8
    storage: tuple = (64, 128)
    tv_threshold: float = 5e-3
    neighbours: int = 3
    # extra training records with the radius log-uniform over [large_radius_mm, 3] mm (the
    # oblate drops, whose patterns are the hardest to learn); the held-out records keep the
    # batched distribution
    large_records: int = 0
    large_radius_mm: float = 0.8


def _torch():
    import torch

    return torch


def trace_cells(ctx: I.Context, sur: I.Surrogate, specs: list, chunk: int = 64, hits: int = 10):
    """Cell probabilities of the tracer's records at the surrogate's grid: a device float32
    tensor [len(specs), nt*np], traced by the batched entry `chunk` records at a time."""
    torch = _torch()
    nt, np_ = sur.cfg.nt, sur.cfg.np
    out = torch.empty((len(specs), nt * np_), dtype=torch.float32, device="cuda")
    st = I.batch_settings(nt, np_, max_internal_hits=hits, precision=I.ICP_FP32, use_graph=False)
    n = min(chunk, len(specs))
    phi = torch.empty(n * (np_ + 1), dtype=torch.float64, device="cuda")
    theta = torch.empty(n * np_ * (nt + 1), dtype=torch.float64, device="cuda")
    for i in range(0, len(specs), chunk):
        part = specs[i:i + chunk]
        reps = (I.DropReport * len(part))()
        I.check(I.LIB.icp_drop_batch_generate_device(ctx.handle, I._items(part), len(part), C.byref(st),
                                                     C.c_void_p(phi.data_ptr()), C.c_void_p(theta.data_ptr()), reps))
        sur.targets(phi.data_ptr(), theta.data_ptr(), len(part), out[i:i + len(part)].data_ptr())
    return out


def _lr(s: TrainSettings, step: int, total: int) -> float:
    if step < s.warmup_steps:
        return s.lr * (step + 1) / s.warmup_steps
    t = (step - s.warmup_steps) / max(1, total - s.warmup_steps)
    return s.lr_final + 0.5 * (s.lr - s.lr_final) * (1 + math.cos(math.pi * min(1.0, t)))


def train(sur: I.Surrogate, specs: list, targets, s: TrainSettings, log=print) -> dict:
    """Adam over whole records; returns the loss history."""
    torch = _torch()
    rng = np.random.default_rng(s.seed)
    n = len(specs)
    steps_per_epoch = n // s.batch
    total = steps_per_epoch * s.epochs
    step, hist = 0, []
    t0 = time.perf_counter()
    for ep in range(s.epochs):
        order = rng.permutation(n)
        acc = 0.0
        for b in range(steps_per_epoch):
            idx = np.sort(order[b * s.batch:(b + 1) * s.batch])
            batch_t = targets[torch.from_numpy(idx).cuda()]
            step += 1
            opt = I.Adam(_lr(s, step - 1, total), 0.9, 0.999, 1e-8, s.weight_decay, step)
            acc += sur.train_step([specs[i] for i in idx], batch_t.data_ptr(), opt)
        hist.append(acc / max(1, steps_per_epoch))
        if log and (ep % 5 == 0 or ep == s.epochs - 1):
            log(f"epoch {ep:4d}  loss {hist[-1]:.5f}  lr {_lr(s, step - 1, total):.2e}  {time.perf_counter() - t0:.1f}s")
    torch.cuda.synchronize()
    return {"loss": hist, "steps": step, "seconds": time.perf_counter() - t0}


def mean_loss(sur: I.Surrogate, specs: list, targets) -> float:
    R = sur.cfg.max_records
    tot = 0.0
    for i in range(0, len(specs), R):
        part = specs[i:i + R]
        loss, _ = sur.gradient(part, targets[i:i + len(part)].data_ptr(), with_grad=False)
        tot += loss * len(part)
    return tot / len(specs)


def predicted_cells(sur: I.Surrogate, specs: list):
    """Cell probabilities of the records the surrogate emits (icp_surrogate_generate at the full
    cell grid, so that the checked output is the served one: the network's geometric part plus the
    analytic diffraction rows), device float64 [len(specs), nt*np]."""
    torch = _torch()
    R, Cn, nt, np_ = sur.cfg.max_records, sur.cells, sur.cfg.nt, sur.cfg.np
    n = min(R, len(specs))
    phi = torch.empty(n * (np_ + 1), dtype=torch.float64, device="cuda")
    theta = torch.empty(n * np_ * (nt + 1), dtype=torch.float64, device="cuda")
    cells = torch.empty((n, Cn), dtype=torch.float32, device="cuda")
    out = torch.empty((len(specs), Cn), dtype=torch.float64, device="cuda")
    for i in range(0, len(specs), R):
        part = specs[i:i + R]
        sur.generate(part, nt, np_, phi.data_ptr(), theta.data_ptr(), raise_on_audit=False)
        sur.targets(phi.data_ptr(), theta.data_ptr(), len(part), cells.data_ptr())
        out[i:i + len(part)] = cells[:len(part)].double()
    return out


def geometric(specs: list) -> list:
    """The same records without the diffraction stage: the network's training targets (the
    surrogate adds the analytic diffraction rows itself)."""
    return [I.DropSpec(sp.coefficients, sp.radius_mm, sp.interior_index, sp.rays, seed=sp.seed,
                       inclination_deg=sp.inclination_deg, wavelength_nm=sp.wavelength_nm, diffraction=False)
            for sp in specs]


def coarse(p, nt, np_, ct, cp):
    """Cell probabilities [n, nt*np] summed onto a (ct, cp) storage grid."""
    return p.reshape(p.shape[0], ct, nt // ct, cp, np_ // cp).sum(dim=(2, 4)).reshape(p.shape[0], -1)


def tv(a, b):
    return 0.5 * (a - b).abs().sum(dim=1)


def truth_records(ctx: I.Context, sur: I.Surrogate, specs: list, truth_rays: float, hits: int = 10):
    """Two independent tracer records per spec at truth_rays / 2: (their mean, A, B)."""
    half = int(truth_rays // 2)

    def twin(sp, salt):
        return I.DropSpec(sp.coefficients, sp.radius_mm, sp.interior_index, half, seed=sp.seed ^ salt,
                          inclination_deg=sp.inclination_deg, wavelength_nm=sp.wavelength_nm,
                          diffraction=sp.diffraction)

    pa = trace_cells(ctx, sur, [twin(sp, 0x5DEECE66D) for sp in specs], hits=hits).double()
    pb = trace_cells(ctx, sur, [twin(sp, 0x2545F4914F6CDD1D) for sp in specs], hits=hits).double()
    return 0.5 * (pa + pb), pa, pb


def evaluate(ctx: I.Context, sur: I.Surrogate, specs: list, s: TrainSettings) -> dict:
    """Held-out check of the surrogate against tracer truth records of truth_rays rays."""
    nt, np_ = sur.cfg.nt, sur.cfg.np
    ct, cp = s.storage
    truth, pa, pb = truth_records(ctx, sur, specs, s.truth_rays, s.max_internal_hits)
    q = predicted_cells(sur, specs)
    out = {"cell_grid": [nt, np_], "storage_grid": [ct, cp], "truth_rays": s.truth_rays}
    for name, f in (("cells", lambda x: x), ("storage", lambda x: coarse(x, nt, np_, ct, cp))):
        t_sur = tv(f(q), f(truth)).cpu().numpy()
        floor = (0.5 * tv(f(pa), f(pb))).cpu().numpy()  # truth noise: TV(A, B) / 2
        out[name] = {"tv": t_sur.tolist(), "truth_floor": floor.tolist(), "tv_mean": float(t_sur.mean()),
                     "tv_median": float(np.median(t_sur)), "floor_mean": float(floor.mean())}
    t = np.asarray(out["storage"]["tv"])
    out["passed"] = (t <= s.tv_threshold).tolist()
    out["pass_fraction"] = float(np.mean(t <= s.tv_threshold))
    return out


def _key(sp) -> np.ndarray:
    return np.array([(math.log(sp.radius_mm) - math.log(0.1)) / math.log(30.0), (sp.wavelength_nm - 400.0) / 300.0,
                     (sp.inclination_deg + 90.0) / 180.0])


@dataclass
class FallbackGate:
    """Serve by the surrogate only where the k nearest checked held-out records all passed."""
    keys: np.ndarray
    passed: np.ndarray
    k: int = 3

    @staticmethod
    def of(specs: list, passed, k: int = 3) -> "FallbackGate":
        return FallbackGate(np.stack([_key(sp) for sp in specs]), np.asarray(passed, dtype=bool), k)

    def trusted(self, sp) -> bool:
        d = np.linalg.norm(self.keys - _key(sp), axis=1)
        if d.min() == 0.0:
            return bool(self.passed[np.argmin(d)])  # a checked record itself
        return bool(self.passed[np.argsort(d)[:self.k]].all())

    def as_dict(self) -> dict:
        return {"keys": self.keys.tolist(), "passed": self.passed.tolist(), "k": self.k}

    @staticmethod
    def from_dict(d: dict) -> "FallbackGate":
        return FallbackGate(np.asarray(d["keys"]), np.asarray(d["passed"], dtype=bool), int(d["k"]))


def serve(ctx: I.Context, sur: I.Surrogate, specs: list, gate: FallbackGate, ct: int, cp: int, phi, theta,
          hits: int = 10) -> dict:
    """Records for `specs` into device arrays phi[n*(cp+1)], theta[n*cp*(ct+1)]: the surrogate for
    trusted records whose CDF audit passes, the batched tracer for the rest."""
    torch = _torch()
    R = sur.cfg.max_records
    trusted = [gate.trusted(sp) for sp in specs]
    fallback = [i for i, t in enumerate(trusted) if not t]
    use = [i for i, t in enumerate(trusted) if t]
    for i in range(0, len(use), R):
        idx = use[i:i + R]
        part = [specs[j] for j in idx]
        if idx == list(range(idx[0], idx[0] + len(idx))):
            # a contiguous run is written in place
            reps = sur.generate(part, ct, cp, phi[idx[0] * (cp + 1):].data_ptr(),
                                theta[idx[0] * cp * (ct + 1):].data_ptr(), raise_on_audit=False)
        else:
            sp_ = torch.empty(len(idx) * (cp + 1), dtype=torch.float64, device="cuda")
            st_ = torch.empty(len(idx) * cp * (ct + 1), dtype=torch.float64, device="cuda")
            reps = sur.generate(part, ct, cp, sp_.data_ptr(), st_.data_ptr(), raise_on_audit=False)
            for k, j in enumerate(idx):
                phi[j * (cp + 1):(j + 1) * (cp + 1)] = sp_[k * (cp + 1):(k + 1) * (cp + 1)]
                theta[j * cp * (ct + 1):(j + 1) * cp * (ct + 1)] = st_[k * cp * (ct + 1):(k + 1) * cp * (ct + 1)]
        fallback += [j for j, r in zip(idx, reps) if r.status != 0]
    fallback.sort()
    if fallback:
        nt, np_ = sur.cfg.nt, sur.cfg.np
        st = I.batch_settings(nt, np_, ct, cp, max_internal_hits=hits, precision=I.ICP_FP32, use_graph=False)
        part = [specs[j] for j in fallback]
        fp = torch.empty(len(part) * (cp + 1), dtype=torch.float64, device="cuda")
        ft = torch.empty(len(part) * cp * (ct + 1), dtype=torch.float64, device="cuda")
        reps = (I.DropReport * len(part))()
        I.check(I.LIB.icp_drop_batch_generate_device(ctx.handle, I._items(part), len(part), C.byref(st),
                                                     C.c_void_p(fp.data_ptr()), C.c_void_p(ft.data_ptr()), reps))
        for k, j in enumerate(fallback):
            phi[j * (cp + 1):(j + 1) * (cp + 1)] = fp[k * (cp + 1):(k + 1) * (cp + 1)]
            theta[j * cp * (ct + 1):(j + 1) * cp * (ct + 1)] = ft[k * cp * (ct + 1):(k + 1) * cp * (ct + 1)]
    return {"surrogate": len(specs) - len(fallback), "tracer": len(fallback), "fallback": fallback}


def save(path, sur: I.Surrogate, extra: dict) -> None:
    cfg = {}
    for k, _ in I.SurrogateConfig._fields_:
        v = getattr(sur.cfg, k)
        cfg[k] = v if isinstance(v, (int, float)) else list(v)
    np.savez_compressed(path, parameters=sur.parameters(), config=json.dumps(cfg), extra=json.dumps(extra))


def load(ctx: I.Context, path, max_records: int | None = None) -> tuple[I.Surrogate, dict]:
    z = np.load(path, allow_pickle=False)
    fields = json.loads(str(z["config"]))
    if "reserved" in fields:  # written before the axis harmonics existed: none
        fields["axis_harmonics"] = fields.pop("reserved")
    if max_records:
        fields["max_records"] = max_records
    sur = I.Surrogate(ctx, I.surrogate_config(**fields))
    sur.set_parameters(z["parameters"])
    return sur, json.loads(str(z["extra"]))


def set_head_bias(sur: I.Surrogate, specs: list) -> float:
    """Head bias that centres the log-sum-exp of the prediction at zero over `specs`, so that the
    emitted cell mass exp(y) stays well inside the FP64 range."""
    torch = _torch()
    R, Cn = sur.cfg.max_records, sur.cells
    y = torch.empty((R, Cn), dtype=torch.float32, device="cuda")
    lse = []
    for i in range(0, len(specs), R):
        part = specs[i:i + R]
        sur.predict(part, y.data_ptr())
        lse += torch.logsumexp(y[:len(part)].double(), dim=1).cpu().tolist()
    p = sur.parameters()
    p[-1] -= float(np.mean(lse))
    sur.set_parameters(p)
    return float(p[-1])


def init_parameters(cfg: I.SurrogateConfig, seed: int) -> np.ndarray:
    """He-uniform hidden weights (bound sqrt(6 / fan_in)), zero biases, a small head; FP32 in
    the library's parameter layout."""
    rng = np.random.default_rng(seed)
    h, k0 = cfg.hidden, cfg.input_width
    parts = [rng.uniform(-1, 1, h * k0) * math.sqrt(6.0 / k0), np.zeros(h),
             rng.uniform(-1, 1, h * h) * math.sqrt(6.0 / h), np.zeros(h),
             rng.uniform(-1, 1, h * h) * math.sqrt(6.0 / h), np.zeros(h),
             rng.uniform(-1, 1, h) * math.sqrt(3.0 / h), np.zeros(1)]
    return np.concatenate(parts).astype(np.float32)


def run_training(ctx: I.Context, s: TrainSettings, cfg_over: dict | None = None, log=print):
    """The whole pipeline: training set, training, held-out check, fallback gate.  Returns
    (surrogate, gate, held-out specs, report)."""
    torch = _torch()
    cfg = I.surrogate_config(**{"max_records": s.batch, **(cfg_over or {})})
    sur = I.Surrogate(ctx, cfg)
    sur.set_parameters(init_parameters(cfg, s.seed))
    # the held-out records come from their own seed, so that runs with different training sets
    # are checked on the same records
    train_specs = I.batched_record_specs(s.records, seed=1000 * s.seed + 1, rays_max=s.rays_max, rays_min=s.rays_min,
                                         diffraction=True)
    held = I.batched_record_specs(s.heldout, seed=1000 * s.seed + 3, rays_max=s.rays_max, rays_min=s.rays_min,
                                  diffraction=True)
    if s.large_records:
        train_specs = train_specs + I.batched_record_specs(s.large_records, seed=1000 * s.seed + 2,
                                                           rays_max=s.rays_max, rays_min=s.rays_min, diffraction=True,
                                                           radius_range=(s.large_radius_mm, 3.0))
    t0 = time.perf_counter()
    targets = trace_cells(ctx, sur, geometric(train_specs), hits=s.max_internal_hits)
    held_targets = trace_cells(ctx, sur, geometric(held), hits=s.max_internal_hits)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    rays = sum(sp.rays for sp in train_specs)
    if log:
        log(f"training set: {len(train_specs)} records, {rays:.3e} rays in {t_data:.1f}s")
    loss0 = mean_loss(sur, held, held_targets)
    hist = train(sur, train_specs, targets, s, log)
    loss1 = mean_loss(sur, held, held_targets)
    train_loss = mean_loss(sur, train_specs[:s.heldout], targets[:s.heldout])
    hb = set_head_bias(sur, train_specs[:256])
    del targets
    t1 = time.perf_counter()
    ev = evaluate(ctx, sur, held, s)
    t_truth = time.perf_counter() - t1
    gate = FallbackGate.of(held, ev["passed"], s.neighbours)
    report = {"settings": asdict(s),
              "config": {k: getattr(cfg, k) for k in ("nt", "np", "hidden", "input_width", "theta_frequencies",
                                                      "phi_frequencies", "axis_harmonics")},
              "training_set": {"records": len(train_specs), "rays": rays, "seconds": t_data},
              "training": hist, "heldout_kl_before": loss0, "heldout_kl_after": loss1,
              "train_kl_after": train_loss, "head_bias": hb, "truth_seconds": t_truth, "heldout": ev,
              "gate": gate.as_dict()}
    if log:
        log(f"held-out KL {loss0:.4f} -> {loss1:.4f} (train {train_loss:.4f}); TV cells "
            f"{ev['cells']['tv_mean']:.4f} (truth floor {ev['cells']['floor_mean']:.4f}), storage "
            f"{ev['storage']['tv_mean']:.4f} (floor {ev['storage']['floor_mean']:.4f}), "
            f"pass {ev['pass_fraction']:.3f}")
    return sur, gate, held, report


def profile(mode: str, records: int, steps: int, warmup: int = 2, device: int = 0, log=print) -> dict:
    """A fixed surrogate workload for timing and kernel capture: the default network
    (256 x 512 cells, 3 x 256 SiLU layers), He-initialised parameters (seed 0), `records` fresh
    records of the batched distribution; `warmup` untimed steps, then `steps` timed steps of
    `mode` (train: icp_surrogate_train_step against random cell distributions; predict:
    icp_surrogate_predict; generate: icp_surrogate_generate at 64 x 128 storage).  Reports the
    library's kernel-launch count before the timed steps (the `-s` of an ncu launch list) and
    the launches per step (its `-c`)."""
    torch = _torch()
    cfg = I.surrogate_config(max_records=records)
    specs = I.batched_record_specs(records, seed=7)
    with I.Context(device) as ctx:
        sur = I.Surrogate(ctx, cfg)
        sur.set_parameters(init_parameters(cfg, 0))
        n, cells = len(specs), sur.cells
        gen = torch.Generator(device="cuda").manual_seed(0)
        target = torch.rand((n, cells), generator=gen, device="cuda", dtype=torch.float32)
        target /= target.sum(dim=1, keepdim=True)
        y = torch.empty((n, cells), dtype=torch.float32, device="cuda")
        ct, cp = 64, 128
        phi = torch.empty(n * (cp + 1), dtype=torch.float64, device="cuda")
        theta = torch.empty(n * cp * (ct + 1), dtype=torch.float64, device="cuda")
        opt = I.Adam(1e-4, 0.9, 0.999, 1e-8, 0.0, 0)

        def step():
            if mode == "train":
                opt.step += 1
                sur.train_step(specs, target.data_ptr(), opt)
            elif mode == "predict":
                sur.predict(specs, y.data_ptr())
            else:
                sur.generate(specs, ct, cp, phi.data_ptr(), theta.data_ptr(), raise_on_audit=False)

        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        before = I.kernel_launches()
        stream = torch.cuda.ExternalStream(I.LIB.icp_context_stream(ctx.handle))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        out = {"mode": mode, "records": n, "cells": cells, "launches_before_timed_steps": before,
               "launches_per_step": (I.kernel_launches() - before) // max(1, steps),
               "ms_per_step": e0.elapsed_time(e1) / max(1, steps)}
        sur.close()
    log(json.dumps(out))
    return out


def main(argv=None) -> int:
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = p.add_subparsers(dest="cmd", required=True)
    q = sub.add_parser("profile", help="a fixed workload for timing and ncu launch lists")
    q.add_argument("--mode", choices=["train", "predict", "generate"], required=True)
    q.add_argument("--records", type=int, default=16)
    q.add_argument("--steps", type=int, default=1)
    q.add_argument("--warmup", type=int, default=2)
    t = sub.add_parser("train")
    t.add_argument("--out", required=True)
    for f in ("records", "heldout", "epochs", "batch", "seed", "max_internal_hits", "warmup_steps", "neighbours",
              "large_records"):
        t.add_argument("--" + f.replace("_", "-"), type=int, default=getattr(TrainSettings, f))
    for f in ("lr", "lr_final", "weight_decay", "rays_max", "rays_min", "truth_rays", "tv_threshold", "large_radius_mm"):
        t.add_argument("--" + f.replace("_", "-"), type=float, default=getattr(TrainSettings, f))
    t.add_argument("--nt", type=int, default=256)
    t.add_argument("--np", type=int, default=512)
    t.add_argument("--hidden", type=int, default=256)
    t.add_argument("--input-width", type=int, default=128)
    t.add_argument("--theta-frequencies", type=int, default=40)
    t.add_argument("--phi-frequencies", type=int, default=12)
    t.add_argument("--axis-harmonics", type=int, default=16)
    a = p.parse_args(argv)
    if a.cmd == "profile":
        profile(a.mode, a.records, a.steps, a.warmup)
        return 0
    s = TrainSettings(**{k: getattr(a, k) for k in TrainSettings.__dataclass_fields__ if hasattr(a, k)})
    over = {"nt": a.nt, "np": a.np, "hidden": a.hidden, "input_width": a.input_width,
            "theta_frequencies": a.theta_frequencies, "phi_frequencies": a.phi_frequencies,
            "axis_harmonics": a.axis_harmonics, "max_records": s.batch}
    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    with I.Context(0) as ctx:
        sur, gate, held, report = run_training(ctx, s, over)
        save(out / "surrogate.npz", sur, {"gate": gate.as_dict(), "storage": list(s.storage)})
        (out / "report.json").write_text(json.dumps(report, indent=1))
        sur.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
