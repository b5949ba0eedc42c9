"""CPU oracle of the learned surrogate: feature rows, forward pass, per-record softmax loss,
backward pass and Adam, in numpy FP64.

TEST INFRASTRUCTURE ONLY.  Imported by tests/ and __graft_entry__.smoke() as the checker of the
device kernels (ice_crystal_phase_b200/csrc/icp_mlp*.cu, icp_capi_mlp.cu); the product never
imports it.

The reference project has no surrogate (its records come from the tracer alone), so there is no
reference algorithm to restate: this file restates the network the library defines.  Two modes:

* ``emulate=True`` rounds every tensor the device stores in BF16 (features, z and h of each
  layer, the backpropagated dz) at the same points as the device, so that the device's results
  differ only by FP32 accumulation order and fast-math exponentials;
* ``emulate=False`` is the exact FP64 network, whose analytic gradient the CPU tests check
  against central finite differences.

Parameter layout (FP32 on the device): W1[H][K0], b1[H], W2[H][H], b2[H], W3[H][H], b3[H],
w4[H], head bias.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def bf16(x) -> np.ndarray:
    """Round to FP32, then to BF16 (nearest even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF
    r = np.where(np.isnan(f), 0x7FC0, r).astype(np.uint32)
    return (r << 16).view(np.float32).astype(np.float64)


def bf16_bits(x) -> np.ndarray:
    return (np.ascontiguousarray(bf16(x).astype(np.float32)).view(np.uint32) >> 16).astype(np.uint16)


def from_bits(b) -> np.ndarray:
    return (np.asarray(b, dtype=np.uint32) << 16).view(np.float32).astype(np.float64)


@dataclass
class Config:
    nt: int = 256
    np: int = 512
    hidden: int = 256
    input_width: int = 128
    theta_frequencies: int = 40
    phi_frequencies: int = 12
    axis_harmonics: int = 16
    log_radius_mm: tuple = (math.log(0.1), math.log(3.0))
    wavelength_nm: tuple = (400.0, 700.0)
    log_wavelength_over_radius: tuple = (math.log(400e-6 / 3.0), math.log(700e-6 / 0.1))
    index_center: float = 1.337
    index_scale: float = 0.0065
    coefficient_scale: tuple = (12, 20, 5, 40, 33, 60, 400, 140)

    @staticmethod
    def of(cfg) -> "Config":
        """From the library's SurrogateConfig structure."""
        return Config(cfg.nt, cfg.np, cfg.hidden, cfg.input_width, cfg.theta_frequencies, cfg.phi_frequencies,
                      cfg.axis_harmonics, tuple(cfg.log_radius_mm), tuple(cfg.wavelength_nm),
                      tuple(cfg.log_wavelength_over_radius), cfg.index_center, cfg.index_scale,
                      tuple(cfg.coefficient_scale))


def _unit(x, r):
    return 2.0 * (x - r[0]) / (r[1] - r[0]) - 1.0


def record_features(cfg: Config, radius_mm, wavelength_nm, inclination_deg, interior_index, coefficients) -> np.ndarray:
    """The 16 record features in FP64 (before rounding)."""
    f = np.zeros(16)
    deg = inclination_deg * (math.pi / 180.0)
    f[0] = _unit(math.log(radius_mm), cfg.log_radius_mm)
    f[1] = _unit(wavelength_nm, cfg.wavelength_nm)
    f[2] = inclination_deg / 90.0
    f[3] = math.sin(deg)
    f[4] = math.cos(deg)
    f[5] = _unit(math.log(wavelength_nm * 1e-6 / radius_mm), cfg.log_wavelength_over_radius)
    f[6] = (interior_index - cfg.index_center) / cfg.index_scale
    c = list(coefficients) + [0.0] * (8 - len(coefficients))
    for n in range(8):
        f[7 + n] = c[n] * cfg.coefficient_scale[n]
    return f


def cell_geometry(cfg: Config) -> tuple[np.ndarray, np.ndarray]:
    """(cos theta, sin theta sin phi) of every cell centre, phi the column's azimuth in [-pi, pi)
    (the binning's convention), with the C library's cos / sin."""
    ct = np.empty(cfg.nt * cfg.np)
    sts = np.empty(cfg.nt * cfg.np)
    for i in range(cfg.nt):
        th = math.pi * (i + 0.5) / cfg.nt
        c, s = math.cos(th), math.sin(th)
        for j in range(cfg.np):
            ph = -math.pi + 2.0 * math.pi * (j + 0.5) / cfg.np
            ct[i * cfg.np + j] = c
            sts[i * cfg.np + j] = s * math.sin(ph)
    return ct, sts


def axis_features(cfg: Config, inclination_deg, geometry=None) -> np.ndarray:
    """Axis harmonics [R*C, P]: T_1..T_P(cos psi), cos psi = -(sin a cos theta) -
    (cos a sin theta sin phi), the cosine of the angle between a cell's direction and the drop's
    symmetry axis; FP64 without contraction, Chebyshev recurrence T_{k+1} = (2x) T_k - T_{k-1}."""
    ct, sts = geometry if geometry is not None else cell_geometry(cfg)
    out = []
    for a in inclination_deg:
        deg = a * (math.pi / 180.0)
        sa, ca = math.sin(deg), math.cos(deg)
        x = -(sa * ct) - (ca * sts)
        cols, tm, t = [], np.ones_like(x), x
        for _ in range(cfg.axis_harmonics):
            cols.append(t)
            tm, t = t, 2.0 * x * t - tm
        out.append(np.stack(cols, axis=1) if cols else np.zeros((x.size, 0)))
    return np.concatenate(out, axis=0)


def cell_features(cfg: Config) -> np.ndarray:
    """Cell table [nt*np, K0-16] in FP64 (before rounding), theta-major cells; the last
    axis_harmonics columns are zero (they depend on the record: axis_features)."""
    kc = cfg.input_width - 16
    i = np.repeat(np.arange(cfg.nt), cfg.np).astype(np.float64)
    j = np.tile(np.arange(cfg.np), cfg.nt).astype(np.float64)
    th = math.pi * (i + 0.5) / cfg.nt
    ph = 2.0 * math.pi * (j + 0.5) / cfg.np
    f = np.zeros((cfg.nt * cfg.np, kc))
    f[:, 0] = 2.0 * (i + 0.5) / cfg.nt - 1.0
    f[:, 1] = np.cos(th)
    f[:, 2] = (i == 0)
    f[:, 3] = (i == cfg.nt - 1)
    F, G = cfg.theta_frequencies, cfg.phi_frequencies
    for k in range(1, F + 1):
        f[:, 4 + 2 * (k - 1)] = np.sin(k * th)
        f[:, 5 + 2 * (k - 1)] = np.cos(k * th)
    for l in range(1, G + 1):
        f[:, 4 + 2 * F + (l - 1)] = np.cos(l * (ph - 0.5 * math.pi))
    return f


def parameter_count(cfg: Config) -> int:
    h = cfg.hidden
    return h * cfg.input_width + 2 * h * h + 4 * h + 1


def unpack(cfg: Config, p: np.ndarray) -> dict:
    h, k0 = cfg.hidden, cfg.input_width
    p = np.asarray(p, dtype=np.float64)
    o, out = 0, {}
    for name, shape in (("W1", (h, k0)), ("b1", (h,)), ("W2", (h, h)), ("b2", (h,)), ("W3", (h, h)), ("b3", (h,)),
                        ("w4", (h,)), ("hb", (1,))):
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    assert o == p.size
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([np.ravel(d[k]) for k in ("W1", "b1", "W2", "b2", "W3", "b3", "w4", "hb")])


def init_parameters(cfg: Config, seed: int) -> np.ndarray:
    """Uniform(+-sqrt(6 / fan_in)) hidden weights (He-uniform for SiLU), zero biases, small head."""
    rng = np.random.default_rng(seed)
    h, k0 = cfg.hidden, cfg.input_width
    d = {"W1": rng.uniform(-1, 1, (h, k0)) * math.sqrt(6.0 / k0), "b1": np.zeros(h),
         "W2": rng.uniform(-1, 1, (h, h)) * math.sqrt(6.0 / h), "b2": np.zeros(h),
         "W3": rng.uniform(-1, 1, (h, h)) * math.sqrt(6.0 / h), "b3": np.zeros(h),
         "w4": rng.uniform(-1, 1, h) * math.sqrt(3.0 / h), "hb": np.zeros(1)}
    return pack(d).astype(np.float32)


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def inputs(cfg: Config, rec: np.ndarray, cells: np.ndarray, inclination_deg=None) -> np.ndarray:
    """X [R*C, K0]: record row r (16 values) beside every cell row, the last axis_harmonics
    columns the record's axis harmonics (rounded to BF16 like the device's)."""
    R, C = rec.shape[0], cells.shape[0]
    X = np.empty((R * C, cfg.input_width))
    for r in range(R):
        X[r * C:(r + 1) * C, :16] = rec[r]
        X[r * C:(r + 1) * C, 16:] = cells
    P = cfg.axis_harmonics
    if P:
        X[:, cfg.input_width - P:] = bf16(axis_features(cfg, inclination_deg))
    return X


def forward(cfg: Config, params, X: np.ndarray, emulate: bool = True) -> dict:
    q = unpack(cfg, params)
    rnd = bf16 if emulate else (lambda v: np.asarray(v, dtype=np.float64))
    W1, W2, W3 = rnd(q["W1"]), rnd(q["W2"]), rnd(q["W3"])
    t = {"X": rnd(X), "W1": W1, "W2": W2, "W3": W3, "q": q}
    z1 = t["X"] @ W1.T + q["b1"]
    t["z1"], t["h1"] = rnd(z1), rnd(_silu(z1))
    z2 = t["h1"] @ W2.T + q["b2"]
    t["z2"], t["h2"] = rnd(z2), rnd(_silu(z2))
    z3 = t["h2"] @ W3.T + q["b3"]
    t["z3"] = rnd(z3)
    t["y"] = _silu(z3) @ q["w4"] + q["hb"][0]
    return t


def loss_and_dy(y: np.ndarray, target: np.ndarray, records: int) -> tuple[np.ndarray, np.ndarray]:
    """Per-record KL divergence of the target from softmax(y), and dy of their mean."""
    Y = y.reshape(records, -1)
    P = np.asarray(target, dtype=np.float64).reshape(records, -1)
    mx = Y.max(axis=1, keepdims=True)
    lse = mx + np.log(np.exp(Y - mx).sum(axis=1, keepdims=True))
    logq = Y - lse
    pos = P > 0
    kl = np.where(pos, P * (np.log(np.where(pos, P, 1.0)) - logq), 0.0).sum(axis=1)
    dy = (np.exp(logq) - P) / records
    return kl, dy.ravel()


def backward(cfg: Config, t: dict, dy: np.ndarray, emulate: bool = True) -> np.ndarray:
    rnd = bf16 if emulate else (lambda v: np.asarray(v, dtype=np.float64))
    q = t["q"]
    g = {k: np.zeros_like(v) for k, v in q.items()}
    z3 = t["z3"]
    dz3f = dy[:, None] * q["w4"][None, :] * _silu_grad(z3)
    g["w4"] = dy @ _silu(z3)
    g["b3"] = dz3f.sum(axis=0)
    dz3 = rnd(dz3f)
    g["W3"] = dz3.T @ t["h2"]
    dz2f = (dz3 @ t["W3"]) * _silu_grad(t["z2"])
    g["b2"] = dz2f.sum(axis=0)
    dz2 = rnd(dz2f)
    g["W2"] = dz2.T @ t["h1"]
    dz1f = (dz2 @ t["W2"]) * _silu_grad(t["z1"])
    g["b1"] = dz1f.sum(axis=0)
    dz1 = rnd(dz1f)
    g["W1"] = dz1.T @ t["X"]
    return pack(g)


def gradient(cfg: Config, params, X: np.ndarray, target: np.ndarray, records: int, emulate: bool = True):
    """(mean loss, gradient in the parameter layout)."""
    t = forward(cfg, params, X, emulate)
    kl, dy = loss_and_dy(t["y"], target, records)
    return float(kl.mean()), backward(cfg, t, dy, emulate)


def adam(params, grad, m, v, step: int, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8,
         weight_decay: float = 0.0):
    """One Adam step (decoupled weight decay) on every parameter but the head bias."""
    p = np.asarray(params, dtype=np.float64).copy()
    n = p.size - 1
    g = np.asarray(grad, dtype=np.float64)[:n]
    m = beta1 * m[:n] + (1 - beta1) * g
    v = beta2 * v[:n] + (1 - beta2) * g * g
    mh = m / (1 - beta1 ** step)
    vh = v / (1 - beta2 ** step)
    p[:n] -= lr * (mh / (np.sqrt(vh) + eps) + weight_decay * p[:n])
    return p, m, v
