"""Learned sub-grid force correction for the coarse PM step.

A small MLP (30 -> 64 -> 64 -> 3, SiLU; BF16 weights and activations, FP32
accumulation on the tensor cores) maps a particle's coarse-grid features -- the
3x3x3 CIC density stencil around its cell as log(1 + rho/rho_bar) - log 2, and
its sub-cell offset -- to the residual between a fine-grid PM acceleration and
the coarse one. The step adds ``out_scale * MLP(features)`` to the coarse PM
acceleration before the kick (``Sim.set_correction``); plain PM stays the
fallback (no correction set) and the yardstick of the error.

Everything on the GPU runs through the library's own kernels: features
(``sd_mlp_features``), forward and backward passes (``sd_mlp_loss_grad``), the
Adam update (``sd_mlp_adam``) and the fused inference inside the step
(``sd_mlp_infer``). PyTorch only holds device buffers and shuffles batch
indices. The reference has no counterpart of any of this.

Both grids solve the same physical model: Newtonian gravity (G = 1, total mass 1)
of Gaussian-smoothed particles of width ``softening`` (box units), i.e.
``softening_cells = softening * grid``; the FP64 Ewald sum with the same width
is the exact answer both approximate.
"""
from __future__ import annotations

import ctypes
import json
import math
import time
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .scenes import zeldovich
from .sim import Sim, SimConfig

N_PARAMS = 6792
# offsets (floats) of the packed FP32 parameter vector; W[k][n] maps input k to output n
LAYOUT = {"W1": (0, (32, 64)), "b1": (2048, (64,)), "W2": (2112, (64, 64)), "b2": (6208, (64,)),
          "W3": (6272, (64, 8)), "b3": (6784, (8,))}


def init_params(seed: int = 0) -> np.ndarray:
    """Scaled-normal initial weights; padded inputs (30, 31) and outputs (3..7)
    are zero and stay zero (their gradients vanish)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)

    def put(name, a):
        o, sh = LAYOUT[name]
        p[o:o + int(np.prod(sh))] = np.asarray(a, np.float32).reshape(-1)

    w1 = rng.standard_normal((32, 64)) * math.sqrt(1.0 / 30.0)
    w1[30:] = 0.0
    put("W1", w1)
    put("W2", rng.standard_normal((64, 64)) * math.sqrt(1.0 / 64.0))
    w3 = rng.standard_normal((64, 8)) * (0.1 / math.sqrt(64.0))
    w3[:, 3:] = 0.0
    put("W3", w3)
    return p


@dataclass
class Correction:
    """A trained correction: parameters and the setup it was trained for."""

    params: np.ndarray
    out_scale: float
    softening: float          # box units
    coarse_grid: int
    fine_grid: int

    def save(self, path: str) -> None:
        np.savez(path, params=self.params.astype(np.float32), out_scale=self.out_scale, softening=self.softening,
                 coarse_grid=self.coarse_grid, fine_grid=self.fine_grid)

    @classmethod
    def load(cls, path: str) -> "Correction":
        z = np.load(path)
        return cls(z["params"].astype(np.float32), float(z["out_scale"]), float(z["softening"]),
                   int(z["coarse_grid"]), int(z["fine_grid"]))


def _torch():
    import torch

    return torch


def pm_config(n: int, grid: int, softening: float, **kw) -> SimConfig:
    """Newtonian PM configuration of the periodic unit box (G = 1, total mass 1)."""
    kw.setdefault("keep_density", 1)
    return SimConfig(particle_count=n, grid_size=grid, gravity=1.0, softening_cells=softening * grid,
                     units=L.SD_UNITS_NEWTON, order=L.SD_ORDER_TILED, **kw)


class PMField:
    """PM accelerations (and the kept density) of one particle set on one grid."""

    def __init__(self, pos_dev, grid: int, softening: float, correction: Correction | None = None):
        torch = _torch()
        self.n = int(pos_dev.shape[0])
        self.grid = grid
        self.sim = Sim(0)
        # the library's calls below return before their kernels finish: order
        # them with the torch tensors that receive the results
        self.sim.set_stream(torch.cuda.current_stream())
        self.sim.init(pm_config(self.n, grid, softening))
        vel = torch.zeros_like(pos_dev)
        self.sim.set_particles(pos_dev, vel)
        if correction is not None:
            self.set_correction(correction)

    def set_correction(self, c: Correction | None) -> None:
        set_correction(self.sim, c)

    def accel(self):
        torch = _torch()
        out = torch.empty((self.n, 4), dtype=torch.float32, device="cuda")
        L.check(L.lib().sd_get_accel(self.sim.handle, out.data_ptr(), self.n, L.SD_DEVICE), "sd_get_accel")
        return out

    def density(self):
        """Density (count units) of the last field solve, as a CUDA tensor."""
        torch = _torch()
        out = torch.empty((self.grid,) * 3, dtype=torch.float32, device="cuda")
        L.check(L.lib().sd_get_density(self.sim.handle, out.data_ptr(), L.SD_DEVICE), "sd_get_density")
        return out

    def close(self):
        self.sim.close()


def set_correction(sim: Sim, c: Correction | None) -> None:
    """Enable (or with None disable) the learned correction in a Sim's step."""
    torch = _torch()
    if c is None:
        L.check(L.lib().sd_set_mlp(sim.handle, None, ctypes.c_float(0.0)), "sd_set_mlp")
        return
    p = torch.from_numpy(np.ascontiguousarray(c.params, np.float32)).cuda()
    L.check(L.lib().sd_set_mlp(sim.handle, p.data_ptr(), ctypes.c_float(c.out_scale)), "sd_set_mlp")
    torch.cuda.synchronize()


def features(pos_dev, rho_dev, grid: int, n_norm: int | None = None):
    """BF16 (n, 32) features of the particles (sd_mlp_features)."""
    torch = _torch()
    n = int(pos_dev.shape[0])
    inv_mean = grid ** 3 / float(n_norm or n)
    out = torch.empty((n, 32), dtype=torch.bfloat16, device="cuda")
    L.check(L.lib().sd_mlp_features(pos_dev.data_ptr(), None, n, rho_dev.data_ptr(), grid, ctypes.c_float(inv_mean),
                                    out.data_ptr(), None), "sd_mlp_features")
    return out


def training_pairs(seeds, n_side: int = 128, coarse: int = 128, fine: int = 512, softening: float = 1.0 / 128,
                   log=None):
    """Features and residual targets a_fine - a_coarse of Zel'dovich scenes, one per seed."""
    torch = _torch()
    xs, ts = [], []
    for sd in seeds:
        t0 = time.time()
        pos, _ = zeldovich(n_side, int(sd))
        pd = torch.from_numpy(pos).cuda()
        fc = PMField(pd, coarse, softening)
        ac = fc.accel()
        x = features(pd, fc.density(), coarse)
        fc.close()
        ff = PMField(pd, fine, softening)
        af = ff.accel()
        ff.close()
        xs.append(x)
        ts.append((af - ac)[:, :3].contiguous())
        if log:
            log(f"pairs seed {sd}: {len(pos)} particles in {time.time() - t0:.1f}s")
    return torch.cat(xs), torch.cat(ts)


def train(X, T, epochs: int = 12, batch: int = 16384, lr: float = 2e-3, seed: int = 0, params=None,
          log=None) -> tuple[np.ndarray, float, list]:
    """Adam on the mean squared error of the residual scaled to unit RMS.

    Returns (params, out_scale, per-epoch RMS relative residual error)."""
    torch = _torch()
    lib = L.lib()
    rows = (int(X.shape[0]) // batch) * batch
    out_scale = float(torch.sqrt(torch.mean(T.double() ** 2)).item())
    Tn = (T / out_scale).float().contiguous()
    p = torch.from_numpy(init_params(seed) if params is None else np.asarray(params, np.float32)).cuda()
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    g = torch.zeros_like(p)
    ws = torch.empty(int(lib.sd_mlp_train_workspace_bytes(batch)), dtype=torch.uint8, device="cuda")
    nb = rows // batch
    sse = torch.zeros(nb, dtype=torch.float32, device="cuda")
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    history = []
    step = 0
    total = epochs * nb
    for ep in range(epochs):
        idx = torch.randperm(int(X.shape[0]), device="cuda", generator=gen)[:rows]
        Xs = X.index_select(0, idx)
        Ts = Tn.index_select(0, idx)
        for b in range(nb):
            step += 1
            lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * (step - 1) / total))  # cosine decay
            xb = Xs[b * batch:(b + 1) * batch]
            tb = Ts[b * batch:(b + 1) * batch]
            L.check(lib.sd_mlp_loss_grad(p.data_ptr(), xb.data_ptr(), tb.data_ptr(), batch, g.data_ptr(),
                                         sse[b:].data_ptr(), ws.data_ptr(), ws.numel(), None), "sd_mlp_loss_grad")
            L.check(lib.sd_mlp_adam(p.data_ptr(), m.data_ptr(), v.data_ptr(), g.data_ptr(), step,
                                    ctypes.c_float(lr_t), ctypes.c_float(0.9), ctypes.c_float(0.999),
                                    ctypes.c_float(1e-8), None), "sd_mlp_adam")
        # residual left / residual before (the targets have unit mean square per component)
        rel = math.sqrt(float(sse.sum().item()) / (3.0 * rows))
        history.append(rel)
        if log:
            log(f"epoch {ep}: rms residual left {rel:.4f}")
    return p.cpu().numpy(), out_scale, history


def step_rate(pos, vel, grid: int, softening: float, correction: Correction | None = None, dt: float = 1e-3,
              steps: int = 20, warmup: int = 4) -> float:
    """Particle-steps/s of the full step (sort, deposit, Poisson, [correction],
    gather) through the captured-graph path, timed with CUDA events."""
    torch = _torch()
    n = len(pos)
    stream = torch.cuda.Stream()
    with Sim(0) as sim:
        sim.set_stream(stream)
        sim.init(pm_config(n, grid, softening, sort_interval=1, keep_density=0 if correction is None else 1))
        sim.set_particles(pos, vel)
        if correction is not None:
            sim.set_correction(correction)
        sim.steps(dt, warmup)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.steps(dt, steps)
        e1.record(stream)
        torch.cuda.synchronize()
        return n / (e0.elapsed_time(e1) * 1e-3 / steps)


def equal_error_rate(err: float, plain: dict) -> float | None:
    """Particle-steps/s plain PM would need for force error `err`: log-log
    interpolation between the grids that bracket it (None outside them)."""
    gs = sorted(plain)
    for a, b in zip(gs, gs[1:]):
        ea, eb = plain[a]["error"], plain[b]["error"]
        if eb <= err <= ea:
            t = (math.log(ea) - math.log(err)) / (math.log(ea) - math.log(eb))
            return math.exp((1 - t) * math.log(plain[a]["rate"]) + t * math.log(plain[b]["rate"]))
    return None


def compare(train_seeds=range(8), eval_seed: int = 1000, n_side: int = 128, coarse: int = 128, fine: int = 512,
            softening: float = 1.0 / 128, n_targets: int = 65_536, epochs: int = 10, steps: int = 20,
            log=None) -> dict:
    """Train on (coarse, fine) pairs of `train_seeds`, then measure plain PM on
    coarse..fine grids and coarse + correction on a held-out scene against FP64
    Ewald forces at `n_targets` particles, and time each step."""
    torch = _torch()
    from .ewald import ewald_forces, force_error

    t0 = time.time()
    X, T = training_pairs(train_seeds, n_side, coarse, fine, softening)
    params, scale, hist = train(X, T, epochs=epochs)
    del X, T
    corr = Correction(params, scale, softening, coarse, fine)
    t_train = time.time() - t0
    pos, vel = zeldovich(n_side, eval_seed)
    pd = torch.from_numpy(pos).cuda()
    tgt = np.sort(np.random.default_rng(eval_seed).choice(len(pos), n_targets, replace=False))
    ref = ewald_forces(pd, pd[torch.from_numpy(tgt).cuda()].contiguous(), softening)
    plain = {}
    g = coarse
    while g <= fine:
        f = PMField(pd, g, softening)
        e = force_error(f.accel().cpu().numpy()[tgt], ref)
        f.close()
        plain[g] = {"error": e["rms_rel"], "max_error": e["max_rel"], "rate": step_rate(pos, vel, g, softening,
                                                                                          steps=steps)}
        g *= 2
    f = PMField(pd, coarse, softening, corr)
    e = force_error(f.accel().cpu().numpy()[tgt], ref)
    f.close()
    learned = {"error": e["rms_rel"], "max_error": e["max_rel"],
               "rate": step_rate(pos, vel, coarse, softening, corr, steps=steps)}
    eq = equal_error_rate(learned["error"], plain)
    out = {
        "scene": f"Zel'dovich {n_side}^3 lattice (seed {eval_seed}), softening {softening:.6g} box",
        "error_reference": f"FP64 Ewald, {n_targets} targets, all {len(pos)} sources",
        "plain": {str(k): v for k, v in plain.items()},
        "learned": learned,
        "train": {"seeds": list(train_seeds), "pairs": f"{coarse}^3 vs {fine}^3", "epochs": epochs,
                  "rms_residual_left": hist[-1], "seconds": t_train, "out_scale": scale},
        "error_gain": plain[coarse]["error"] / learned["error"],
        "speed_vs_fine": learned["rate"] / plain[fine]["rate"],
        "reaches_fine_error": learned["error"] <= plain[fine]["error"],
        "speed_vs_plain_at_equal_error": (learned["rate"] / eq) if eq else None,
    }
    if log:
        log(json.dumps(out))
    return out
