"""FP64 reference forces and force errors (the accuracy reference for the PM step).

``ewald_forces`` calls the library's FP64 Ewald summation (sd_ewald_forces):
periodic Newtonian gravity of Gaussian-smoothed masses (G = 1, total mass 1),
the continuum model that the periodic PM step approximates on a grid.
``force_error`` is the reference's scoring metric
eps = RMS(|F - F_ref|) / RMS(|F_ref|)
(.drive/nbody-simulator/method-search/scoring.md:38), plus the maximum.
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib as L


def default_split(softening: float) -> tuple[float, int]:
    """Ewald smoothing length b and mode cutoff for a softening (box units):
    b = 1/16 (or 1.5 x the smoothed-mass width when larger); modes up to
    n_max = ceil(1.75 / b), where exp(-k^2 b^2 / 4) < 1e-12."""
    b = max(1.0 / 16.0, 1.5 * math.sqrt(2.0) * softening)
    return b, int(math.ceil(1.75 / b))


def ewald_forces(src, tgt, softening: float, split_b: float | None = None, nmax: int | None = None) -> np.ndarray:
    """FP64 accelerations at tgt (n_tgt, 3) from all particles in src.

    src, tgt: float32 (n, 4) arrays (host numpy or CUDA torch tensors)."""
    import torch

    b0, n0 = default_split(softening)
    b = b0 if split_b is None else split_b
    nm = n0 if nmax is None else nmax
    s = src if hasattr(src, "is_cuda") and src.is_cuda else torch.from_numpy(np.ascontiguousarray(src, np.float32)).cuda()
    t = tgt if hasattr(tgt, "is_cuda") and tgt.is_cuda else torch.from_numpy(np.ascontiguousarray(tgt, np.float32)).cuda()
    out = torch.empty((t.shape[0], 3), dtype=torch.float64, device="cuda")
    lib = L.lib()
    ws = torch.empty(int(lib.sd_ewald_workspace_bytes(nm)), dtype=torch.uint8, device="cuda")
    L.check(lib.sd_ewald_forces(s.data_ptr(), int(s.shape[0]), t.data_ptr(), int(t.shape[0]), float(softening),
                                float(b), int(nm), out.data_ptr(), ws.data_ptr(), ws.numel(), None),
            "sd_ewald_forces")
    return out.cpu().numpy()


def pm_accel_f64(pos, sample, grid: int, pot_scale: float, softening_cells: float) -> np.ndarray:
    """FP64 particle-mesh accelerations on the same grid as the step, at the
    particles ``pos[sample]``: the CIC density of all live particles (count
    units), the periodic Green's function -exp(-k^2 s^2 / 2) / (4 pi^2 k^2) with
    s = 2 pi softening_cells / grid (k = 0 dropped), central differences
    -(phi[+1] - phi[-1]) * grid / 2 * pot_scale at the 8 CIC corners, the CIC
    weights again (the conventions of Sim.cu:503-629). The reference for the FP32
    step's arithmetic: the same method, with no rounding to speak of.

    pos: float32 (n, 4) host array; sample: indices of live particles."""
    import scipy.fft

    G = int(grid)
    m = G - 1
    p = np.asarray(pos, np.float64)
    live = p[:, 0] >= 0.0
    g = p[live, :3] * G - 0.5
    i0 = np.floor(g).astype(np.int64)
    f = g - i0
    rho = np.zeros(G ** 3)
    for c in range(8):
        o = np.array([c & 1, (c >> 1) & 1, (c >> 2) & 1])
        idx = (((i0[:, 2] + o[2]) & m) * G + ((i0[:, 1] + o[1]) & m)) * G + ((i0[:, 0] + o[0]) & m)
        w = np.prod(np.where(o == 1, f, 1.0 - f), axis=1)
        rho += np.bincount(idx, weights=w, minlength=G ** 3)
    del g, i0, f
    spec = scipy.fft.rfftn(rho.reshape(G, G, G), workers=-1)
    del rho
    kf = np.fft.fftfreq(G, d=1.0 / G)
    k2 = kf[:, None, None] ** 2 + kf[None, :, None] ** 2 + np.arange(G // 2 + 1, dtype=np.float64)[None, None, :] ** 2
    s = 2.0 * np.pi * softening_cells / G
    with np.errstate(divide="ignore"):
        green = -np.exp(-0.5 * k2 * s * s) / (4.0 * np.pi ** 2 * k2)
    green[0, 0, 0] = 0.0
    spec *= green
    del green, k2
    phi = scipy.fft.irfftn(spec, s=(G, G, G), workers=-1).reshape(-1)
    del spec
    q = p[np.asarray(sample), :3] * G - 0.5
    j0 = np.floor(q).astype(np.int64)
    fq = q - j0

    def phi_at(x, y, z):
        return phi[((z & m) * G + (y & m)) * G + (x & m)]

    acc = np.zeros((len(q), 3))
    for c in range(8):
        o = np.array([c & 1, (c >> 1) & 1, (c >> 2) & 1])
        cx, cy, cz = j0[:, 0] + o[0], j0[:, 1] + o[1], j0[:, 2] + o[2]
        w = np.prod(np.where(o == 1, fq, 1.0 - fq), axis=1)
        grad = np.stack([phi_at(cx + 1, cy, cz) - phi_at(cx - 1, cy, cz),
                         phi_at(cx, cy + 1, cz) - phi_at(cx, cy - 1, cz),
                         phi_at(cx, cy, cz + 1) - phi_at(cx, cy, cz - 1)], axis=1)
        acc += w[:, None] * grad
    return -acc * (0.5 * G * pot_scale)


def force_error(a, a_ref) -> dict:
    a = np.asarray(a, np.float64)[:, :3]
    r = np.asarray(a_ref, np.float64)[:, :3]
    d = np.linalg.norm(a - r, axis=1)
    rms = float(np.sqrt(np.mean(np.sum(r * r, axis=1))))
    return {"rms_rel": float(np.sqrt(np.mean(d * d)) / rms), "max_rel": float(d.max() / rms), "rms_ref": rms}
