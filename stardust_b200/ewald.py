"""FP64 reference forces and force errors (the accuracy judge of the PM step).

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


def force_error(a, a_ref) -> dict:
    a = np.asarray(a, np.float64)[:, :3]
    r = np.asarray(a_ref, np.float64)[:, :3]
    d = np.linalg.norm(a - r, axis=1)
    rms = float(np.sqrt(np.mean(np.sum(r * r, axis=1))))
    return {"rms_rel": float(np.sqrt(np.mean(d * d)) / rms), "max_rel": float(d.max() / rms), "rms_ref": rms}
