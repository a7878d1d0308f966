"""Headless point render of a simulation's particles into an RGBA image
(sd_render_points): the reference's kSplatPoints -> kAccumToRGBA path without
OpenGL. ``render(sim, width, height, **view)`` returns an (H, W, 4) uint8 array;
``view_default()`` gives the top-down density view."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L


def view_default(**kw) -> L.SdView:
    v = L.SdView()
    L.lib().sd_view_default(ctypes.byref(v))
    for k, val in kw.items():
        if k in ("rot", "center"):
            getattr(v, k)[:] = [float(x) for x in np.asarray(val, np.float32).reshape(-1)]
        else:
            setattr(v, k, val)
    return v


def view_dict(v: L.SdView) -> dict:
    return {f[0]: (list(getattr(v, f[0])) if f[0] in ("rot", "center", "reserved") else getattr(v, f[0]))
            for f in L.SdView._fields_}


def render_device(pos_ptr: int, vel_ptr: int, n: int, view: L.SdView, width: int, height: int, stream=None):
    """Render device float4 particle arrays; returns a CUDA uint8 tensor (H, W, 4)."""
    import torch

    lib = L.lib()
    ws = torch.empty(int(lib.sd_render_workspace_bytes(width, height)), dtype=torch.uint8, device="cuda")
    out = torch.empty((height, width, 4), dtype=torch.uint8, device="cuda")
    L.check(lib.sd_render_points(pos_ptr, vel_ptr, n, ctypes.byref(view), width, height, ws.data_ptr(), ws.numel(),
                                 out.data_ptr(), stream), "sd_render_points")
    return out


def render(sim, width: int, height: int, **view) -> np.ndarray:
    """Render a Sim's current particles (pending momentum zeroing applied)."""
    import torch

    n = sim.particle_count()
    pos = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    vel = torch.empty_like(pos)
    sim.get_particles_into(pos, vel)
    torch.cuda.synchronize()
    img = render_device(pos.data_ptr(), vel.data_ptr(), n, view_default(**view), width, height)
    return img.cpu().numpy()
