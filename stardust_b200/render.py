"""Headless renders into RGBA images without OpenGL: the point view
(sd_render_points, the reference's kSplatPoints -> kAccumToRGBA) and the grid
view (sd_render_field, its field projections -> kShade). ``render(sim, width,
height, **view)`` and ``render_field(sim, width, height, field, **view)`` return
(H, W, 4) uint8 arrays; ``view_default()`` gives the top-down density view."""
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


def render_field_device(field: int, density_ptr: int, G: int, pos_ptr: int, vel_ptr: int, n: int, view: L.SdView,
                        width: int, height: int, stream=None):
    """Grid view of a device density grid (float[G^3]) or of device particles
    (dispersion); returns a CUDA uint8 tensor (H, W, 4)."""
    import torch

    lib = L.lib()
    ws = torch.empty(int(lib.sd_render_field_workspace_bytes(G)), dtype=torch.uint8, device="cuda")
    out = torch.empty((height, width, 4), dtype=torch.uint8, device="cuda")
    L.check(lib.sd_render_field(field, density_ptr, G, pos_ptr, vel_ptr, n, ctypes.byref(view), width, height,
                                ws.data_ptr(), ws.numel(), out.data_ptr(), stream), "sd_render_field")
    return out


def render_field(sim, width: int, height: int, field: int = L.SD_FIELD_DENSITY, **view) -> np.ndarray:
    """Grid view of a Sim: its density of the step-start positions (of the
    current positions before any step) or the velocity dispersion."""
    import torch

    n, G = sim.particle_count(), sim.grid_size()
    pos = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    vel = torch.empty_like(pos)
    sim.get_particles_into(pos, vel)
    rho = torch.from_numpy(np.ascontiguousarray(sim.density(), np.float32)).cuda() if field == L.SD_FIELD_DENSITY \
        else torch.empty(1, device="cuda")
    torch.cuda.synchronize()
    img = render_field_device(field, rho.data_ptr(), G, pos.data_ptr(), vel.data_ptr(), n, view_default(**view),
                              width, height)
    return img.cpu().numpy()


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
