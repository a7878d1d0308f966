"""Headless renders against the numpy restatements: the point view
(sd_render_points; the reference's kSplatPoints -> kAccumToRGBA) and the grid
view (sd_render_field; kProjectXY / kScatterDispersion -> kHistLog brightness ->
kShade), plus order independence."""
import math

import numpy as np
import pytest

from stardust_b200 import _lib as L
from stardust_b200 import scenes

pytestmark = pytest.mark.gpu


def _gpu_render(cuda, pos, vel, view, W, H):
    from stardust_b200.render import render_device

    pd = cuda.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda()
    vd = cuda.from_numpy(np.ascontiguousarray(vel, np.float32)).cuda()
    img = render_device(pd.data_ptr(), vd.data_ptr(), len(pos), view, W, H)
    cuda.cuda.synchronize()
    return img.cpu().numpy()


def _views():
    from stardust_b200.render import view_default

    a = math.radians(60.0)
    rx = [1, 0, 0, 0, math.cos(a), -math.sin(a), 0, math.sin(a), math.cos(a)]
    return {
        "top_density_astro": view_default(),
        "tilted_speed_thermal_3x3": view_default(rot=rx, zoom=2.0, size_px=3.0, color_by=2, cmap=2, use_cmap=0,
                                                 reinhard=1, bright=4.0),
        "zoomed_gray_5x5": view_default(zoom=4.0, pan_x=0.05, size_px=2.0, cmap=1, bright=2.0, inv_gamma=0.8),
        "fly_speed": view_default(fly=1, center=[0.5, 0.5, -1.0], color_by=2, size_px=1.5),
    }


@pytest.mark.parametrize("name", list(_views()))
def test_render_matches_oracle(cuda, oracle, name):
    from stardust_b200.render import view_dict

    pos, vel = scenes.disk_galaxy(262_144, 3)
    view = _views()[name]
    W, H = 480, 320
    img = _gpu_render(cuda, pos, vel, view, W, H)
    ref = oracle.render_points(pos, vel, view_dict(view), W, H)
    assert img.shape == (H, W, 4) and np.all(img[..., 3] == 255)
    d = np.abs(img[..., :3].astype(np.int32) - ref[..., :3].astype(np.int32))
    assert (d > 1).mean() < 2e-3, (d > 1).mean()
    assert d.mean() < 0.05
    assert ref[..., :3].max() > 100  # the scene is visible


def test_render_is_independent_of_particle_order(cuda):
    from stardust_b200.render import view_default

    pos, vel = scenes.disk_galaxy(100_000, 4)
    view = view_default(zoom=2.0, size_px=3.0, color_by=2)
    a = _gpu_render(cuda, pos, vel, view, 256, 256)
    perm = np.random.default_rng(0).permutation(len(pos))
    b = _gpu_render(cuda, pos[perm], vel[perm], view, 256, 256)
    assert np.array_equal(a, b)


def test_render_of_a_sim_and_of_nothing(cuda):
    from stardust_b200.render import render, render_device, view_default
    from stardust_b200.sim import Sim, SimConfig

    pos, vel = scenes.disk_galaxy(50_000, 5)
    with Sim(0) as s:
        s.init(SimConfig(particle_count=len(pos), grid_size=32))
        s.set_particles(pos, vel)
        s.step(1e-3)
        img = render(s, 128, 96)
    assert img.shape == (96, 128, 4) and img[..., :3].max() > 0
    empty = render_device(0, 0, 0, view_default(), 64, 48).cpu().numpy()
    assert np.all(empty[..., :3] == 0) and np.all(empty[..., 3] == 255)


# ---- grid view (sd_render_field: field projections -> kShade) -------------------

def _field_gpu(cuda, field, rho, pos, vel, G, view, W, H):
    from stardust_b200.render import render_field_device

    r = cuda.from_numpy(np.ascontiguousarray(rho, np.float32).reshape(-1)).cuda()
    pd = cuda.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda()
    vd = cuda.from_numpy(np.ascontiguousarray(vel, np.float32)).cuda()
    img = render_field_device(field, r.data_ptr(), G, pd.data_ptr(), vd.data_ptr(), len(pos), view, W, H)
    cuda.cuda.synchronize()
    return img.cpu().numpy()


def _field_views():
    from stardust_b200.render import view_default

    a = math.radians(50.0)
    ry = [math.cos(a), 0, math.sin(a), 0, 1, 0, -math.sin(a), 0, math.cos(a)]
    return {
        "density_top_astro": (L.SD_FIELD_DENSITY, view_default()),
        "density_zoom_pan_gray": (L.SD_FIELD_DENSITY, view_default(zoom=2.5, pan_x=0.1, pan_y=-0.05, cmap=1,
                                                                   inv_gamma=0.8, bright=2.0)),
        "density_rotated_thermal": (L.SD_FIELD_DENSITY, view_default(rot=ry, rot_on=1, cmap=2)),
        "dispersion_blackbody": (L.SD_FIELD_DISPERSION, view_default(cmap=3, bright=0.5)),
        "dispersion_rotated": (L.SD_FIELD_DISPERSION, view_default(rot=ry, rot_on=1, cmap=0, bright=0.5)),
    }


@pytest.mark.parametrize("name", list(_field_views()))
def test_field_view_matches_oracle(cuda, oracle, name):
    from stardust_b200.render import view_dict
    from stardust_b200.sim import Sim, SimConfig

    G, n = 64, 200_000
    pos, vel = scenes.disk_galaxy(n, 8)
    with Sim(0) as s:
        s.init(SimConfig(particle_count=n, grid_size=G))
        s.set_particles(pos, vel)
        rho = s.density()
    field, view = _field_views()[name]
    W, H = 400, 300
    img = _field_gpu(cuda, field, rho, pos, vel, G, view, W, H)
    ref = oracle.render_field(field, rho, pos, vel, G, view_dict(view), W, H)
    assert img.shape == (H, W, 4) and np.all(img[..., 3] == 255)
    d = np.abs(img[..., :3].astype(np.int32) - ref[..., :3].astype(np.int32))
    assert (d > 1).mean() < 5e-3, (d > 1).mean()
    assert d.mean() < 0.1
    assert ref[..., :3].max() > 60  # the scene is visible


def test_field_view_independent_of_particle_order_and_empty(cuda):
    from stardust_b200.render import view_default

    G = 32
    pos, vel = scenes.disk_galaxy(60_000, 9)
    view = view_default(rot=[0.8, 0.6, 0, -0.6, 0.8, 0, 0, 0, 1], rot_on=1, bright=0.5)
    rho = np.zeros((G, G, G), np.float32)
    a = _field_gpu(cuda, L.SD_FIELD_DISPERSION, rho, pos, vel, G, view, 160, 120)
    perm = np.random.default_rng(2).permutation(len(pos))
    b = _field_gpu(cuda, L.SD_FIELD_DISPERSION, rho, pos[perm], vel[perm], G, view, 160, 120)
    assert np.array_equal(a, b) and a[..., :3].max() > 0
    empty = _field_gpu(cuda, L.SD_FIELD_DENSITY, rho, pos[:1], vel[:1], G, view_default(), 64, 48)
    assert np.all(empty[..., :3] == 0) and np.all(empty[..., 3] == 255)


def test_field_view_of_a_sim(cuda):
    from stardust_b200.render import render_field
    from stardust_b200.sim import Sim, SimConfig

    with Sim(0) as s:
        s.init(SimConfig(particle_count=40_000, grid_size=32, spin=0.4))  # the Filament preset
        s.step(1e-3)
        dens = render_field(s, 128, 96)
        disp = render_field(s, 128, 96, L.SD_FIELD_DISPERSION, cmap=3)
    assert dens.shape == (96, 128, 4) and dens[..., :3].max() > 0 and disp[..., :3].max() > 0
