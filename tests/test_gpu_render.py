"""Headless point render (sd_render_points) against the numpy restatement of the
reference's kSplatPoints -> kAccumToRGBA, and order independence."""
import math

import numpy as np
import pytest

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
