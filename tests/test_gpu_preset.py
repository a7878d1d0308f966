"""Initial conditions of Sim::init / Sim::reset (kPlace's Filament and Empty
presets, spin, Hubble flow, dispersion, centre-of-mass stop) through the C ABI,
against the unmodified reference's output (committed fixtures,
tests/golden/make_reference_fixtures.py) and the numpy restatement."""
import glob
import os

import numpy as np
import pytest

from stardust_b200 import _lib as L
from stardust_b200.sim import Sim, SimConfig

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# positions and velocities agree with the reference to float rounding: both use the
# same hash and the same fast sin/cos; the mean removed by the centre-of-mass stop
# is summed in a different order (FP64 atomics there)
POS_ATOL = 2e-6
VEL_ATOL = 2e-6


def preset_sim(n, G, **kw):
    s = Sim(0)
    s.init(SimConfig(particle_count=n, grid_size=G, **kw))
    return s


def _fixture_cfg(f):
    return dict(preset=int(f["preset"]), dark_matter_fraction=float(f["dark_matter_fraction"]),
                big_bang_shrink=float(f["big_bang_shrink"]), spin=float(f["spin"]), hubble=float(f["hubble"]),
                vel_dispersion=float(f["vel_dispersion"]))


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "reference_preset_*.npz"))),
                         ids=lambda p: os.path.basename(p)[17:-4])
def test_init_lays_down_the_reference_preset(cuda, path):
    f = np.load(path)
    n, G = int(f["n"]), int(f["grid"])
    with preset_sim(n, G, **_fixture_cfg(f)) as s:
        p, v = s.get_particles()
        active = s.active_count()
    live = f["pos"][:, 0] >= 0
    assert np.array_equal(p[:, 0] >= 0, live)
    assert np.array_equal(v[:, 3], f["vel"][:, 3])  # dark-matter marks
    assert np.abs(p[live, :3] - f["pos"][live, :3]).max() <= POS_ATOL
    assert np.abs(v[:, :3] - f["vel"][:, :3]).max() <= VEL_ATOL
    assert active == (n if int(f["preset"]) == L.SD_PRESET_FILAMENT else 0)


def test_filament_matches_oracle_at_size(cuda, oracle):
    n, G = 300_000, 64
    cfg = dict(dark_matter_fraction=0.2, big_bang_shrink=0.85, spin=0.6, hubble=0.3, vel_dispersion=0.08)
    with preset_sim(n, G, **cfg) as s:
        p, v = s.get_particles()
    po, vo = oracle.place_preset(n, oracle.PRESET_FILAMENT, 0.2, 0.85, 0.6, 0.3, 0.08)
    # libm sin/cos in the restatement against the fast intrinsics
    assert np.abs(p[:, :3] - po[:, :3]).max() < 2e-5
    assert np.abs(v[:, :3] - vo[:, :3]).max() < 2e-5
    assert np.array_equal(v[:, 3], vo[:, 3])
    r = np.linalg.norm(p[:, :3].astype(np.float64) - 0.5, axis=1)
    assert r.max() <= 0.5 * 0.85 + 1e-6  # the ball, shrunk
    assert abs((v[:, 3] == -100).mean() - 0.2) < 0.01
    assert np.abs(v[:, :3].astype(np.float64).mean(axis=0)).max() < 1e-6  # centre of mass at rest


def test_reset_lays_the_preset_down_again(cuda):
    n, G = 50_000, 32
    with preset_sim(n, G, spin=0.5, vel_dispersion=0.05) as s:
        p0, v0 = s.get_particles()
        rng = np.random.default_rng(3)
        pos = np.zeros((n, 4), np.float32)
        pos[:, :3] = rng.random((n, 3))
        s.set_particles(pos, np.zeros((n, 4), np.float32))
        s.step(1e-3)
        s.reset()
        assert s.sim_time() == 0.0 and s.step_count() == 0 and s.active_count() == n
        p1, v1 = s.get_particles()
        s.step(1e-3)  # steps from the laid-down preset
        assert s.active_count() == n
    assert np.array_equal(p0, p1) and np.array_equal(v0, v1)


def test_empty_preset_and_state_header(cuda, tmp_path):
    n, G = 20_000, 32
    with preset_sim(n, G, preset=L.SD_PRESET_EMPTY) as s:
        p, v = s.get_particles()
        assert s.active_count() == 0
        assert (p[:, 0] < 0).all()
        s.set_particles(p[:10] * 0 + 0.5, v[:10])
        path = str(tmp_path / "empty.stardust")
        s.save_state(path)
    hdr = np.fromfile(path, dtype=np.int32, count=19)
    assert hdr[5] == L.SD_PRESET_EMPTY  # STARDUST header field `preset` (Sim.cu:5017)
    with Sim(0) as t:
        t.init(SimConfig(particle_count=16, grid_size=16))
        t.load_state(path)
        assert t.config().preset == L.SD_PRESET_EMPTY
