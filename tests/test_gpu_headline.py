"""Whole-step parity at the benchmark sizes, through the C ABI.

16,777,216 particles on a 512^3 grid (the Zel'dovich field of the headline
benchmark) and 4,194,304 particles on 256^3 (the two-galaxy encounter), each in
the reference's row-major order (Sim.cu:2476-2486) and in the tiled order the
timed step runs (the balanced fused deposit, and from the second step on the
merge sort of the keys that changed). Two steps per case: the first from the
seeded input, the second from the GPU's own state after the first, each checked
against one oracle step from the same particles:
  - the density of the step-start positions bit for bit (fixed-point sums);
  - the sort permutation exactly (row-major: the reference's cell-key order;
    tiled: the stable sort of the tile-row keys);
  - the velocity change within DV_RTOL relative RMS and positions within DP_ATOL.
"""
import numpy as np
import pytest

from stardust_b200 import _lib as L
from stardust_b200 import scenes
from stardust_b200.sim import Sim, SimConfig

pytestmark = pytest.mark.gpu

DV_RTOL = 1e-4   # relative RMS of the velocity change against the oracle's
DP_ATOL = 2e-6   # box units

SCENES = {
    "cosmic_web_512": (lambda: scenes.zeldovich(256, 2), 512, 1e-3),
    "two_galaxy_256": (lambda: scenes.two_galaxies(4_194_304, 1), 256, 5e-4),
}
_cache = {}


def scene(name):
    if name not in _cache:
        make, G, dt = SCENES[name]
        pos, vel = make()
        vel = vel.copy()
        vel[:, 3] = np.arange(len(vel), dtype=np.float32)  # ids through the sort
        _cache.clear()  # one large scene in memory at a time
        _cache[name] = (pos, vel, G, dt)
    return _cache[name]


def rel_rms(a, b):
    d = np.sqrt(np.mean(np.sum((a.astype(np.float64) - b) ** 2, axis=-1)))
    return d / np.sqrt(np.mean(np.sum(b.astype(np.float64) ** 2, axis=-1)))


def check_step(oracle, order, G, grav, dt, p0, v0, p1, v1, rho1):
    """One GPU step (p0, v0) -> (p1, v1) with step-start density rho1 against the oracle."""
    p_ref, v_ref, rho_ref, _ = oracle.step(p0, v0, G, grav, 1.0, dt, dt, key_mode=order)
    assert np.array_equal(rho1.view(np.int32), rho_ref.view(np.int32)), "density differs from the oracle"
    ids, ids_ref = v1[:, 3].astype(np.int64), v_ref[:, 3].astype(np.int64)
    assert np.array_equal(ids, ids_ref), "sort permutation differs from the oracle"
    # velocity change per particle: inputs indexed by id through the permutation
    v0_by_id = np.empty_like(v0[:, :3])
    v0_by_id[v0[:, 3].astype(np.int64)] = v0[:, :3]
    dv, dv_ref = v1[:, :3] - v0_by_id[ids], v_ref[:, :3] - v0_by_id[ids_ref]
    err = rel_rms(dv, dv_ref)
    assert err < DV_RTOL, f"velocity change rel RMS {err:.2e}"
    dp = np.abs((p1[:, :3] - p_ref[:, :3] + 0.5) % 1.0 - 0.5).max()
    assert dp < DP_ATOL, f"position difference {dp:.2e}"
    return err


@pytest.mark.parametrize("order", [L.SD_ORDER_TILED, L.SD_ORDER_ROWMAJOR], ids=["tiled", "rowmajor"])
@pytest.mark.parametrize("name", sorted(SCENES))
def test_two_steps_at_benchmark_size(cuda, oracle, name, order):
    pos, vel, G, dt = scene(name)
    n = len(pos)
    grav = float(4 * np.pi * G ** 3)  # Newton G = 1 in the reference's formula
    cfg = SimConfig(particle_count=n, grid_size=G, gravity=grav, softening_cells=1.0, order=order, keep_density=1)
    with Sim(0) as s:
        s.init(cfg)
        s.set_particles(pos, vel)
        s.step(dt)
        p1, v1 = s.get_particles()
        rho1 = s.density()
        s.step(dt)  # tiled: merges the keys the first step changed
        p2, v2 = s.get_particles()
        rho2 = s.density()
    check_step(oracle, order, G, grav, dt, pos, vel, p1, v1, rho1)
    check_step(oracle, order, G, grav, dt, p1, v1, p2, v2, rho2)
