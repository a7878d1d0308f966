"""The isolated (Hockney-Eastwood) boundary, the reference's default: potential,
accelerations and one whole step against the FP64 oracle (clamped deposit,
Green's function of the 2G box, clamped gradient and gather, the wall), through
the C ABI."""
import numpy as np
import pytest

from conftest import random_particles
from stardust_b200 import _lib as L
from stardust_b200.sim import Sim, SimConfig

pytestmark = pytest.mark.gpu


def iso_sim(n, G, **kw):
    kw.setdefault("softening_cells", 1.5)
    s = Sim(0)
    s.init(SimConfig(particle_count=n, grid_size=G, boundary=L.SD_BOUNDARY_ISOLATED, **kw))
    return s


def scene(n, seed, lo=0.05, hi=0.95):
    pos, vel = random_particles(n, seed, clustered=True)
    pos[:, :3] = lo + (hi - lo) * pos[:, :3]
    # a few particles against the walls, where corners are clamped
    pos[:8, 0] = [0.0005, 0.001, 0.0021, 0.999, 0.9985, 0.5, 0.5, 0.5]
    pos[5:8, 2] = [0.0005, 0.9995, 0.001]
    return pos.astype(np.float32), vel.astype(np.float32)


def rel_rms(a, b):
    d = np.sqrt(np.mean(np.sum((np.asarray(a, np.float64) - b) ** 2, axis=-1)))
    return d / np.sqrt(np.mean(np.sum(np.asarray(b, np.float64) ** 2, axis=-1)))


@pytest.mark.parametrize("G", [32, 64])
def test_isolated_potential_and_accel_match_fp64(cuda, oracle, G):
    n = 60_000
    pos, vel = scene(n, G)
    with iso_sim(n, G) as s:
        s.set_particles(pos, vel)
        a = s.accel()[:, :3]
        phi = s.potential()
        rho = s.density()
    rho64 = oracle.density_iso_f64(pos, G)
    assert np.abs(rho - rho64).max() < 1e-5 * rho64.max()
    assert float(rho.sum(dtype=np.float64)) == pytest.approx(n, rel=1e-6)  # clamping keeps every weight
    phi64 = oracle.poisson_isolated_f64(rho64, 1.5)
    assert np.abs(phi - phi64).max() < 2e-5 * np.abs(phi64).max()
    a64 = oracle.pm_accel_iso_f64(pos, G, 1.0 / n, 1.5)
    assert rel_rms(a, a64) < 5e-5


def test_isolated_newton_units_scale_by_grid(cuda):
    G, n = 32, 20_000
    pos, vel = scene(n, 3)
    out = {}
    for units in (L.SD_UNITS_REFERENCE, L.SD_UNITS_NEWTON):
        with iso_sim(n, G, units=units) as s:
            s.set_particles(pos, vel)
            out[units] = s.accel()[:, :3]
    # -1/r in cell units: Newton's G = 1 with masses 1/N is G times the reference's gravity/N
    assert np.allclose(out[L.SD_UNITS_NEWTON], G * out[L.SD_UNITS_REFERENCE], rtol=1e-5, atol=1e-30)


def test_isolated_step_matches_oracle_with_wall(cuda, oracle):
    G, n = 32, 30_000
    pos, vel = scene(n, 5)
    vel[:, :3] *= 0.0
    vel[:8, 0] = [-2.0, -1.0, -3.0, 2.0, 4.0, 0.0, 0.0, 0.0]  # into the walls
    vel[5:8, 2] = [-2.0, 3.0, -1.0]
    vel[:, 3] = np.arange(n, dtype=np.float32)  # identity, carried through the sort
    dt = 1e-3
    with iso_sim(n, G, gravity=50.0) as s:
        s.set_particles(pos, vel)
        s.step(dt)
        p1, v1 = s.get_particles()
    ids = v1[:, 3].astype(np.int64)
    p1, v1 = p1[np.argsort(ids)], v1[np.argsort(ids)]
    a = oracle.pm_accel_iso_f64(pos, G, 50.0 / n, 1.5)
    vk = (vel[:, :3] + a * dt).astype(np.float32)
    pk = (pos[:, :3] + vk * dt).astype(np.float32)
    pw, vw = oracle.isolated_wall(pk, vk)
    vw -= vw.mean(axis=0, dtype=np.float64).astype(np.float32)  # momentum zeroing after the step
    assert np.abs(p1[:, :3] - pw).max() < 2e-6
    assert rel_rms(v1[:, :3], vw) < 1e-4
    # the wall: every coordinate inside [0.002, 0.998], wall hits reversed at a quarter speed
    assert p1[:, :3].min() >= 0.002 and p1[:, :3].max() <= 0.998
    assert p1[3, 0] == np.float32(0.998) and v1[3, 0] < 0
    assert p1[0, 0] == np.float32(0.002) and v1[0, 0] > 0


def test_isolated_mass_conserved_over_steps(cuda):
    G, n = 32, 50_000
    pos, vel = scene(n, 7)
    with iso_sim(n, G, gravity=20.0, order=L.SD_ORDER_TILED) as s:
        s.set_particles(pos, vel)
        m0 = s.measure_total_grid_mass()
        s.steps(1e-3, 20)
        s.step(1e-3)
        m1 = s.measure_total_grid_mass()
        assert s.active_count() == n
    assert m0 == pytest.approx(n, rel=1e-6) and m1 == pytest.approx(n, rel=1e-6)


def test_isolated_state_round_trip(cuda, tmp_path):
    G, n = 32, 10_000
    pos, vel = scene(n, 9)
    path = str(tmp_path / "iso.stardust")
    with iso_sim(n, G) as s:
        s.set_particles(pos, vel)
        s.step(1e-3)
        s.save_state(path)
        p0, v0 = s.get_particles()
    with Sim(0) as t:
        t.init(SimConfig(particle_count=16, grid_size=16))
        t.load_state(path)
        assert t.config().boundary == L.SD_BOUNDARY_ISOLATED and t.grid_size() == G
        p1, v1 = t.get_particles()
    assert np.array_equal(p0, p1) and np.array_equal(v0, v1)


def test_isolated_step_matches_reference_fixture(cuda):
    """One step of the unmodified reference in isolated mode (committed fixture,
    tests/golden/make_reference_fixtures.py) reproduced through the C ABI."""
    import os

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_isolated_g32.npz")
    f = np.load(path)
    G, grav, soft, dt = int(f["grid"]), float(f["gravity"]), float(f["soft"]), float(f["dt"])
    pos0, vel0 = f["pos_in"], f["vel_in"]
    n = len(pos0)
    with iso_sim(n, G, gravity=grav, softening_cells=soft) as s:
        s.set_particles(pos0, vel0)
        rho = s.density()
        s.step(dt)
        p1, v1 = s.get_particles()
    assert np.abs(rho - f["rho_loaded"]).max() <= 2e-5 * float(f["rho_loaded"].max())
    order = np.argsort(v1[:, 3].astype(np.int64))
    ref_order = np.argsort(f["vel_out"][:, 3].astype(np.int64))
    p1, v1 = p1[order], v1[order]
    p_ref, v_ref = f["pos_out"][ref_order], f["vel_out"][ref_order]
    dv, dv_ref = v1[:, :3] - vel0[:, :3], v_ref[:, :3] - vel0[:, :3]
    assert rel_rms(dv, dv_ref) < 1e-4
    assert np.abs(p1[:, :3] - p_ref[:, :3]).max() < 2e-6
