"""The grid hydrodynamics add-ons (cooling toward the cell-mean velocity, a
pressure force from the velocity dispersion; Sim::Impl::doCooling and kPressure)
through the C ABI: against the numpy restatement step by step, against the
unmodified reference with both on (committed fixture), and the schedule under
graph replay."""
import os

import numpy as np
import pytest

from conftest import random_particles
from stardust_b200.sim import Sim, SimConfig

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def hydro_sim(n, G, **kw):
    s = Sim(0)
    kw.setdefault("softening_cells", 1.0)
    s.init(SimConfig(particle_count=n, grid_size=G, **kw))
    return s


def scene(n, seed):
    pos, vel = random_particles(n, seed, clustered=True)
    pos[:, 3] = 0.0  # gas ...
    pos[::10, 3] = 1.0  # ... and every tenth a star: counted in the cells, neither cooled nor pushed
    vel[:, :3] = np.random.default_rng(seed).normal(scale=0.3, size=(n, 3)).astype(np.float32)
    vel[:, 3] = np.arange(n, dtype=np.float32)  # ids: >= 0, so gas and not dark matter
    return pos, vel


def by_id(p, v):
    o = np.argsort(v[:, 3].astype(np.int64))
    return p[o], v[o]


def oracle_steps(oracle, pos, vel, G, dt, steps, pressure, pk, rate):
    """The reference's step order with gravity off: pressure field from the last
    dispersion, a cooling pass every period, kick, drift, wrap, momentum zeroing."""
    p, v = pos.copy(), vel.copy()
    period = 2 if pressure else 8
    disp, dcnt = np.zeros((3, G ** 3)), np.zeros(G ** 3, np.int64)
    for s in range(steps):
        acc = oracle.pressure_field(disp, dcnt, G, pk) if pressure else None
        if s % period == 0:
            k = min(rate * dt * period * 60.0, 0.5)
            v, d2, c2 = oracle.hydro_cool(p, v, G, k, pressure)
            if pressure:
                disp, dcnt = d2, c2
        if acc is not None:
            gas = (p[:, 0] >= 0) & (p[:, 3] <= 0) & (v[:, 3] >= -50)
            a = oracle.sample_field(acc, p, G).astype(np.float32)
            v[gas, :3] = v[gas, :3] + a[gas] * np.float32(dt)
        p[:, :3] = p[:, :3] + v[:, :3] * np.float32(dt)
        p[:, :3] -= np.floor(p[:, :3])
        live = p[:, 0] >= 0
        mean = (v[live, :3].astype(np.float64).sum(axis=0) / live.sum()).astype(np.float32)
        v[live, :3] -= mean
    return p, v


@pytest.mark.parametrize("pressure,cooling", [(1, 1), (1, 0), (0, 1)])
def test_hydro_steps_match_oracle(cuda, oracle, pressure, cooling):
    G, n, dt, steps = 16, 60_000, 1e-3, 9
    pos, vel = scene(n, 5)
    with hydro_sim(n, G, gravity=0.0, pressure_enabled=pressure, cooling_enabled=cooling) as s:
        s.set_particles(pos, vel)
        for _ in range(steps):
            s.step(dt)
        p1, v1 = by_id(*s.get_particles())
    po, vo = oracle_steps(oracle, pos, vel, G, dt, steps, bool(pressure), 0.45, 0.08 if cooling else 0.0)
    dv, dvo = v1[:, :3] - vel[:, :3], vo[:, :3] - vel[:, :3]
    assert np.sqrt(np.mean((dv - dvo) ** 2)) <= 1e-4 * np.sqrt(np.mean(dvo ** 2))
    assert np.abs(((p1[:, :3] - po[:, :3]) + 0.5) % 1.0 - 0.5).max() < 1e-6
    assert np.sqrt(np.mean(dvo ** 2)) > 1e-3  # the add-ons did change the velocities


def test_hydro_graph_replay_matches_eager(cuda):
    G, n = 16, 40_000
    pos, vel = scene(n, 6)
    outs = []
    for mode in ("eager", "graph"):
        with hydro_sim(n, G, gravity=50.0, pressure_enabled=1, cooling_enabled=1, order=2) as s:
            s.set_particles(pos, vel)
            if mode == "eager":
                for _ in range(11):
                    s.step(1e-3)
            else:  # odd counts move the cooling phase between graph captures
                s.steps(1e-3, 3)
                s.step(1e-3)
                s.steps(1e-3, 4)
                s.steps(1e-3, 3)
            outs.append(s.get_particles())
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def test_toggling_hydro_keeps_the_particles(cuda):
    G, n = 16, 20_000
    pos, vel = scene(n, 7)
    with hydro_sim(n, G, gravity=1.0) as s:
        s.set_particles(pos, vel)
        s.step(1e-3)
        p0, v0 = s.get_particles()
        cfg = s.config()
        cfg.pressure_enabled = 1
        cfg.cooling_enabled = 1
        s.reconfigure(cfg)
        p1, v1 = s.get_particles()
        s.steps(1e-3, 4)
        assert s.active_count() == n
    assert np.array_equal(p0, p1) and np.array_equal(v0, v1)


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLDEN, "reference_hydro_g16.npz")),
                    reason="no hydro fixture committed")
def test_hydro_steps_match_reference_fixture(cuda):
    """Three steps of the unmodified reference with pressure and cooling on."""
    f = np.load(os.path.join(GOLDEN, "reference_hydro_g16.npz"))
    G, grav, soft = int(f["grid"]), float(f["gravity"]), float(f["soft"])
    pos0, vel0 = f["pos_in"], f["vel_in"]
    n = len(pos0)
    with hydro_sim(n, G, gravity=grav, softening_cells=soft, pressure_enabled=1, pressure_k=float(f["pressure_k"]),
                   cooling_enabled=1, cooling_rate=float(f["cooling_rate"])) as s:
        s.set_particles(pos0, vel0)
        for k, dt in enumerate(f["dt_used"]):
            s.step(float(dt))
            p1, v1 = by_id(*s.get_particles())
            pr, vr = by_id(f["pos_steps"][k], f["vel_steps"][k])
            dv, dvr = v1[:, :3] - vel0[:, :3], vr[:, :3] - vel0[:, :3]
            err = np.sqrt(np.mean((dv - dvr) ** 2)) / np.sqrt(np.mean(dvr ** 2))
            assert err < 2e-4, (k, err)
            assert np.abs(((p1[:, :3] - pr[:, :3]) + 0.5) % 1.0 - 0.5).max() < 2e-6
