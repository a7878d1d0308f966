"""Whole-step parity and behaviour of the simulation handle (through the C ABI)."""
import numpy as np
import pytest

from conftest import random_particles
from stardust_b200 import _lib as L
from stardust_b200 import scenes
from stardust_b200.sim import Sim, SimConfig

pytestmark = pytest.mark.gpu

# one step from identical inputs: relative RMS of the velocity change and the
# absolute position difference (box units) allowed against the oracle
DV_RTOL = 1e-4
DP_ATOL = 2e-6


def make_sim(cuda, n, G, **kw):
    cfg = SimConfig(particle_count=n, grid_size=G, **kw)
    s = Sim(0)
    s.init(cfg)
    return s


def rel_rms(a, b):
    d = np.sqrt(np.mean(np.sum((a.astype(np.float64) - b) ** 2, axis=-1)))
    r = np.sqrt(np.mean(np.sum(b.astype(np.float64) ** 2, axis=-1)))
    return d / r


def wrapdiff(a, b):
    return (a - b + 0.5) % 1.0 - 0.5


@pytest.mark.parametrize("order", [L.SD_ORDER_ROWMAJOR, L.SD_ORDER_MORTON, L.SD_ORDER_TILED])
def test_one_step_matches_oracle(cuda, oracle, order):
    G, n = 64, 262_144
    pos, vel = scenes.disk_galaxy(n, 0)
    vel[:, 3] = np.arange(n, dtype=np.float32)
    grav = float(4 * np.pi * G ** 3)  # Newton G = 1 in the reference's formula
    dt = 1e-3
    with make_sim(cuda, n, G, gravity=grav, softening_cells=1.0, order=order) as s:
        s.set_particles(pos, vel)
        rho0 = s.density()  # density of the loaded positions
        s.step(dt)
        p1, v1 = s.get_particles()
        rho1 = s.density()
    ref_rho = oracle.density_fixed(pos, G)
    assert np.array_equal(rho0.view(np.int32), ref_rho.view(np.int32))
    assert np.array_equal(rho1.view(np.int32), ref_rho.view(np.int32))  # sort does not move particles
    p_ref, v_ref, _, _ = oracle.step(pos, vel, G, grav, 1.0, dt, dt, key_mode=order)
    ids, ids_ref = v1[:, 3].astype(np.int64), v_ref[:, 3].astype(np.int64)
    assert np.array_equal(ids, ids_ref)  # identical sort permutation
    dv = v1[:, :3] - vel[ids, :3]
    dv_ref = v_ref[:, :3] - vel[ids_ref, :3]
    assert rel_rms(dv, dv_ref) < DV_RTOL
    assert np.abs(wrapdiff(p1[:, :3], p_ref[:, :3])).max() < DP_ATOL


def test_multi_step_determinism_and_graph_replay(cuda):
    G, n = 64, 200_000
    pos, vel = random_particles(n, 1, empty_every=101, clustered=True)
    outs = []
    for mode in ("eager", "eager", "graph"):
        with make_sim(cuda, n, G, gravity=100.0, softening_cells=1.0) as s:
            s.set_particles(pos, vel)
            if mode == "graph":
                s.steps(1e-3, 7)
            else:
                for _ in range(7):
                    s.step(1e-3)
            outs.append(s.get_particles())
            assert s.step_count() == 7
            assert s.sim_time() == pytest.approx(7e-3)
    for p, v in outs[1:]:
        assert np.array_equal(p.view(np.int32), outs[0][0].view(np.int32))
        assert np.array_equal(v.view(np.int32), outs[0][1].view(np.int32))


def test_mass_conservation_and_momentum_zeroing(cuda):
    # reference invariant: mass conservation over 50 steps, rel < 1e-3 (tests/sim_tests.cpp:31-52)
    G, n = 64, 100_000
    pos, vel = random_particles(n, 3, clustered=True)
    with make_sim(cuda, n, G, gravity=500.0) as s:
        s.set_particles(pos, vel)
        m0 = s.measure_total_grid_mass()
        for _ in range(50):
            s.step(1e-3)
        m1 = s.measure_total_grid_mass()
        p, v = s.get_particles()
    assert m0 == pytest.approx(n, rel=1e-6)
    assert abs(m1 - m0) / m0 < 1e-3
    assert np.abs(v[:, :3].astype(np.float64).mean(axis=0)).max() < 1e-6
    assert ((p[:, :3] >= 0) & (p[:, :3] < 1)).all()


def test_clumping_increases_with_gravity(cuda):
    # reference invariant (tests/sim_tests.cpp:58-82): stronger gravity -> denser peaks
    G, n = 32, 50_000
    pos, vel = random_particles(n, 4)
    vel[:, :3] = 0
    peaks = []
    # Newton G = 0 and G = 10 (growth rate sqrt(4 pi G rho) ~ 11 per unit time)
    for grav in (0.0, 10.0):
        with make_sim(cuda, n, G, gravity=grav, units=L.SD_UNITS_NEWTON, softening_cells=0.5) as s:
            s.set_particles(pos, vel)
            for _ in range(60):
                s.step(5e-3)
            s.step(1e-6)
            peaks.append(s.measure_max_density())
    assert peaks[1] > 1.5 * peaks[0]


def test_step_auto_uses_reference_cfl(cuda, oracle):
    G, n = 32, 20_000
    pos, vel = random_particles(n, 5)
    vel[7, :3] = (20.0, 0.0, 0.0)  # fast particle: CFL must clamp
    with make_sim(cuda, n, G, gravity=1.0, time_scale=1.0) as s:
        s.set_particles(pos, vel)
        s.step()
        t = s.timings()
    vmax = oracle.max_speed(pos, vel)
    expect = min(np.float32(0.0016), np.float32(0.8) * np.float32(1.0 / G) / np.float32(vmax))
    assert t["max_speed"] == pytest.approx(vmax, rel=1e-6)
    assert t["dt_used"] == pytest.approx(float(expect), rel=1e-6)


def test_save_load_round_trip(cuda, tmp_path):
    G, n = 32, 30_000
    pos, vel = random_particles(n, 6, empty_every=9)
    path = tmp_path / "state.bin"
    with make_sim(cuda, n, G, gravity=50.0) as s:
        s.set_particles(pos, vel)
        for _ in range(3):
            s.step(1e-3)
        s.save_state(str(path))
        p_a, v_a = s.get_particles()
        for _ in range(2):
            s.step(1e-3)
        p_b, v_b = s.get_particles()
    raw = open(path, "rb").read()
    assert raw[:8] == b"STARDUST" and len(raw) == 76 + 32 * n
    with make_sim(cuda, 10, 16) as s2:
        s2.load_state(str(path))
        assert s2.particle_count() == n and s2.grid_size() == G
        p_l, v_l = s2.get_particles()
        assert np.array_equal(p_l, p_a) and np.array_equal(v_l, v_a)
        assert s2.sim_time() == pytest.approx(3e-3, rel=1e-6)
        for _ in range(2):
            s2.step(1e-3)
        p_c, v_c = s2.get_particles()
    assert np.array_equal(p_c.view(np.int32), p_b.view(np.int32))
    assert np.array_equal(v_c.view(np.int32), v_b.view(np.int32))


def test_leapfrog_energy_conservation_better_than_kd(cuda):
    G, n = 32, 40_000
    pos, vel = scenes.zeldovich(32, 9)
    n = len(pos)
    drift = {}
    for integ in (L.SD_INT_KD, L.SD_INT_KDK):
        with make_sim(cuda, n, G, gravity=1.0, units=L.SD_UNITS_NEWTON, integrator=integ, softening_cells=1.0,
                      diagnostics=0) as s:
            s.set_particles(pos, vel)
            s.accel()  # field of the current positions for the potential energy
            d0 = s.diagnostics()
            for _ in range(40):
                s.step(2e-3)
            s.synchronize()
            s.accel()
            d1 = s.diagnostics()
        e0 = d0["kinetic"] + d0["potential"]
        e1 = d1["kinetic"] + d1["potential"]
        drift[integ] = abs(e1 - e0) / abs(d0["potential"])
    assert drift[L.SD_INT_KDK] < drift[L.SD_INT_KD]


def test_accel_matches_fp64_pm(cuda, oracle):
    """Force error of the float pipeline against the FP64 PM oracle on the same grid."""
    G, n = 64, 100_000
    pos, vel = random_particles(n, 10, clustered=True)
    with make_sim(cuda, n, G, gravity=1.0, units=L.SD_UNITS_NEWTON, softening_cells=1.0) as s:
        s.set_particles(pos, vel)
        a = s.accel()[:, :3]
    a64 = oracle.pm_accel_f64(pos, G, 4 * np.pi * G ** 3 / n, 1.0)
    err = oracle.force_error(a, a64)
    assert err["rms_rel"] < 1e-5, err
    assert err["max_rel"] < 1e-3, err


def test_kernel_launches_counted(cuda):
    with make_sim(cuda, 1000, 16) as s:
        pos, vel = random_particles(1000, 2)
        s.set_particles(pos, vel)
        before = Sim.kernel_launches()
        s.step(1e-3)
        assert Sim.kernel_launches() - before >= 10


@pytest.mark.parametrize("G,n,clustered", [(16, 30_000, True), (64, 262_144, True), (128, 400_000, False),
                                         (512, 2_000_000, True)])
def test_fused_tiled_deposit_equals_generic_path(cuda, G, n, clustered):
    """The tiled order deposits inside the first FFT pass; the row-major order uses
    int64 atomics on a grid. Both are fixed-point, so after sorting the same
    particles the densities and the resulting step must agree bit for bit."""
    pos, vel = random_particles(n, G + 7, empty_every=41, clustered=clustered)
    out = {}
    for order in (L.SD_ORDER_ROWMAJOR, L.SD_ORDER_TILED):
        with make_sim(cuda, n, G, gravity=float(4 * np.pi * G ** 3), softening_cells=1.0, order=order) as s:
            s.set_particles(pos, vel)
            s.step(1e-3)
            rho = s.density()
            p, v = s.get_particles()
        key = np.lexsort((v[:, 3],))  # compare as sets keyed by particle id
        out[order] = (rho, p[key], v[key])
    a, b = out[L.SD_ORDER_ROWMAJOR], out[L.SD_ORDER_TILED]
    assert np.array_equal(a[0].view(np.int32), b[0].view(np.int32))
    assert np.array_equal(a[1].view(np.int32), b[1].view(np.int32))
    assert np.array_equal(a[2].view(np.int32), b[2].view(np.int32))


def test_tiled_graph_replay_matches_eager(cuda):
    G, n = 64, 150_000
    pos, vel = random_particles(n, 12, clustered=True)
    outs = []
    for mode in ("eager", "graph"):
        with make_sim(cuda, n, G, gravity=300.0, softening_cells=1.0, order=L.SD_ORDER_TILED) as s:
            s.set_particles(pos, vel)
            if mode == "graph":
                s.steps(1e-3, 6)
            else:
                for _ in range(6):
                    s.step(1e-3)
            outs.append(s.get_particles())
    assert np.array_equal(outs[0][0].view(np.int32), outs[1][0].view(np.int32))
    assert np.array_equal(outs[0][1].view(np.int32), outs[1][1].view(np.int32))


def test_graph_replay_across_calls_and_parity(cuda):
    """Odd step counts and interleaved eager steps leave the particles in either
    ping-pong buffer; later graph replays must still match plain stepping."""
    G, n = 32, 60_000
    pos, vel = random_particles(n, 21, clustered=True)
    outs = []
    for mode in ("eager", "mixed"):
        with make_sim(cuda, n, G, gravity=200.0, softening_cells=1.0, order=L.SD_ORDER_TILED) as s:
            s.set_particles(pos, vel)
            if mode == "eager":
                for _ in range(12):
                    s.step(1e-3)
            else:
                s.steps(1e-3, 3)
                s.step(1e-3)
                s.steps(1e-3, 5)
                s.steps(1e-3, 3)
            outs.append(s.get_particles())
    assert np.array_equal(outs[0][0].view(np.int32), outs[1][0].view(np.int32))
    assert np.array_equal(outs[0][1].view(np.int32), outs[1][1].view(np.int32))


@pytest.mark.parametrize("order", [L.SD_ORDER_TILED, L.SD_ORDER_MORTON])
def test_sort_counts_follow_new_particles(cuda, order):
    """The gather leaves the next sort's first-pass digit counts behind; replacing
    the particles between (graph-replayed) steps must not let a stale count reach
    the sort: the run equals a fresh one stepped eagerly from the new particles."""
    G, n = 32, 80_000
    a = random_particles(n, 31, clustered=True)
    b = random_particles(n, 32, empty_every=53, clustered=True)
    with make_sim(cuda, n, G, gravity=200.0, softening_cells=1.0, order=order) as s:
        s.set_particles(*a)
        s.steps(1e-3, 4)
        s.set_particles(*b)
        s.steps(1e-3, 4)
        s.step(1e-3)
        s.steps(1e-3, 2)
        got = s.get_particles()
    with make_sim(cuda, n, G, gravity=200.0, softening_cells=1.0, order=order) as t:
        t.set_particles(*b)
        for _ in range(7):
            t.step(1e-3)
        want = t.get_particles()
    assert np.array_equal(got[0].view(np.int32), want[0].view(np.int32))
    assert np.array_equal(got[1].view(np.int32), want[1].view(np.int32))


def test_per_step_diagnostics_record_energy_and_momentum(cuda):
    """diagnostics = 1: every step (eager or graph-replayed) appends an FP64 record
    whose potential is that of the step-start state and whose kinetic energy is
    that of the zeroed end velocities."""
    pos, vel = scenes.zeldovich(32, 9)
    n = len(pos)
    with make_sim(cuda, n, 32, gravity=1.0, units=L.SD_UNITS_NEWTON, softening_cells=1.0, diagnostics=1,
                  order=L.SD_ORDER_TILED) as s:
        s.set_particles(pos, vel)
        s.accel()
        d0 = s.diagnostics()
        s.step(1e-3)
        h = s.diagnostics_history()
        assert h.shape == (1, 8)
        assert h[0, 2] == pytest.approx(d0["potential"], rel=1e-5)
        d1 = s.diagnostics()
        assert h[0, 1] == pytest.approx(d1["kinetic"], rel=1e-9)
        assert np.abs(h[0, 3:6]).max() <= 1e-6 * np.sqrt(2 * h[0, 1])
        assert h[0, 6] == n
        s.steps(1e-3, 10)  # captured-graph replays record too
        h = s.diagnostics_history()
        assert h.shape == (11, 8)
        assert np.array_equal(h[:, 0], np.arange(11))
        e = h[:, 1] + h[:, 2]
        assert np.abs(e - e[0]).max() <= 1e-2 * abs(h[0, 2])


@pytest.mark.parametrize("order,diag", [(L.SD_ORDER_TILED, 1), (L.SD_ORDER_ROWMAJOR, 0)])
def test_step_host_equals_set_step_get(cuda, order, diag):
    """sd_step_host overlaps its copies with the step; the result is that of
    set_particles + step + get_particles, bit for bit (also with n below capacity)."""
    G, N, n = 32, 70_000, 65_000
    outs = []
    for mode in ("separate", "host"):
        with make_sim(cuda, N, G, gravity=300.0, softening_cells=1.0, order=order, diagnostics=diag) as s:
            for k in range(3):
                pos, vel = random_particles(n, 40 + k, clustered=True)
                if mode == "separate":
                    s.set_particles(pos, vel)
                    s.step(1e-3)
                    p, v = s.get_particles(n)
                else:
                    p, v = s.step_host(pos, vel, 1e-3)
                outs.append((p, v))
    for (a, b), (c, d) in zip(outs[:3], outs[3:]):
        assert np.array_equal(a.view(np.int32), c.view(np.int32))
        assert np.array_equal(b.view(np.int32), d.view(np.int32))


@pytest.mark.parametrize("order", [L.SD_ORDER_ROWMAJOR, L.SD_ORDER_TILED])
def test_pipelined_offload_equals_offload_step(cuda, order):
    """sd_step_host_async queues upload, step and download and returns; five calls
    in a row (inputs staged in a third particle set while the previous result
    downloads) give each step's result bit for bit as sd_step_host does, also with
    n below capacity, and the handle is usable normally afterwards."""
    G, N, n = 32, 70_000, 65_000
    ins = [random_particles(n, 60 + k, clustered=True) for k in range(5)]
    with make_sim(cuda, N, G, gravity=300.0, softening_cells=1.0, order=order) as s:
        ref = [s.step_host(p, v, 1e-3) for p, v in ins]
    pinned = [(cuda.from_numpy(p).pin_memory(), cuda.from_numpy(v).pin_memory()) for p, v in ins]
    outs = [(cuda.empty((n, 4), dtype=cuda.float32).pin_memory(), cuda.empty((n, 4), dtype=cuda.float32).pin_memory())
            for _ in ins]
    with make_sim(cuda, N, G, gravity=300.0, softening_cells=1.0, order=order) as s:
        for (p, v), o in zip(pinned, outs):
            s.step_host_async(p, v, 1e-3, o)
        s.step_host_wait()
        for (p, v), (a, b) in zip(ref, outs):
            assert np.array_equal(p.view(np.int32), a.numpy().view(np.int32))
            assert np.array_equal(v.view(np.int32), b.numpy().view(np.int32))
        # the handle holds the last result and steps on from it as usual
        p_last, v_last = s.get_particles(n)
        assert np.array_equal(p_last.view(np.int32), outs[-1][0].numpy().view(np.int32))
        s.step(1e-3)
        assert s.get_particles(n)[0].shape == (n, 4)


@pytest.mark.parametrize("n,speed,merges", [(1 << 22, 0.05, True), (1 << 22, 3.0, False), (300_000, 0.05, False)])
def test_merge_gives_way_to_the_full_sort_when_many_keys_change(cuda, n, speed, merges):
    """By default the merge sort measures the share of changed keys; above 10 % the
    steps run the full radix sort instead, and below 2^22 particles they always
    do. Slow particles keep merging, fast ones switch, a small scene never
    merges; every step equals the full sort's bit for bit, eagerly and in graph
    replay."""
    G = 64
    pos, vel = _mover_scene(n, 7, speed)
    outs = []
    for full in (0, 1):
        with make_sim(cuda, n, G, gravity=100.0, softening_cells=1.0, order=L.SD_ORDER_TILED, full_sort=full) as s:
            s.set_particles(pos, vel)
            for _ in range(4):
                s.step(1e-3)
            s.get_particles()  # the measured share reaches the host by the time this returns
            s.steps(1e-3, 6)
            s.step(1e-3)
            outs.append(s.get_particles())
            if not full:
                assert s.merge_sorting() == merges
                frac = s.changed_fraction()
                if n >= 1 << 22:
                    assert 0.0 <= frac <= 1.0
                    assert (frac <= 0.10) == merges
                else:
                    assert frac == -1.0  # never merged, never measured
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a.view(np.int32), b.view(np.int32))


def _mover_scene(n, seed, speed):
    """Particles moving fast enough that many cross rows (y and z, across the
    4x4-row bundles) every step, with empty slots."""
    pos, vel = random_particles(n, seed, empty_every=37, clustered=True)
    rng = np.random.default_rng(seed)
    vel[:, :3] = rng.normal(scale=speed, size=(n, 3)).astype(np.float32)
    vel[:, 3] = np.arange(n, dtype=np.float32)
    return pos, vel


# (16, 1000): fewer positions than one chunk of change words; (64, 262144): n / 32
# an exact number of chunks, so the padding word opens a chunk of its own;
# (64, 2.5M, fast): nearly every key changes, and the changed set's sort loops its
# grids over more tiles than they hold CTAs
@pytest.mark.parametrize("G,n,speed", [(16, 40_000, 3.0), (64, 300_000, 1.0), (128, 200_000, 0.2), (16, 1_000, 3.0),
                                       (64, 262_144, 1.0), (64, 2_500_000, 40.0)])
def test_merge_sort_equals_full_sort(cuda, G, n, speed):
    """After a sorted step the tiled order merges the keys that changed into the
    rest instead of radix-sorting everything; the particles must come out the
    same, bit for bit, eagerly and under graph replay, across a reload."""
    pos, vel = _mover_scene(n, G, speed)
    b_pos, b_vel = _mover_scene(n, G + 1, speed)
    outs = []
    for full in (1, -1):  # the full sort, and the merge forced at these sizes
        with make_sim(cuda, n, G, gravity=200.0, softening_cells=1.0, order=L.SD_ORDER_TILED, full_sort=full) as s:
            s.set_particles(pos, vel)
            got = []
            for _ in range(5):
                s.step(1e-3)
            got.append(s.get_particles())
            s.steps(1e-3, 6)
            got.append(s.get_particles())
            s.set_particles(b_pos, b_vel)
            s.step(1e-3)
            s.steps(1e-3, 3)
            got.append(s.get_particles())
            outs.append(got)
    for (p0, v0), (p1, v1) in zip(outs[0], outs[1]):
        assert np.array_equal(p0.view(np.int32), p1.view(np.int32))
        assert np.array_equal(v0.view(np.int32), v1.view(np.int32))


def test_merge_sort_with_particles_lost_and_keys_unchanged(cuda):
    """A step where nothing crosses a row (all keys unchanged) and steps where
    some particles are lost (non-finite) merge like the full sort."""
    G, n = 32, 50_000
    pos, vel = random_particles(n, 3, clustered=True)
    vel[:, :3] = 0.0
    vel[:, 3] = np.arange(n, dtype=np.float32)
    outs = []
    for full in (1, -1):  # the full sort, and the merge forced at these sizes
        with make_sim(cuda, n, G, gravity=0.0, softening_cells=1.0, order=L.SD_ORDER_TILED, full_sort=full) as s:
            s.set_particles(pos, vel)
            s.step(1e-3)
            s.step(1e-3)  # no key changes: the merge is the identity
            p, v = s.get_particles()
            v[::997, 0] = np.inf  # lose a few particles in the next step
            v[::13, :3] = np.random.default_rng(1).normal(scale=5.0, size=(len(v[::13]), 3))
            s.set_particles(p, v)
            s.step(1e-3)
            s.step(1e-3)
            s.step(1e-3)
            outs.append(s.get_particles())
    assert np.array_equal(outs[0][0].view(np.int32), outs[1][0].view(np.int32))
    assert np.array_equal(outs[0][1].view(np.int32), outs[1][1].view(np.int32))


def test_merge_sort_across_sort_interval_changes(cuda):
    """Sorting every step, every other step or never, and every step again (eager
    and graph-replayed): change bits written before the unsorted steps are never
    merged, and the merges that follow still give the full sort's particles."""
    G, n = 64, 200_000
    pos, vel = _mover_scene(n, 5, 1.0)
    outs = []
    for full in (1, -1):  # the full sort, and the merge forced at these sizes
        with make_sim(cuda, n, G, gravity=200.0, softening_cells=1.0, order=L.SD_ORDER_TILED, full_sort=full) as s:
            s.set_particles(pos, vel)
            got = []
            for interval, eager in ((1, True), (2, True), (1, True), (1, False), (0, False), (1, False), (2, False),
                                    (1, True)):
                cfg = s.config()
                cfg.sort_interval = interval
                s.reconfigure(cfg)
                if eager:
                    for _ in range(3):
                        s.step(1e-3)
                else:
                    s.steps(1e-3, 4)
                got.append(s.get_particles())
            outs.append(got)
    for (p0, v0), (p1, v1) in zip(outs[0], outs[1]):
        assert np.array_equal(p0.view(np.int32), p1.view(np.int32))
        assert np.array_equal(v0.view(np.int32), v1.view(np.int32))
