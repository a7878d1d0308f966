"""CPU checks of the oracle: against FP64 numpy, against its own invariants, and
against fixtures produced by the reference itself (tests/golden)."""
import glob
import os

import numpy as np
import pytest

from conftest import random_particles

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("G", [16, 32, 64])
def test_fixed_deposit_matches_fp64(oracle, G):
    pos, _ = random_particles(4000, G, empty_every=37)
    rho = oracle.density_fixed(pos, G)
    ref = oracle.density_f64(pos, G)
    assert np.abs(rho - ref).max() < 4e-7 * max(1.0, ref.max())
    assert rho.sum(dtype=np.float64) == pytest.approx((pos[:, 0] >= 0).sum(), rel=1e-6)


def test_fixed_deposit_is_order_independent(oracle):
    pos, _ = random_particles(20000, 3, clustered=True)
    a = oracle.deposit_fixed(pos, 32)
    b = oracle.deposit_fixed(pos[np.random.default_rng(1).permutation(len(pos))], 32)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("G,soft", [(16, 0.0), (32, 1.5), (64, 3.0)])
def test_poisson_matches_fp64(oracle, G, soft):
    pos, _ = random_particles(6000, G + 1)
    rho = oracle.density_fixed(pos, G)
    phi = oracle.poisson_periodic(rho, soft)
    ref = oracle.poisson_periodic_f64(rho.astype(np.float64), soft)
    assert np.abs(phi - ref).max() <= 2e-6 * np.abs(ref).max()


def test_poisson_point_mass_symmetry(oracle):
    G = 32
    rho = np.zeros((G, G, G), np.float32)
    rho[5, 9, 13] = 1.0
    phi = oracle.poisson_periodic(rho, 0.0)
    # symmetric about the source along each axis, minimum at the source
    assert np.argmin(phi) == np.ravel_multi_index((5, 9, 13), rho.shape)
    assert abs(phi[5, 9, 14] - phi[5, 9, 12]) < 1e-6 * abs(phi).max()
    assert abs(phi.mean()) < 1e-6 * abs(phi).max()  # k = 0 removed


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_stable_sort_matches_numpy(oracle, mode):
    pos, _ = random_particles(30001, 5, empty_every=11, clustered=True)
    G = 64
    keys = oracle.cell_keys(pos, G, mode)
    perm = oracle.stable_sort_perm(keys, oracle.key_bits(G, mode))
    assert np.array_equal(perm, np.argsort(keys, kind="stable"))
    assert (keys[perm[: (keys == -1).sum()]] == -1).all()  # empty slots first


def test_rowmajor_key_is_reference_formula(oracle):
    G = 64
    pos = np.array([[0.0, 0.0, 0.0, 0], [0.999999, 0.5, 0.25, 0], [1.0, 1.0, 1.0, 0], [-1, -1, -1, 0],
                    [0.015625, 0.03125, 0.046875, 0]], np.float32)
    keys = oracle.cell_keys(pos, G, 0)
    # kCellKey: c = clamp((int)(p*G), 0, G-1), key = (cz*G + cy)*G + cx, empty -> -1
    assert keys.tolist() == [0, (16 * G + 32) * G + 63, (63 * G + 63) * G + 63, -1, (3 * G + 2) * G + 1]


def test_integrate_conserves_momentum_zero(oracle):
    pos, vel = random_particles(5000, 9, empty_every=13)
    vel2, sums = oracle.momentum_zero(pos, vel)
    live = pos[:, 0] >= 0
    assert np.abs(vel2[live, :3].astype(np.float64).mean(axis=0)).max() < 1e-6
    assert sums[3] == live.sum()


def test_step_mass_and_momentum(oracle):
    pos, vel = random_particles(8000, 12, clustered=True)
    p2, v2, rho, mom = oracle.step(pos, vel, 32, gravity=1.0, soft_cells=1.0, dt_kick=1e-3, dt_drift=1e-3)
    assert rho.sum(dtype=np.float64) == pytest.approx(8000, rel=1e-6)
    assert ((p2[:, :3] >= 0) & (p2[:, :3] < 1)).all()
    assert np.abs(v2[:, :3].astype(np.float64).mean(axis=0)).max() < 1e-6
    # ids survive the sort
    assert sorted(v2[:, 3].astype(np.int64).tolist()) == list(range(8000))


def test_pm_accel_f64_two_particles_antisymmetric(oracle):
    G = 32
    pos = np.array([[0.3, 0.5, 0.5, 0], [0.6, 0.5, 0.5, 0]], np.float32)
    a = oracle.pm_accel_f64(pos, G, 1.0 / 2, 0.0)
    assert a[0, 0] > 0 and a[1, 0] < 0  # attraction
    assert abs(a[0, 0] + a[1, 0]) < 1e-9 * abs(a[0, 0]) + 1e-12


def _golden_files(isolated=False):
    """One-step plain-PM fixtures holding their inputs (not the preset, hydro,
    field or compact fixtures)."""
    files = sorted(glob.glob(os.path.join(GOLDEN, "reference_*.npz")))
    files = [f for f in files if not os.path.basename(f).startswith(
        ("reference_preset_", "reference_hydro_", "reference_fields_")) and "pos_in" in np.load(f).files]
    return [f for f in files if ("isolated" in os.path.basename(f)) == isolated]


def _compact_files():
    """One-step fixtures stored without their inputs (rebuilt from the seeded scene)."""
    return [f for f in sorted(glob.glob(os.path.join(GOLDEN, "reference_*.npz"))) if "digest" in np.load(f).files]


@pytest.mark.skipif(not _compact_files(), reason="no compact reference fixture committed")
@pytest.mark.parametrize("path", _compact_files(), ids=lambda p: os.path.basename(p)[10:-4])
def test_oracle_against_reference_at_benchmark_scale(oracle, path):
    """One step of the unmodified reference at the first benchmark configuration's
    scale (262,144 disk-galaxy particles on 64^3): the seeded inputs are rebuilt
    and checked against the fixture's digest, then the oracle's step must give the
    reference's sort permutation exactly, its loaded density within float-atomic
    rounding, and on a sample of output slots its velocity change and positions."""
    import hashlib

    from stardust_b200 import scenes

    f = np.load(path)
    kind, n, seed = str(f["scene"][0]), int(f["n"]), int(f["seed"])
    pos, vel = scenes.disk_galaxy(n, seed) if kind == "disk" else scenes.two_galaxies(n, seed)
    pos = np.ascontiguousarray(pos, np.float32)
    vel = np.ascontiguousarray(vel, np.float32)
    vel[:, 3] = np.arange(n, dtype=np.float32)
    assert hashlib.sha256(pos.tobytes() + vel.tobytes()).hexdigest() == str(f["digest"][0]), "scene inputs drifted"
    G = int(f["grid"])
    rho = oracle.density_fixed(pos, G)
    assert np.abs(rho - f["rho_loaded"]).max() <= 2e-5 * max(1.0, float(f["rho_loaded"].max()))
    p1, v1, _, _ = oracle.step(pos, vel, G, gravity=float(f["gravity"]), soft_cells=float(f["soft"]),
                               dt_kick=float(f["dt"]), dt_drift=float(f["dt"]))
    assert np.array_equal(v1[:, 3].astype(np.int64), f["ids_out"].astype(np.int64))
    slots = f["slots"]
    ids = f["ids_out"][slots].astype(np.int64)
    dv_ref = f["vel_out"][:, :3] - vel[ids, :3]
    dv = v1[slots, :3] - vel[ids, :3]
    scale = np.sqrt(np.mean(np.sum(dv_ref.astype(np.float64) ** 2, axis=1)))
    err = np.sqrt(np.mean(np.sum((dv - dv_ref).astype(np.float64) ** 2, axis=1))) / scale
    assert err < 2e-4, err
    dp = (p1[slots, :3] - f["pos_out"][:, :3] + 0.5) % 1.0 - 0.5
    assert np.abs(dp).max() < 1e-5


FIELDS = os.path.join(GOLDEN, "reference_fields_g32.npz")


@pytest.mark.skipif(not os.path.exists(FIELDS), reason="no field fixture committed")
@pytest.mark.parametrize("view", ["top", "rot"])
def test_render_fields_oracle_against_reference(oracle, view):
    """The screen grids the headless grid view shades, against the unmodified
    reference's Sim::fieldDevicePtr (kProjectXY; kScatterDispersion and
    kDivideInto) on the same loaded scene, straight down and through a view
    rotation: the density projection of the reference's own loaded density, and
    the velocity dispersion of the particles. The reference sums with float
    atomics in no fixed order, hence the tolerances."""
    f = np.load(FIELDS)
    G = int(f["grid"])
    v = {"rot_on": 0} if view == "top" else {"rot_on": 1, "rot": f["rot"], "center": (0.5, 0.5, 0.5)}
    dens = oracle.project_field(f["rho_loaded"], v)
    ref = f[f"density_{view}"].astype(np.float64)
    assert np.abs(dens - ref).max() <= 1e-5 * ref.max()
    disp = oracle.dispersion_field(f["pos"], f["vel"], G, v)
    ref = f[f"dispersion_{view}"].astype(np.float64)
    assert np.abs(disp - ref).max() <= 1e-4 * ref.max()


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "reference_preset_*.npz"))),
                         ids=lambda p: os.path.basename(p)[17:-4])
def test_preset_oracle_against_reference_fixtures(oracle, path):
    """place_preset reproduces the particles the unmodified reference's Sim::init
    lays down (kPlace, spin, Hubble flow, dispersion, centre-of-mass stop): the
    same hashes pick the same slots and dark-matter marks; positions differ only
    by libm sin/cos against the reference's fast intrinsics (arguments up to ~50)."""
    f = np.load(path)
    po, vo = oracle.place_preset(int(f["n"]), int(f["preset"]), float(f["dark_matter_fraction"]),
                                 float(f["big_bang_shrink"]), float(f["spin"]), float(f["hubble"]),
                                 float(f["vel_dispersion"]))
    live = f["pos"][:, 0] >= 0
    assert np.array_equal(po[:, 0] >= 0, live)
    assert np.array_equal(vo[:, 3], f["vel"][:, 3])
    assert np.abs(po[live, :3] - f["pos"][live, :3]).max() < 4e-6
    assert np.abs(vo[:, :3] - f["vel"][:, :3]).max() < 4e-6


@pytest.mark.skipif(not _golden_files(), reason="no reference fixtures committed")
@pytest.mark.parametrize("path", _golden_files())
def test_oracle_against_reference_fixtures(oracle, path):
    """The oracle reproduces outputs of the unmodified reference (src/sim/Sim.cu,
    run on a B200 through oracle/ref) on the same inputs."""
    f = np.load(path)
    G = int(f["grid"])
    pos0, vel0 = f["pos_in"], f["vel_in"]
    # density after loadState = deposit of the loaded positions (float atomics there)
    rho_ref = f["rho_loaded"]
    rho = oracle.density_fixed(pos0, G)
    assert np.abs(rho - rho_ref).max() <= 2e-5 * max(1.0, float(rho_ref.max()))
    # one step: sort permutation is exact; positions / velocities within FP32 tolerance
    p1, v1, rho1, _ = oracle.step(pos0, vel0, G, gravity=float(f["gravity"]), soft_cells=float(f["soft"]),
                                  dt_kick=float(f["dt"]), dt_drift=float(f["dt"]))
    ids_ref = f["vel_out"][:, 3].astype(np.int64)
    ids = v1[:, 3].astype(np.int64)
    assert np.array_equal(ids, ids_ref)
    dv_ref = f["vel_out"][:, :3] - vel0[ids_ref, :3]
    dv = v1[:, :3] - vel0[ids, :3]
    scale = np.sqrt(np.mean(np.sum(dv_ref.astype(np.float64) ** 2, axis=1)))
    err = np.sqrt(np.mean(np.sum((dv - dv_ref).astype(np.float64) ** 2, axis=1))) / scale
    assert err < 2e-4, err
    dp = (p1[:, :3] - f["pos_out"][:, :3] + 0.5) % 1.0 - 0.5
    assert np.abs(dp).max() < 1e-5


def test_isolated_oracle_two_particles_attract_newtonianly(oracle):
    """The FP64 isolated solve: two particles far from the walls and from each
    other's padding copies attract with ~1/(r + soft)^2 in cell units."""
    G = 32
    pos = np.array([[0.40, 0.5, 0.5, 0], [0.60, 0.5, 0.5, 0]], np.float32)
    a = oracle.pm_accel_iso_f64(pos, G, 1.0, 1.0)
    r_cells = 0.2 * G
    assert a[0, 0] > 0 and a[1, 0] < 0
    assert abs(a[0, 0] + a[1, 0]) < 1e-9 * abs(a[0, 0])  # equal and opposite
    # gravity 1, unit masses in count units: F ~ d/dr [1/(r + soft)] in cells, times 1/2 G per cell of gradient
    assert a[0, 0] == pytest.approx(1.0 / (r_cells + 1.0) ** 2 * G, rel=0.15)
    # no periodic images: the force on a particle near a wall points only to its partner
    pos2 = np.array([[0.05, 0.5, 0.5, 0], [0.25, 0.5, 0.5, 0]], np.float32)
    b = oracle.pm_accel_iso_f64(pos2, G, 1.0, 1.0)
    assert b[0, 0] > 0 and b[0, 0] == pytest.approx(a[0, 0], rel=0.05)


@pytest.mark.skipif(not _golden_files(True), reason="no isolated reference fixture committed")
@pytest.mark.parametrize("path", _golden_files(True))
def test_isolated_oracle_against_reference_fixture(oracle, path):
    """The FP64 isolated oracle (clamped deposit, 2G-box Green's function,
    clamped gradient and gather, the wall, momentum zeroing) reproduces one step
    of the unmodified reference in its default isolated mode."""
    f = np.load(path)
    G, grav, soft, dt = int(f["grid"]), float(f["gravity"]), float(f["soft"]), float(f["dt"])
    pos0, vel0 = f["pos_in"], f["vel_in"]
    n = len(pos0)
    rho = oracle.density_iso_f64(pos0, G)
    assert np.abs(rho - f["rho_loaded"]).max() <= 2e-5 * float(rho.max())
    a = oracle.pm_accel_iso_f64(pos0, G, grav / n, soft)
    vk = (vel0[:, :3] + a * dt).astype(np.float32)
    pk = (pos0[:, :3] + vk.astype(np.float64) * dt).astype(np.float32)
    pw, vw = oracle.isolated_wall(pk, vk)
    vw = vw - vw.mean(axis=0, dtype=np.float64).astype(np.float32)
    ids = f["vel_out"][:, 3].astype(np.int64)
    p_ref, v_ref = f["pos_out"][:, :3], f["vel_out"][:, :3]
    dv_ref = v_ref - vel0[ids, :3]
    dv = vw[ids] - vel0[ids, :3]
    scale = np.sqrt(np.mean(np.sum(dv_ref.astype(np.float64) ** 2, axis=1)))
    err = np.sqrt(np.mean(np.sum((dv - dv_ref).astype(np.float64) ** 2, axis=1))) / scale
    assert err < 2e-4, err
    assert np.abs(pw[ids] - p_ref).max() < 1e-5
    assert p_ref.min() >= 0.002 and p_ref.max() <= 0.998
