"""The FP64 Ewald reference forces: oracle self-consistency (CPU) and the GPU kernel against
the oracle (GPU)."""
import numpy as np
import pytest

from conftest import random_particles


def _small(seed=0, n=300):
    rng = np.random.default_rng(seed)
    src = np.zeros((n, 4), np.float32)
    src[:, :3] = rng.random((n, 3))
    return src


def test_oracle_ewald_independent_of_split(oracle):
    src = _small()
    a1 = oracle.ewald_forces_f64(src, src[:25], 1.0 / 64, 1.0 / 16, 28)
    a2 = oracle.ewald_forces_f64(src, src[:25], 1.0 / 64, 1.0 / 12, 21)
    assert np.abs(a1 - a2).max() <= 1e-10 * np.abs(a1).max()


def test_oracle_ewald_is_the_pm_continuum_limit(oracle):
    """FP64 PM with the same Gaussian softening converges toward the Ewald forces
    as the grid is refined (the grid error shrinks)."""
    src = _small(1, 400)
    s = 1.0 / 32
    ref = oracle.ewald_forces_f64(src, src[:40], s, 1.0 / 16, 28)
    errs = []
    for G in (32, 64, 128):
        a = oracle.pm_accel_f64(src, G, 4 * np.pi * G ** 3 / len(src), s * G)[:40]
        errs.append(oracle.force_error(a, ref)["rms_rel"])
    assert errs[0] > errs[1] > errs[2]
    assert errs[2] < 0.02


@pytest.mark.gpu
def test_gpu_ewald_matches_oracle(cuda, lib, oracle):
    from stardust_b200.ewald import ewald_forces

    src, _ = random_particles(2000, 3, clustered=True)
    tgt = src[:64]
    for s, b, nm in ((1.0 / 64, 1.0 / 16, 28), (1.0 / 128, 1.0 / 12, 22)):
        got = ewald_forces(src, tgt, s, b, nm)
        ref = oracle.ewald_forces_f64(src, tgt, s, b, nm)
        assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max()


@pytest.mark.gpu
def test_gpu_ewald_two_particles_is_newtonian_at_short_range(cuda, lib):
    """Two particles a few softening lengths apart attract with ~G m / r^2 (plus
    a small periodic-image correction)."""
    from stardust_b200.ewald import ewald_forces

    src = np.array([[0.5, 0.5, 0.5, 0], [0.52, 0.5, 0.5, 0]], np.float32)
    a = ewald_forces(src, src, 1e-3)
    m, r = 0.5, 0.02
    assert a[0, 0] > 0 and a[1, 0] < 0
    assert a[0, 0] == pytest.approx(m / r ** 2, rel=2e-3)


def test_fp64_pm_reference_matches_the_oracle(oracle):
    """The FP64 particle-mesh reference the benchmark reports the force error against
    (stardust_b200.ewald.pm_accel_f64) is the oracle's FP64 PM on the same grid."""
    from stardust_b200.ewald import pm_accel_f64

    rng = np.random.default_rng(3)
    n, G = 30000, 32
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = (rng.random((8, 3))[rng.integers(0, 8, n)] + rng.normal(scale=0.05, size=(n, 3))) % 1.0
    pos[:, :3][pos[:, :3] >= 1.0] = 0.0
    pos[::17] = (-1.0, -1.0, -1.0, 0.0)  # empty slots deposit nothing
    live = np.nonzero(pos[:, 0] >= 0)[0]
    sample = live[::37]
    for soft in (0.0, 1.5):
        a = pm_accel_f64(pos, sample, G, 0.37, soft)
        b = oracle.pm_accel_f64(pos[pos[:, 0] >= 0], G, 0.37, soft)[np.searchsorted(live, sample)]
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
