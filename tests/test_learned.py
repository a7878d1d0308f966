"""The learned sub-grid correction inside the step: the correction off or zero is
the plain PM step, the in-step inference matches the oracle MLP, eager and
graph-replayed steps agree, and a trained network lowers the FP64-measured force
error of the coarse grid on a scene it was not trained on."""
import numpy as np
import pytest

from stardust_b200 import _lib as L


def _scene(n_side, seed):
    from stardust_b200.scenes import zeldovich

    return zeldovich(n_side, seed)


@pytest.mark.gpu
def test_zero_correction_is_the_plain_step(cuda):
    from stardust_b200.learned import Correction, pm_config
    from stardust_b200.sim import Sim

    pos, vel = _scene(24, 5)
    n = len(pos)
    out = []
    for corr in (None, Correction(np.zeros(6792, np.float32), 3.0, 1 / 32, 32, 128)):
        with Sim(0) as s:
            s.init(pm_config(n, 32, 1 / 32))
            s.set_particles(pos, vel)
            if corr is not None:
                s.set_correction(corr)
            s.steps(1e-3, 4)
            out.append(s.get_particles())
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


@pytest.mark.gpu
def test_in_step_correction_matches_oracle_mlp(cuda, oracle):
    from stardust_b200.learned import Correction, PMField

    pos, _ = _scene(24, 6)
    n, G = len(pos), 32
    rng = np.random.default_rng(2)
    params = (rng.standard_normal(6792) * 0.2).astype(np.float32)
    corr = Correction(params, 0.5, 1 / 32, G, 128)
    pd = cuda.from_numpy(pos).cuda()
    f = PMField(pd, G, 1 / 32)
    plain = f.accel().cpu().numpy()
    rho = f.density().cpu().numpy()
    f.set_correction(corr)
    with_mlp = f.accel().cpu().numpy()
    f.close()
    y, _ = oracle.mlp_forward(params, oracle.mlp_features(pos, rho, G, G ** 3 / n))
    got = with_mlp[:, :3] - plain[:, :3]
    ref = 0.5 * y
    assert np.abs(got - ref).max() <= 2e-2 * np.abs(ref).max()


@pytest.mark.gpu
def test_graph_replay_with_correction_matches_eager_steps(cuda):
    from stardust_b200.learned import Correction, init_params, pm_config
    from stardust_b200.sim import Sim

    pos, vel = _scene(24, 7)
    n = len(pos)
    corr = Correction(init_params(3) * 3, 2.0, 1 / 32, 32, 128)
    res = []
    for graph in (False, True):
        with Sim(0) as s:
            s.init(pm_config(n, 32, 1 / 32))
            s.set_particles(pos, vel)
            s.set_correction(corr)
            if graph:
                s.steps(1e-3, 4)
            else:
                for _ in range(4):
                    s.step(1e-3)
            res.append(s.get_particles())
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])


@pytest.mark.gpu
def test_trained_correction_lowers_fp64_force_error(cuda):
    """32^3-particle scenes, 32^3 coarse grid, 128^3 fine grid, one softening
    (1/32 box) for both: train on 4 seeds, measure a held-out seed against the
    FP64 Ewald forces of the same smoothed-mass model."""
    from stardust_b200.ewald import ewald_forces, force_error
    from stardust_b200.learned import Correction, PMField, train, training_pairs

    soft = 1.0 / 32
    X, T = training_pairs(range(20, 24), n_side=32, coarse=32, fine=128, softening=soft)
    params, scale, hist = train(X, T, epochs=40, batch=4096, lr=3e-3)
    assert hist[-1] < 0.9 * hist[0]
    corr = Correction(params, scale, soft, 32, 128)
    pos, _ = _scene(32, 99)
    pd = cuda.from_numpy(pos).cuda()
    tgt = np.random.default_rng(0).choice(len(pos), 4096, replace=False)
    ref = ewald_forces(pd, pd[cuda.from_numpy(tgt).cuda()].contiguous(), soft)
    f = PMField(pd, 32, soft)
    e_plain = force_error(f.accel().cpu().numpy()[tgt], ref)["rms_rel"]
    f.set_correction(corr)
    e_mlp = force_error(f.accel().cpu().numpy()[tgt], ref)["rms_rel"]
    f.close()
    print(f"coarse {e_plain:.4f} -> coarse+MLP {e_mlp:.4f}")
    assert e_mlp < 0.85 * e_plain
