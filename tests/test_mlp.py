"""The learned correction's MLP: the oracle's backward against finite
differences (CPU), and the tensor-core kernels against the oracle (GPU)."""
import ctypes

import numpy as np
import pytest

from conftest import random_particles
from stardust_b200 import _lib as L


def _params(seed=0, scale=0.3):
    rng = np.random.default_rng(seed)
    p = (rng.standard_normal(6792) * scale).astype(np.float32)
    return p


def _batch(rows, seed=1):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((rows, 32)).astype(np.float32)
    X[:, 30:] = 0
    T = rng.standard_normal((rows, 3)).astype(np.float32)
    return X, T


def test_oracle_gradient_matches_finite_differences(oracle):
    p = _params().astype(np.float64)
    X, T = _batch(48)
    _, g = oracle.mlp_loss_grad(p, X, T, round_bf16=False)
    rows = len(X)
    rng = np.random.default_rng(3)
    for idx in list(rng.choice(6792, 40, replace=False)) + [2048, 6784, 6785]:
        if idx in range(6787, 6792) or (6272 <= idx < 6784 and (idx - 6272) % 8 >= 3):
            continue  # padded outputs: no gradient
        h = 1e-4
        pp, pm = p.copy(), p.copy()
        pp[idx] += h
        pm[idx] -= h
        lp = oracle.mlp_loss_grad(pp, X, T, round_bf16=False)[0] / (3 * rows)
        lm = oracle.mlp_loss_grad(pm, X, T, round_bf16=False)[0] / (3 * rows)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-5 * max(1.0, abs(fd)), (idx, fd, g[idx])


@pytest.mark.gpu
def test_gpu_features_match_oracle(cuda, lib, oracle):
    G, n = 32, 5000
    pos, _ = random_particles(n, 2, empty_every=97, clustered=True)
    rho = oracle.density_fixed(pos, G)
    inv_mean = G ** 3 / n
    out = cuda.empty((n, 32), dtype=cuda.bfloat16, device="cuda")
    pd, rd = cuda.from_numpy(pos).cuda(), cuda.from_numpy(rho).cuda()
    L.check(lib.sd_mlp_features(pd.data_ptr(), None, n, rd.data_ptr(), G, ctypes.c_float(inv_mean), out.data_ptr(),
                                None), "features")
    got = out.float().cpu().numpy()
    ref = oracle.bf16(oracle.mlp_features(pos, rho, G, inv_mean))
    # log1p in float32 on the GPU vs float64 here: at most one bf16 step apart
    assert np.abs(got - ref).max() <= 2 ** -7 * max(1.0, np.abs(ref).max())


@pytest.mark.gpu
@pytest.mark.parametrize("G,n", [(32, 3001), (64, 300_001)])
def test_gpu_infer_matches_oracle(cuda, lib, oracle, G, n):
    # 300,001 particles: 2,344 tiles of 128, more than one per CTA of the tensor-core kernel
    pos, _ = random_particles(n, 5, clustered=True)
    rho = oracle.density_fixed(pos, G)
    inv_mean = G ** 3 / n
    params = _params(7, 0.2)
    out = cuda.empty((n, 4), dtype=cuda.float32, device="cuda")
    prm, pd, rd = (cuda.from_numpy(a).cuda() for a in (params, pos, rho))
    L.check(lib.sd_mlp_infer(prm.data_ptr(), pd.data_ptr(), None, n, rd.data_ptr(), G, ctypes.c_float(inv_mean),
                             ctypes.c_float(2.0), out.data_ptr(), None), "infer")
    got = out.cpu().numpy()
    X = oracle.mlp_features(pos, rho, G, inv_mean)
    ref, _ = oracle.mlp_forward(params, X)
    ref *= 2.0
    err = np.abs(got[:, :3] - ref).max() / np.abs(ref).max()
    assert err < 2e-2, err
    assert np.all(got[:, 3] == 0)
    assert lib.sd_mlp_wait_timeouts() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("rows", [256, 16384])
def test_gpu_loss_grad_matches_oracle(cuda, lib, oracle, rows):
    params = _params(11, 0.2)
    X, T = _batch(rows, 4)
    Xb = cuda.from_numpy(X).cuda().to(cuda.bfloat16)
    Td, prm = cuda.from_numpy(T).cuda(), cuda.from_numpy(params).cuda()
    grad = cuda.empty(6792, dtype=cuda.float32, device="cuda")
    sse = cuda.empty(1, dtype=cuda.float32, device="cuda")
    ws = cuda.empty(int(lib.sd_mlp_train_workspace_bytes(rows)), dtype=cuda.uint8, device="cuda")
    L.check(lib.sd_mlp_loss_grad(prm.data_ptr(), Xb.data_ptr(), Td.data_ptr(), rows, grad.data_ptr(), sse.data_ptr(),
                                 ws.data_ptr(), ws.numel(), None), "loss_grad")
    g = grad.cpu().numpy()
    sse_ref, g_ref = oracle.mlp_loss_grad(params, X, T)
    assert float(sse.cpu()) == pytest.approx(sse_ref, rel=1e-3)
    for name, (o, sh) in oracle.MLP_OFF.items():
        a, b = g[o:o + int(np.prod(sh))], g_ref[o:o + int(np.prod(sh))]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert rel < 3e-2, (name, rel)


@pytest.mark.gpu
def test_gpu_adam_step(cuda, lib):
    n = 6792
    rng = np.random.default_rng(0)
    p0 = rng.standard_normal(n).astype(np.float32)
    g = rng.standard_normal(n).astype(np.float32)
    p, m, v, gd = (cuda.from_numpy(a.copy()).cuda() for a in (p0, np.zeros(n, np.float32), np.zeros(n, np.float32), g))
    L.check(lib.sd_mlp_adam(p.data_ptr(), m.data_ptr(), v.data_ptr(), gd.data_ptr(), 1, ctypes.c_float(1e-3),
                            ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8), None), "adam")
    # first Adam step moves each parameter by lr * sign(g)
    assert np.allclose(p.cpu().numpy(), p0 - 1e-3 * np.sign(g), atol=1e-6)
