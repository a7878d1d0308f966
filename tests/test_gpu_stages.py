"""Stage-by-stage parity of the CUDA kernels against the oracle, through the C ABI.

Bit-exact: cell keys, sort permutation, fixed-point density, gather/kick/drift
given the same potential. Tolerance: the FFT Poisson solve (FP32, checked
against FP64 numpy at a relative max error of 2e-5 of the field's range).
"""
import ctypes

import numpy as np
import pytest

from conftest import random_particles
from stardust_b200 import _lib as L

pytestmark = pytest.mark.gpu

POISSON_RTOL = 2e-5


def dev(torch, a):
    """Upload to the GPU. Callers keep the returned tensor alive while a kernel
    uses its pointer (a dropped temporary goes back to torch's allocator)."""
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def ws(torch, nbytes):
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device="cuda")


def sync(torch):
    torch.cuda.synchronize()


def edge_positions():
    G = 64
    e = np.float32(np.nextafter(np.float32(1.0), np.float32(0.0)))
    rows = [[0, 0, 0], [e, e, e], [0.5 / G, 0.5 / G, 0.5 / G], [1.0 / G, 2.0 / G, 3.0 / G], [0.999, 0.001, 0.5],
            [1e-9, 1e-9, 1e-9], [0.5, 0.5, 0.5]]
    p = np.zeros((len(rows), 4), np.float32)
    p[:, :3] = rows
    return p


@pytest.mark.parametrize("order", [0, 1, 2])
@pytest.mark.parametrize("G", [16, 64, 512])
def test_cell_keys_bit_exact(cuda, lib, oracle, order, G):
    pos, _ = random_particles(100_003, G + order, empty_every=17, clustered=True)
    pos = np.concatenate([pos, edge_positions()])
    keys = cuda.empty(len(pos), dtype=cuda.int32, device="cuda")
    pd = dev(cuda, pos)
    L.check(lib.sd_cell_keys(pd.data_ptr(), len(pos), G, order, keys.data_ptr(), None), "keys")
    sync(cuda)
    ref = oracle.cell_keys(pos, G, order).astype(np.int64)
    ref = np.maximum(ref, 0) if order == 2 else ref + 1  # tiled: row index, empty slots share row 0
    assert np.array_equal(keys.cpu().numpy().view(np.uint32).astype(np.int64), ref)


@pytest.mark.parametrize("n", [0, 1, 2047, 2048, 2049, 100_000, 1_000_003])
def test_sort_permutation_bit_exact(cuda, lib, oracle, n):
    rng = np.random.default_rng(n)
    bits = 19
    keys = rng.integers(0, 1 << bits, n, dtype=np.int64).astype(np.uint32)
    if n > 10:
        keys[: n // 3] = keys[0]  # many duplicates: stability matters
        keys[n // 2:] = np.sort(keys[n // 2:])  # a presorted run
    kin = dev(cuda, keys.view(np.int32))
    kout, ktmp = cuda.empty_like(kin), cuda.empty_like(kin)
    vout = cuda.empty(max(n, 1), dtype=cuda.int32, device="cuda")
    vtmp = cuda.empty_like(vout)
    w = ws(cuda, lib.sd_sort_workspace_bytes(n))
    L.check(lib.sd_sort_pairs(kin.data_ptr(), None, kout.data_ptr(), vout.data_ptr(), ktmp.data_ptr(),
                              vtmp.data_ptr(), n, bits, w.data_ptr(), w.numel(), None), "sort")
    sync(cuda)
    perm = vout.cpu().numpy()[:n]
    assert np.array_equal(perm, np.argsort(keys, kind="stable"))
    assert np.array_equal(kout.cpu().numpy()[:n].view(np.uint32), np.sort(keys, kind="stable"))


def test_sort_with_a_dirty_workspace(cuda, lib):
    """A workspace handed to sd_sort_pairs may hold anything: the sort clears the
    sums it accumulates into before using them."""
    rng = np.random.default_rng(5)
    n, bits = 300_007, 18
    keys = rng.integers(0, 1 << bits, n, dtype=np.int64).astype(np.uint32)
    kin = dev(cuda, keys.view(np.int32))
    kout, ktmp = cuda.empty_like(kin), cuda.empty_like(kin)
    vout, vtmp = cuda.empty_like(kin), cuda.empty_like(kin)
    w = ws(cuda, lib.sd_sort_workspace_bytes(n))
    w.fill_(0xAB)
    for _ in range(2):  # garbage, then the state a sort leaves
        L.check(lib.sd_sort_pairs(kin.data_ptr(), None, kout.data_ptr(), vout.data_ptr(), ktmp.data_ptr(),
                                  vtmp.data_ptr(), n, bits, w.data_ptr(), w.numel(), None), "sort")
        sync(cuda)
        assert np.array_equal(vout.cpu().numpy(), np.argsort(keys, kind="stable"))


def test_sort_full_32_bits_and_values(cuda, lib):
    rng = np.random.default_rng(7)
    n = 300_001
    keys = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    vals = rng.integers(-1000, 1000, n).astype(np.int32)
    kin, vin = dev(cuda, keys.view(np.int32)), dev(cuda, vals)
    kout, ktmp, vout, vtmp = (cuda.empty_like(kin), cuda.empty_like(kin), cuda.empty_like(vin),
                              cuda.empty_like(vin))
    w = ws(cuda, lib.sd_sort_workspace_bytes(n))
    L.check(lib.sd_sort_pairs(kin.data_ptr(), vin.data_ptr(), kout.data_ptr(), vout.data_ptr(), ktmp.data_ptr(),
                              vtmp.data_ptr(), n, 32, w.data_ptr(), w.numel(), None), "sort")
    sync(cuda)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(vout.cpu().numpy(), vals[order])


@pytest.mark.parametrize("order", [0, 1, 2])
def test_sort_cell_keys_matches_oracle_and_reorder(cuda, lib, oracle, order):
    G = 64
    pos, vel = random_particles(200_000, 11 + order, empty_every=29, clustered=True)
    n = len(pos)
    pd, vd = dev(cuda, pos), dev(cuda, vel)
    keys = cuda.empty(n, dtype=cuda.int32, device="cuda")
    L.check(lib.sd_cell_keys(pd.data_ptr(), n, G, order, keys.data_ptr(), None), "keys")
    kout, ktmp = cuda.empty_like(keys), cuda.empty_like(keys)
    vout, vtmp = cuda.empty_like(keys), cuda.empty_like(keys)
    bits = lib.sd_key_bits(G, order)
    w = ws(cuda, lib.sd_sort_workspace_bytes(n))
    L.check(lib.sd_sort_pairs(keys.data_ptr(), None, kout.data_ptr(), vout.data_ptr(), ktmp.data_ptr(),
                              vtmp.data_ptr(), n, bits, w.data_ptr(), w.numel(), None), "sort")
    p2, v2 = cuda.empty_like(pd), cuda.empty_like(vd)
    L.check(lib.sd_reorder(pd.data_ptr(), vd.data_ptr(), vout.data_ptr(), p2.data_ptr(), v2.data_ptr(), n, None),
            "reorder")
    sync(cuda)
    okeys = oracle.cell_keys(pos, G, order)
    if order == 2:  # tiled keys are row indices with empty slots in row 0
        ref_perm = np.argsort(np.maximum(okeys, 0), kind="stable").astype(np.int32)
    else:
        ref_perm = oracle.stable_sort_perm(okeys, bits)
    assert np.array_equal(vout.cpu().numpy(), ref_perm)
    assert np.array_equal(p2.cpu().numpy(), pos[ref_perm])
    assert np.array_equal(v2.cpu().numpy(), vel[ref_perm])


@pytest.mark.parametrize("G,n,clustered", [(16, 5000, False), (64, 262_144, True), (128, 500_000, False),
                                            (256, 300_000, True)])
def test_deposit_bit_exact(cuda, lib, oracle, G, n, clustered):
    pos, _ = random_particles(n, G, empty_every=23, clustered=clustered)
    pos = np.concatenate([pos, edge_positions()])
    rho = cuda.empty(G ** 3, dtype=cuda.float32, device="cuda")
    w = ws(cuda, lib.sd_deposit_workspace_bytes(G))
    pd = dev(cuda, pos)
    L.check(lib.sd_deposit(pd.data_ptr(), len(pos), G, rho.data_ptr(), w.data_ptr(), w.numel(), None), "deposit")
    sync(cuda)
    got = rho.cpu().numpy().reshape(G, G, G)
    ref = oracle.density_fixed(pos, G)
    assert np.array_equal(got.view(np.int32), ref.view(np.int32))
    assert got.sum(dtype=np.float64) == pytest.approx((pos[:, 0] >= 0).sum(), rel=1e-6)


def test_deposit_deterministic_across_runs_and_orders(cuda, lib):
    G = 64
    pos, _ = random_particles(400_000, 5, clustered=True)
    perm = np.random.default_rng(2).permutation(len(pos))
    outs = []
    for p in (pos, pos, pos[perm]):
        rho = cuda.empty(G ** 3, dtype=cuda.float32, device="cuda")
        w = ws(cuda, lib.sd_deposit_workspace_bytes(G))
        pd = dev(cuda, p)
        L.check(lib.sd_deposit(pd.data_ptr(), len(p), G, rho.data_ptr(), w.data_ptr(), w.numel(), None), "deposit")
        outs.append(rho.cpu().numpy())
    assert np.array_equal(outs[0].view(np.int32), outs[1].view(np.int32))
    assert np.array_equal(outs[0].view(np.int32), outs[2].view(np.int32))


def gpu_poisson(cuda, lib, rho, soft):
    G = rho.shape[0]
    phi = cuda.empty(G ** 3, dtype=cuda.float32, device="cuda")
    w = ws(cuda, lib.sd_poisson_workspace_bytes(G))
    rd = dev(cuda, rho)
    L.check(lib.sd_poisson(rd.data_ptr(), G, ctypes.c_float(soft), phi.data_ptr(), w.data_ptr(), w.numel(), None),
            "poisson")
    sync(cuda)
    return phi.cpu().numpy().reshape(G, G, G)


@pytest.mark.parametrize("G,soft", [(16, 0.0), (32, 1.0), (64, 3.0), (128, 0.0), (256, 2.0), (512, 1.0)])
def test_poisson_against_fp64(cuda, lib, oracle, G, soft):
    rng = np.random.default_rng(G)
    if G <= 128:
        pos, _ = random_particles(min(8 * G ** 3 // 8, 400_000), G, clustered=True)
        rho = oracle.density_fixed(pos, G)
    else:  # smooth random field plus point sources, cheaper than a deposit at 512^3
        rho = rng.random((G, G, G), dtype=np.float32)
        rho[rng.integers(0, G, 50), rng.integers(0, G, 50), rng.integers(0, G, 50)] += 100.0
    phi = gpu_poisson(cuda, lib, rho, soft)
    ref = oracle.poisson_periodic_f64(rho.astype(np.float64), soft)
    rng_ref = ref.max() - ref.min()
    assert np.abs(phi - ref).max() <= POISSON_RTOL * rng_ref


def test_poisson_single_mode_exact_green(cuda, lib, oracle):
    """A single Fourier mode must come back scaled by the Green's function."""
    G = 64
    z, y, x = np.meshgrid(*(3 * [np.arange(G)]), indexing="ij")
    k = (3, 5, 7)
    rho = np.cos(2 * np.pi * (k[0] * x + k[1] * y + k[2] * z) / G).astype(np.float32)
    phi = gpu_poisson(cuda, lib, rho, 0.0)
    expect = -rho / (4 * np.pi ** 2 * (k[0] ** 2 + k[1] ** 2 + k[2] ** 2))
    assert np.abs(phi - expect).max() < 1e-5 * np.abs(expect).max()


@pytest.mark.parametrize("G,n", [(32, 20_000), (64, 262_144), (256, 200_000)])
def test_gather_kick_drift_bit_exact(cuda, lib, oracle, G, n):
    """Given the same potential, the fused gradient+gather+kick+drift equals the
    reference's kGridAccel -> sampleAcc -> kIntegrate sequence bit for bit."""
    pos, vel = random_particles(n, G + 3, empty_every=31, clustered=True)
    pos = np.concatenate([pos, edge_positions()])
    vel = np.concatenate([vel, np.zeros((len(edge_positions()), 4), np.float32)])
    n = len(pos)
    rho = oracle.density_fixed(pos, G)
    phi = gpu_poisson(cuda, lib, rho, 1.0)
    pot_scale = np.float32(4 * np.pi * G ** 3 / n)  # Newton-scale forces, exercises the clamp rarely
    dt = np.float32(1e-3)
    pd, vd = dev(cuda, pos), dev(cuda, vel)
    mom = cuda.zeros(4, dtype=cuda.float64, device="cuda")
    w = ws(cuda, lib.sd_gather_workspace_bytes(n))
    phid = dev(cuda, phi)
    L.check(lib.sd_gather_kick_drift(phid.data_ptr(), G, ctypes.c_float(pot_scale), pd.data_ptr(),
                                     vd.data_ptr(), n, ctypes.c_float(dt), ctypes.c_float(dt),
                                     ctypes.c_float(1e4), None, mom.data_ptr(), w.data_ptr(), w.numel(), None),
            "gather")
    sync(cuda)
    acc = oracle.grid_accel(phi, float(pot_scale))
    p_ref, v_ref = oracle.integrate(acc, pos, vel, float(dt), float(dt), 1e4)
    assert np.array_equal(pd.cpu().numpy().view(np.int32), p_ref.view(np.int32))
    assert np.array_equal(vd.cpu().numpy().view(np.int32), v_ref.view(np.int32))
    live = p_ref[:, 0] >= 0
    m = mom.cpu().numpy()
    assert m[3] == live.sum()
    assert m[:3] == pytest.approx(v_ref[live, :3].astype(np.float64).sum(axis=0), rel=1e-9, abs=1e-9)


def test_gather_light_speed_clamp_and_nan(cuda, lib, oracle):
    G = 32
    pos, vel = random_particles(1000, 4)
    vel[0, :3] = (300.0, 0.0, 0.0)      # above c = 100: clamped
    vel[1, :3] = (np.nan, 0.0, 0.0)     # NaN -> empty slot
    vel[2, :3] = (np.inf, 0.0, 0.0)
    phi = np.zeros((G, G, G), np.float32)
    pd, vd, phid = dev(cuda, pos), dev(cuda, vel), dev(cuda, phi)
    L.check(lib.sd_gather_kick_drift(phid.data_ptr(), G, ctypes.c_float(1.0), pd.data_ptr(),
                                     vd.data_ptr(), len(pos), ctypes.c_float(1e-3), ctypes.c_float(1e-3),
                                     ctypes.c_float(1e4), None, None, None, 0, None), "gather")
    sync(cuda)
    p, v = pd.cpu().numpy(), vd.cpu().numpy()
    assert abs(np.linalg.norm(v[0, :3]) - 100.0) < 1e-3
    assert (p[1] == (-1, -1, -1, 0)).all() and (v[1] == 0).all()
    assert (p[2] == (-1, -1, -1, 0)).all()
    acc = oracle.grid_accel(phi, 1.0)
    p_ref, v_ref = oracle.integrate(acc, pos, vel, 1e-3, 1e-3, 1e4)
    assert np.array_equal(p.view(np.int32), p_ref.view(np.int32))
    assert np.array_equal(v.view(np.int32), v_ref.view(np.int32))


def test_interpolate_accel_matches_oracle_sample(cuda, lib, oracle):
    G = 64
    pos, vel = random_particles(50_000, 8)
    phi = gpu_poisson(cuda, lib, oracle.density_fixed(pos, G), 1.0)
    out = cuda.empty((len(pos), 4), dtype=cuda.float32, device="cuda")
    phid, pd = dev(cuda, phi), dev(cuda, pos)
    L.check(lib.sd_interpolate_accel(phid.data_ptr(), G, ctypes.c_float(0.5), pd.data_ptr(), out.data_ptr(), len(pos),
                                     None), "interp")
    sync(cuda)
    acc = oracle.grid_accel(phi, 0.5)
    # kick with dt=1 from zero velocity, no drift: v = a exactly (fma(a, 1, 0) = a)
    z = np.zeros_like(vel)
    _, v_ref = oracle.integrate(acc, pos, z, 1.0, 0.0, 1e30)
    assert np.array_equal(out.cpu().numpy()[:, :3].view(np.int32), v_ref[:, :3].view(np.int32))
