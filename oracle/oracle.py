"""Python bindings of the CPU oracle (``pm_oracle.c``) plus FP64 references.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` leg of ``bench.py`` as the checker. The product path never
imports this module.

The C functions restate the reference's periodic PM step (chdnl0420-svg/stardust,
``src/sim/Sim.cu``); each wrapper names the reference lines it follows.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_pm.so")

KEY_ROWMAJOR = 0  # kCellKey, Sim.cu:2476-2486
KEY_MORTON = 1
KEY_TILEROW = 2

FIXED_ONE = np.float32(4294967296.0)

_lib = None


def build() -> str:
    """Compile ``liboracle_pm.so`` with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        i32, f32 = ctypes.c_int, ctypes.c_float
        L.or_cell_keys.argtypes = [P, i32, i32, i32, P]
        L.or_stable_sort_perm.argtypes = [P, i32, i32, P]
        L.or_reorder.argtypes = [P, P, i32, P]
        L.or_deposit_fixed.argtypes = [P, i32, i32, P]
        L.or_fixed_to_float.argtypes = [P, ctypes.c_size_t, P]
        L.or_deposit_float.argtypes = [P, i32, i32, P]
        L.or_poisson_periodic.argtypes = [P, i32, f32, P]
        L.or_grid_accel.argtypes = [P, i32, f32, P]
        L.or_integrate.argtypes = [P, P, P, i32, i32, f32, f32, f32]
        L.or_momentum_zero.argtypes = [P, P, i32, P]
        L.or_max_speed.argtypes = [P, P, i32]
        L.or_max_speed.restype = f32
        L.or_step.argtypes = [P, P, i32, i32, f32, f32, f32, f32, f32, i32, i32, P, P]
        L.or_step.restype = i32
        L.or_num_threads.restype = i32
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


def _f4(a) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    assert a.ndim == 2 and a.shape[1] == 4
    return a


def num_threads() -> int:
    return int(lib().or_num_threads())


def key_bits(G: int, mode: int) -> int:
    """Bits of the shifted key (key + 1) that a stable LSD sort must cover."""
    top = G * G if mode == KEY_TILEROW else G ** 3
    return int(top).bit_length()


def cell_keys(pos, G: int, mode: int = KEY_ROWMAJOR) -> np.ndarray:
    pos = _f4(pos)
    out = np.empty(len(pos), np.int32)
    lib().or_cell_keys(_p(pos), len(pos), G, mode, _p(out))
    return out


def stable_sort_perm(keys: np.ndarray, bits: int = 32) -> np.ndarray:
    keys = np.ascontiguousarray(keys, np.int32)
    perm = np.empty(len(keys), np.int32)
    lib().or_stable_sort_perm(_p(keys), len(keys), bits, _p(perm))
    return perm


def deposit_fixed(pos, G: int) -> np.ndarray:
    """int64 fixed-point CIC sums (weights rounded to multiples of 2^-32)."""
    pos = _f4(pos)
    acc = np.zeros(G ** 3, np.int64)
    lib().or_deposit_fixed(_p(pos), len(pos), G, _p(acc))
    return acc.reshape(G, G, G)


def fixed_to_float(acc: np.ndarray) -> np.ndarray:
    acc = np.ascontiguousarray(acc, np.int64)
    out = np.empty(acc.shape, np.float32)
    lib().or_fixed_to_float(_p(acc), acc.size, _p(out))
    return out


def density_fixed(pos, G: int) -> np.ndarray:
    return fixed_to_float(deposit_fixed(pos, G))


def density_float(pos, G: int) -> np.ndarray:
    """The reference's float deposit (kScatter, Sim.cu:503-521), index order."""
    pos = _f4(pos)
    rho = np.zeros(G ** 3, np.float32)
    lib().or_deposit_float(_p(pos), len(pos), G, _p(rho))
    return rho.reshape(G, G, G)


def poisson_periodic(rho: np.ndarray, soft_cells: float) -> np.ndarray:
    """kPoissonPeriodic + cuFFT round trip (Sim.cu:528-557, 3586-3603), float."""
    rho = np.ascontiguousarray(rho, np.float32)
    G = rho.shape[0]
    phi = np.empty_like(rho)
    lib().or_poisson_periodic(_p(rho), G, soft_cells, _p(phi))
    return phi


def grid_accel(phi: np.ndarray, pot_scale: float) -> np.ndarray:
    """kGridAccel, periodic (Sim.cu:589-611). Returns (G,G,G,4) float32."""
    phi = np.ascontiguousarray(phi, np.float32)
    G = phi.shape[0]
    acc = np.empty((G, G, G, 4), np.float32)
    lib().or_grid_accel(_p(phi), G, pot_scale, _p(acc))
    return acc


def integrate(acc, pos, vel, dt_kick: float, dt_drift: float, c2: float = 1.0e4):
    """Plain-PM kIntegrate on a periodic box (Sim.cu:685-906). Returns new (pos, vel)."""
    acc = np.ascontiguousarray(acc, np.float32)
    pos = _f4(pos).copy()
    vel = _f4(vel).copy()
    G = acc.shape[0]
    lib().or_integrate(_p(acc), _p(pos), _p(vel), len(pos), G, dt_kick, dt_drift, c2)
    return pos, vel


def momentum_zero(pos, vel):
    """kMomentumAccum + kSubtractMeanVelDev (Sim.cu:2252-2291)."""
    pos = _f4(pos)
    vel = _f4(vel).copy()
    out = np.zeros(4, np.float64)
    lib().or_momentum_zero(_p(pos), _p(vel), len(pos), _p(out))
    return vel, out


def max_speed(pos, vel) -> float:
    pos, vel = _f4(pos), _f4(vel)
    return float(lib().or_max_speed(_p(pos), _p(vel), len(pos)))


def step(pos, vel, G: int, gravity: float, soft_cells: float, dt_kick: float, dt_drift: float,
         c2: float = 1.0e4, key_mode: int = KEY_ROWMAJOR, deterministic: bool = True):
    """One reference-order step (Sim::step, Sim.cu:4240-4525, extras off).

    Returns (pos, vel, rho, momentum sums)."""
    pos = _f4(pos).copy()
    vel = _f4(vel).copy()
    rho = np.empty(G ** 3, np.float32)
    mom = np.zeros(4, np.float64)
    rc = lib().or_step(_p(pos), _p(vel), len(pos), G, gravity, soft_cells, dt_kick, dt_drift, c2,
                       key_mode, 1 if deterministic else 0, _p(rho), _p(mom))
    if rc != 0:
        raise MemoryError("oracle step: allocation failed")
    return pos, vel, rho.reshape(G, G, G), mom


# ---------------------------------------------------------------------------
# FP64 references (numpy)
# ---------------------------------------------------------------------------

def green_periodic_f64(G: int, soft_cells: float) -> np.ndarray:
    """The reference's periodic Green's function on the rfft half spectrum, FP64:
    -1/(4 pi^2 k^2) * exp(-k^2 s^2 / 2), s = 2 pi soft / G, k = 0 -> 0
    (kPoissonPeriodic, Sim.cu:528-557; FFT normalisation 1/G^3 included)."""
    k = np.fft.fftfreq(G, d=1.0 / G)
    kx = np.arange(G // 2 + 1, dtype=np.float64)
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + kx[None, None, :] ** 2
    with np.errstate(divide="ignore"):
        m = -1.0 / (4.0 * np.pi ** 2 * k2) / float(G) ** 3
    m[0, 0, 0] = 0.0
    if soft_cells > 0:
        s = 2.0 * np.pi * soft_cells / G
        m *= np.exp(-0.5 * k2 * s * s)
    return m


def poisson_periodic_f64(rho: np.ndarray, soft_cells: float) -> np.ndarray:
    """FP64 periodic solve with the reference's conventions (unnormalised FFT
    pair, Green's function scaled by 1/G^3)."""
    G = rho.shape[0]
    spec = np.fft.rfftn(rho.astype(np.float64))
    spec *= green_periodic_f64(G, soft_cells)
    return np.fft.irfftn(spec, s=rho.shape, axes=(0, 1, 2)) * float(G) ** 3


def central_gradient_f64(phi: np.ndarray, pot_scale: float) -> np.ndarray:
    """kGridAccel's central difference in FP64: (G,G,G,3) with axes (x,y,z)."""
    G = phi.shape[0]
    h = 0.5 * G * pot_scale
    ax = -(np.roll(phi, -1, axis=2) - np.roll(phi, 1, axis=2)) * h
    ay = -(np.roll(phi, -1, axis=1) - np.roll(phi, 1, axis=1)) * h
    az = -(np.roll(phi, -1, axis=0) - np.roll(phi, 1, axis=0)) * h
    return np.stack([ax, ay, az], axis=-1)


def cic_weights_f64(pos: np.ndarray, G: int):
    """CIC base cells and the 8 corner weights in FP64 (Sim.cu:509-518)."""
    g = pos[:, :3].astype(np.float64) * G - 0.5
    i = np.floor(g).astype(np.int64)
    f = g - i
    out_idx, out_w = [], []
    for k in range(8):
        o = np.array([k & 1, (k >> 1) & 1, (k >> 2) & 1])
        c = (i + o) % G
        w = np.prod(np.where(o[None, :] == 1, f, 1.0 - f), axis=1)
        out_idx.append(c)
        out_w.append(w)
    return out_idx, out_w


def density_f64(pos: np.ndarray, G: int) -> np.ndarray:
    live = pos[:, 0] >= 0
    p = pos[live]
    rho = np.zeros((G, G, G), np.float64)
    idx, w = cic_weights_f64(p, G)
    for c, wk in zip(idx, w):
        np.add.at(rho, (c[:, 2], c[:, 1], c[:, 0]), wk)
    return rho


def pm_accel_f64(pos: np.ndarray, G: int, pot_scale: float, soft_cells: float) -> np.ndarray:
    """Per-particle PM acceleration in FP64 with the reference's operators: CIC
    deposit, periodic Green's function, central difference, CIC gather."""
    rho = density_f64(pos, G)
    phi = poisson_periodic_f64(rho, soft_cells)
    grad = central_gradient_f64(phi, pot_scale)
    idx, w = cic_weights_f64(pos, G)
    a = np.zeros((len(pos), 3), np.float64)
    for c, wk in zip(idx, w):
        a += grad[c[:, 2], c[:, 1], c[:, 0]] * wk[:, None]
    return a


# ---------------------------------------------------------------------------
# Isolated boundary in FP64 (Hockney-Eastwood on the 2G box, the reference's
# kScatter with clamped corners Sim.cu:96-100,503-521, kGreen Sim.cu:563-576,
# kMulSpec + FFT normalisation Sim.cu:3586-3603, kGridAccel and sampleAcc with
# clamped indices Sim.cu:589-629).
# ---------------------------------------------------------------------------
def cic_weights_iso_f64(pos: np.ndarray, G: int):
    """CIC corner cells clamped to [0, G) and their weights in FP64."""
    g = pos[:, :3].astype(np.float64) * G - 0.5
    i = np.floor(g).astype(np.int64)
    f = g - i
    out_idx, out_w = [], []
    for k in range(8):
        o = np.array([k & 1, (k >> 1) & 1, (k >> 2) & 1])
        out_idx.append(np.clip(i + o, 0, G - 1))
        out_w.append(np.prod(np.where(o[None, :] == 1, f, 1.0 - f), axis=1))
    return out_idx, out_w


def density_iso_f64(pos: np.ndarray, G: int) -> np.ndarray:
    p = pos[pos[:, 0] >= 0]
    rho = np.zeros((G, G, G), np.float64)
    idx, w = cic_weights_iso_f64(p, G)
    for c, wk in zip(idx, w):
        np.add.at(rho, (c[:, 2], c[:, 1], c[:, 0]), wk)
    return rho


def green_isolated_f64(S: int, soft_cells: float) -> np.ndarray:
    """kGreen: -1/(r + soft) in cells to the nearest corner copy of the S^3 box,
    soft floored at half a cell (buildGreen, Sim.cu:3572)."""
    soft = max(float(soft_cells), 0.5)
    d = np.arange(S)
    d = np.minimum(d, S - d).astype(np.float64)
    r = np.sqrt(d[:, None, None] ** 2 + d[None, :, None] ** 2 + d[None, None, :] ** 2)
    return -1.0 / (r + soft)


def poisson_isolated_f64(rho: np.ndarray, soft_cells: float) -> np.ndarray:
    """Potential on the G^3 region: the zero-padded density convolved with the
    isolated kernel on the 2G box (what the reference's FFT pair computes)."""
    G = rho.shape[0]
    S = 2 * G
    pad = np.zeros((S, S, S), np.float64)
    pad[:G, :G, :G] = rho
    spec = np.fft.rfftn(pad) * np.fft.rfftn(green_isolated_f64(S, soft_cells))
    return np.fft.irfftn(spec, s=(S, S, S), axes=(0, 1, 2))[:G, :G, :G]


def central_gradient_iso_f64(phi: np.ndarray, pot_scale: float) -> np.ndarray:
    """kGridAccel with neighbours clamped to [0, G): (G,G,G,3), axes (x,y,z)."""
    G = phi.shape[0]
    h = 0.5 * G * pot_scale
    i = np.arange(G)
    ip, im = np.minimum(i + 1, G - 1), np.maximum(i - 1, 0)
    ax = -(phi[:, :, ip] - phi[:, :, im]) * h
    ay = -(phi[:, ip, :] - phi[:, im, :]) * h
    az = -(phi[ip, :, :] - phi[im, :, :]) * h
    return np.stack([ax, ay, az], axis=-1)


def pm_accel_iso_f64(pos: np.ndarray, G: int, pot_scale: float, soft_cells: float) -> np.ndarray:
    rho = density_iso_f64(pos, G)
    grad = central_gradient_iso_f64(poisson_isolated_f64(rho, soft_cells), pot_scale)
    idx, w = cic_weights_iso_f64(pos, G)
    a = np.zeros((len(pos), 3), np.float64)
    for c, wk in zip(idx, w):
        a += grad[c[:, 2], c[:, 1], c[:, 0]] * wk[:, None]
    return a


def isolated_wall(p: np.ndarray, v: np.ndarray):
    """The reference's isolated wall (Sim.cu:895-903), float32: a coordinate past
    0.002 / 0.998 is set there and its velocity reversed inward at a quarter speed."""
    p = p.astype(np.float32).copy()
    v = v.astype(np.float32).copy()
    for ax in range(3):
        lo = p[:, ax] < np.float32(0.002)
        p[lo, ax] = np.float32(0.002)
        v[lo, ax] = np.abs(v[lo, ax]) * np.float32(0.25)
        hi = p[:, ax] > np.float32(0.998)
        p[hi, ax] = np.float32(0.998)
        v[hi, ax] = -np.abs(v[hi, ax]) * np.float32(0.25)
    return p, v


def force_error(a: np.ndarray, a_ref: np.ndarray) -> dict:
    """eps = RMS(|a - a_ref|) / RMS(|a_ref|), the reference's scoring metric
    (.drive/nbody-simulator/method-search/scoring.md:38), plus the max."""
    d = np.linalg.norm(np.asarray(a, np.float64) - a_ref, axis=1)
    r = np.sqrt(np.mean(np.sum(a_ref * a_ref, axis=1)))
    return {"rms_rel": float(np.sqrt(np.mean(d * d)) / r), "max_rel": float(d.max() / r)}


def ewald_forces_f64(src: np.ndarray, tgt: np.ndarray, softening: float, split_b: float, nmax: int) -> np.ndarray:
    """FP64 Ewald forces of Gaussian-smoothed masses, vectorised numpy (small
    systems only): the same split as the GPU Ewald kernels, written independently.
    Long range over modes 0 < |n| <= nmax (all of them, no half-space folding),
    short range over all sources at their nearest image with the pair kernel
    -m [erf(r/a) - erf(r/b)]/r, a = sqrt(2) softening."""
    from scipy.special import erf

    xs = np.asarray(src, np.float64)[:, :3]
    xt = np.asarray(tgt, np.float64)[:, :3]
    m = 1.0 / len(xs)
    r = np.arange(-nmax, nmax + 1)
    n = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3)
    n2 = np.sum(n * n, axis=1)
    n = n[(n2 > 0) & (n2 <= nmax * nmax)]
    k = 2.0 * np.pi * n.astype(np.float64)
    k2 = np.sum(k * k, axis=1)
    c = 4.0 * np.pi * np.exp(-0.25 * k2 * split_b * split_b) / k2
    rho = m * np.exp(-1j * (xs @ k.T)).sum(axis=0)                    # (modes,)
    ph = np.exp(1j * (xt @ k.T))                                         # (tgt, modes)
    a_long = -(np.imag(ph * rho[None, :]) * c[None, :]) @ k              # (tgt, 3)
    d = xt[:, None, :] - xs[None, :, :]
    d -= np.rint(d)
    r2 = np.sum(d * d, axis=2)
    rr = np.sqrt(np.maximum(r2, 1e-300))
    a_len = np.sqrt(2.0) * softening
    e = erf(rr / a_len) - erf(rr / split_b)
    dfdr = (2.0 / (np.sqrt(np.pi) * a_len) * np.exp(-r2 / a_len ** 2)
            - 2.0 / (np.sqrt(np.pi) * split_b) * np.exp(-r2 / split_b ** 2)) / rr - e / rr ** 2
    g = np.where((r2 > 1e-24) & (r2 <= 0.25), m * dfdr / rr, 0.0)
    a_short = np.sum(g[:, :, None] * d, axis=1)
    return a_long + a_short


# ---------------------------------------------------------------------------
# Learned correction: features and the MLP, numpy, with the GPU's BF16 rounding
# points (inputs, weights and hidden activations rounded to bf16, products
# accumulated in float64 here), as the checker of the tensor-core kernels.
# ---------------------------------------------------------------------------
MLP_IN, MLP_H, MLP_OUT = 32, 64, 8
MLP_OFF = {"W1": (0, (32, 64)), "b1": (2048, (64,)), "W2": (2112, (64, 64)), "b2": (6208, (64,)),
           "W3": (6272, (64, 8)), "b3": (6784, (8,))}
MLP_PARAMS = 6792


def bf16(x) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)


def mlp_unpack(params):
    p = np.asarray(params, np.float32)
    return {k: p[o:o + int(np.prod(sh))].reshape(sh) for k, (o, sh) in MLP_OFF.items()}


def mlp_features(pos, rho, G: int, inv_mean: float) -> np.ndarray:
    """(n, 32) float32 features (before the bf16 rounding)."""
    pos = _f4(pos)
    n = len(pos)
    f = np.zeros((n, 32), np.float32)
    live = pos[:, 0] >= 0
    p = pos[live, :3]
    c = np.clip((p * np.float32(G)).astype(np.int64), 0, G - 1)
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                r = rho[(c[:, 2] + dz) % G, (c[:, 1] + dy) % G, (c[:, 0] + dx) % G]
                f[live, (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)] = (np.log1p(r.astype(np.float64) * inv_mean)
                                                                   - np.log(2.0))
    f[live, 27:30] = p * np.float32(G) - c.astype(np.float32) - np.float32(0.5)
    return f


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def _rounder(round_bf16: bool):
    """bf16 rounding (through float32, as the kernels store) or exact float64."""
    if round_bf16:
        return lambda a: bf16(np.asarray(a, np.float32)).astype(np.float64)
    return lambda a: np.asarray(a, np.float64)


def mlp_forward(params, X, round_bf16: bool = True):
    """Y (n, 3) and the cache of the forward pass."""
    P = mlp_unpack(params) if round_bf16 else {k: np.asarray(params, np.float64)[o:o + int(np.prod(sh))].reshape(sh)
                                               for k, (o, sh) in MLP_OFF.items()}
    r = _rounder(round_bf16)
    Xb = r(X)
    W1, W2, W3 = (r(P[k]) for k in ("W1", "W2", "W3"))
    z1 = Xb @ W1 + P["b1"]
    h1 = r(_silu(z1))
    z2 = h1 @ W2 + P["b2"]
    h2 = r(_silu(z2))
    y = h2 @ W3 + P["b3"]
    return y[:, :3], dict(X=Xb, z1=z1, h1=h1, z2=z2, h2=h2, W1=W1, W2=W2, W3=W3)


def mlp_loss_grad(params, X, T, round_bf16: bool = True):
    """Sum of squared errors and the gradient (packed like params) of the mean
    squared error over rows and the 3 outputs."""
    r = _rounder(round_bf16)
    y, c = mlp_forward(params, X, round_bf16)
    rows = len(X)
    diff = y - T
    sse = float(np.sum(diff * diff))
    dy = np.zeros((rows, MLP_OUT))
    dy[:, :3] = 2.0 * diff / (3.0 * rows)
    dy = r(dy)
    g = np.zeros(MLP_PARAMS, np.float64)

    def put(name, val):
        o, sh = MLP_OFF[name]
        g[o:o + int(np.prod(sh))] = val.reshape(-1)

    put("W3", c["h2"].T @ dy)
    put("b3", dy.sum(axis=0))
    dh2 = dy @ c["W3"].T
    dz2 = r(dh2 * _silu_grad(c["z2"]))
    put("W2", c["h1"].T @ dz2)
    put("b2", dz2.sum(axis=0))
    dh1 = dz2 @ c["W2"].T
    dz1 = r(dh1 * _silu_grad(c["z1"]))
    put("W1", c["X"].T @ dz1)
    put("b1", dz1.sum(axis=0))
    return sse, g


# ---------------------------------------------------------------------------
# Headless point render (kSplatPoints -> kAccumToRGBA, src/gfx/RenderField.cu
# 318-735; projectPoint src/sim/ViewRot.h:76-96), numpy float64 math with the
# same 2^-24 fixed-point accumulation as the GPU.
# ---------------------------------------------------------------------------
_ASTRO_C = np.array([[0.00, 0.00, 0.00], [0.05, 0.06, 0.19], [0.16, 0.14, 0.47], [0.47, 0.27, 0.67],
                     [0.88, 0.55, 0.27], [1.00, 0.84, 0.51], [1.00, 1.00, 0.94]])
_ASTRO_S = np.array([0.00, 0.18, 0.38, 0.58, 0.76, 0.90, 1.00])


# ---- grid hydrodynamics add-ons (doCooling, kPressure; Sim.cu:1212-1415, 3605-3868) ----

def containing_cell(pos, G: int) -> np.ndarray:
    """Flat index (z G + y) G + x of the containing cell, clamp((int)(p G), 0, G-1)
    (kAccumCellVel, Sim.cu:1227-1230)."""
    c = np.clip((np.asarray(pos, np.float32)[:, :3] * np.float32(G)).astype(np.int64), 0, G - 1)
    return (c[:, 2] * G + c[:, 1]) * G + c[:, 0]


def hydro_cool(pos, vel, G: int, k: float, pressure: bool):
    """One cooling pass (kAccumCellVel + kCoolCell, Sim.cu:1212-1310) with sums in
    float64: returns the cooled float32 velocities and, with pressure, the
    dispersion grids (3, G^3) and their counts (G^3)."""
    pos = np.asarray(pos, np.float32)
    vel = np.array(vel, np.float32)
    cells = G ** 3
    live = (pos[:, 0] >= 0) & np.isfinite(vel[:, :3]).all(axis=1) & (vel[:, 3] >= -50)
    c = containing_cell(pos, G)
    sums = np.zeros((3, cells))
    cnt = np.zeros(cells, np.int64)
    for d in range(3):
        np.add.at(sums[d], c[live], vel[live, d].astype(np.float64))
    np.add.at(cnt, c[live], 1)
    act = live & (cnt[c] >= 2)
    inv = (np.float32(1.0) / cnt[c[act]].astype(np.float32))
    dv = np.stack([sums[d][c[act]].astype(np.float32) * inv - vel[act, d] for d in range(3)], axis=1)
    disp = np.zeros((3, cells))
    dcnt = np.zeros(cells, np.int64)
    if pressure:
        for d in range(3):
            np.add.at(disp[d], c[act], (dv[:, d] * dv[:, d]).astype(np.float64))
        np.add.at(dcnt, c[act], 1)
    gas = pos[act, 3] <= 0
    idx = np.nonzero(act)[0][gas]
    vel[idx, :3] = vel[idx, :3] + np.float32(k) * dv[gas]
    return vel, disp, dcnt


def pressure_field(disp, dcnt, G: int, pressure_k: float, periodic: bool = True) -> np.ndarray:
    """kPressure (Sim.cu:1368-1400): -(disp_d[+1] - disp_d[-1]) G/2 k / count per
    axis, clamped to +-5, zero where the count is zero; (G^3, 3) float32."""
    d = np.asarray(disp, np.float64).reshape(3, G, G, G).astype(np.float32)
    rho = np.asarray(dcnt).reshape(G, G, G).astype(np.float32)

    def shift(a, axis, s):
        if periodic:
            return np.roll(a, -s, axis=axis)
        idx = np.clip(np.arange(G) + s, 0, G - 1)
        return np.take(a, idx, axis=axis)

    h = np.where(rho > 0, np.float32(0.5) * np.float32(G) * np.float32(pressure_k) / np.where(rho > 0, rho, 1),
                 0).astype(np.float32)
    out = np.zeros((G, G, G, 3), np.float32)
    for ax, axis in ((0, 2), (1, 1), (2, 0)):  # x is the last array axis
        g = -(shift(d[ax], axis, 1) - shift(d[ax], axis, -1)) * h
        out[..., ax] = np.clip(g, -5.0, 5.0)
    out[rho < 1e-6] = 0
    return out.reshape(-1, 3)


def sample_field(field, pos, G: int, periodic: bool = True) -> np.ndarray:
    """CIC sample of a (G^3, 3) field at the positions (sampleAcc, Sim.cu:614-629)."""
    pos = np.asarray(pos, np.float64)
    f = np.asarray(field, np.float64)
    g = pos[:, :3] * G - 0.5
    i0 = np.floor(g).astype(np.int64)
    fr = g - i0
    a = np.zeros((len(pos), 3))
    for k in range(8):
        o = np.array([k & 1, (k >> 1) & 1, (k >> 2) & 1])
        c = i0 + o
        c = (c & (G - 1)) if periodic else np.clip(c, 0, G - 1)
        w = np.prod(np.where(o == 1, fr, 1 - fr), axis=1)
        a += w[:, None] * f[(c[:, 2] * G + c[:, 1]) * G + c[:, 0]]
    return a


# ---- initial conditions of Sim::reset (Sim.cu:4160-4238) -------------------------

PRESET_FILAMENT, PRESET_EMPTY = 0, 1
_U32 = np.uint32


def pcg_hash(v) -> np.ndarray:
    """pcgHash (Sim.cu:78-82), uint32 arithmetic modulo 2^32."""
    with np.errstate(over="ignore"):
        s = np.asarray(v, _U32) * _U32(747796405) + _U32(2891336453)
        w = ((s >> ((s >> _U32(28)) + _U32(4))) ^ s) * _U32(277803737)
        return (w >> _U32(22)) ^ w


def rnd01(s) -> np.ndarray:
    """rnd01 (Sim.cu:84-86): the hash rounded to float32 times 2^-32."""
    return pcg_hash(s).astype(np.float32) * np.float32(2.3283064365386963e-10)


def _mul(s, a: int, b: int):
    with np.errstate(over="ignore"):
        return np.asarray(s, _U32) * _U32(a) + _U32(b)


def _sphere_dir(s):
    f = np.float32
    cz = rnd01(_mul(s, 3, 1)) * f(2.0) - f(1.0)
    sz = np.sqrt(np.maximum(f(1.0) - cz * cz, f(0.0))).astype(f)
    ph = rnd01(_mul(s, 7, 5)) * f(6.2831853)
    return cz, sz, ph


def _at_radius(r, cz, sz, ph):
    f = np.float32
    return (r * sz * np.cos(ph).astype(f), r * sz * np.sin(ph).astype(f), r * cz)


def place_preset(n: int, preset: int = PRESET_FILAMENT, dark_frac: float = 0.0, shrink: float = 0.0,
                 spin: float = 0.0, hubble: float = 0.0, vrms: float = 0.0):
    """Sim::reset's particles in float32: kPlace (Sim.cu:281-407) with seed 12345
    (Sim.cu:3642) for the Filament / Empty presets, then kAddSpin, kAddHubble and
    kAddDispersion (Sim.cu:2406-2476, seed 24680) and, for Filament, the
    centre-of-mass stop over all n slots (Sim.cu:4218-4235). Angles use libm
    sin/cos where the reference uses the fast intrinsics, so positions agree with
    it to a few 1e-7."""
    f = np.float32
    i = np.arange(n, dtype=_U32)
    s = _mul(i, 2654435761, 12345)
    pos = np.zeros((n, 4), f)
    vel = np.zeros((n, 4), f)
    dark = (rnd01(_mul(s, 13, 7)) < f(dark_frac)) if dark_frac > 0 else np.zeros(n, bool)
    if preset == PRESET_FILAMENT:
        cz, sz, ph = _sphere_dir(s ^ _U32(0x6C8E9CF5))
        r = f(0.5) * np.cbrt(np.maximum(rnd01(s ^ _U32(0x6C8E9CF5)), f(1e-9))).astype(f)
        bx, by, bz = _at_radius(r, cz, sz, ph)
        x, y, z = f(0.5) + bx, f(0.5) + by, f(0.5) + bz
        dx = np.zeros(n, f)
        dy = np.zeros(n, f)
        dz = np.zeros(n, f)
        for m in range(3):
            fm = f(m)
            k = f(6.2831853) * (f(2.0) + fm * f(2.0))
            amp = f(0.16) / (f(1.0) + fm)
            dx = dx + amp * np.sin(k * (y + f(0.13) * fm)).astype(f) * np.cos(k * (z + f(0.29))).astype(f)
            dy = dy + amp * np.sin(k * (z + f(0.19) * fm)).astype(f) * np.cos(k * (x + f(0.37))).astype(f)
            dz = dz + amp * np.sin(k * (x + f(0.23) * fm)).astype(f) * np.cos(k * (y + f(0.11))).astype(f)
        px, py, pz = x + dx, y + dy, z + dz
        rx, ry, rz = px - f(0.5), py - f(0.5), pz - f(0.5)
        rr = np.sqrt(rx * rx + ry * ry + rz * rz).astype(f)
        out = rr > f(0.5)
        q = np.where(out, f(0.5) / np.where(out, rr, f(1.0)), f(1.0)).astype(f)
        px = np.where(out, f(0.5) + rx * q, px)
        py = np.where(out, f(0.5) + ry * q, py)
        pz = np.where(out, f(0.5) + rz * q, pz)
        if shrink > 0:
            sh = f(shrink)
            px, py, pz = f(0.5) + (px - f(0.5)) * sh, f(0.5) + (py - f(0.5)) * sh, f(0.5) + (pz - f(0.5)) * sh
        pos[:, 0], pos[:, 1], pos[:, 2] = px, py, pz
        vel[:, 3] = np.where(dark, f(-100.0), f(0.0))
    else:
        pos[:, :3] = -1.0
        if dark.any():  # the dark fraction still lands in a halo (bulgePoint, Sim.cu:228-236)
            sd = s[dark] ^ _U32(0x2545F491)
            u = rnd01(sd)
            cz, sz, ph = _sphere_dir(sd)
            hx, hy, hz = _at_radius(f(0.42) * u * u, cz, sz, ph)
            pos[dark, 0], pos[dark, 1], pos[dark, 2] = f(0.5) + hx, f(0.5) + hy, f(0.5) + hz
            vel[dark, 3] = -100.0
    live = pos[:, 0] >= 0
    v = vel[:, :3]
    if spin != 0:
        om = f(spin)
        ry, rx = pos[:, 1] - f(0.5), pos[:, 0] - f(0.5)
        v[live, 0] += -om * ry[live]
        v[live, 1] += om * rx[live]
    if hubble != 0:
        v[live] += f(hubble) * (pos[live, :3] - f(0.5))
    if vrms > 0:
        sd = _mul(i, 2654435761, 24680)
        cz, sz, ph = _sphere_dir(sd)
        g = (rnd01(_mul(sd, 11, 3)) + rnd01(_mul(sd, 13, 7)) + rnd01(_mul(sd, 17, 9))) / f(1.5)
        a = f(vrms) * g
        add = np.stack([a * sz * np.cos(ph).astype(f), a * sz * np.sin(ph).astype(f), a * cz], axis=1)
        v[live] += add[live]
    if preset == PRESET_FILAMENT and n > 0:
        mean = (v[live].astype(np.float64).sum(axis=0) / n).astype(f)
        v[live] -= mean
    return pos, vel


def _cmap(kind: int, t: np.ndarray) -> np.ndarray:
    t = np.clip(np.asarray(t, np.float64), 0.0, 1.0)
    if kind == 1:
        return np.stack([t, t, t], axis=-1)
    if kind == 2:
        return np.stack([np.minimum(t * 2.2, 1.0), np.clip((t - 0.32) * 1.9, 0.0, 1.0),
                         np.clip((t - 0.70) * 3.2, 0.0, 1.0)], axis=-1)
    if kind == 3:  # cmapBlackbody (RenderField.cu:60-82)
        u = np.where(t < 0.5, t * 2.0, (t - 0.5) * 2.0)
        r = np.where(t < 0.5, 1.0, 1.0 - 0.38 * u)
        g = np.where(t < 0.5, 0.32 + 0.68 * u, 1.0 - 0.30 * u)
        b = np.where(t < 0.5, 0.08 + 0.80 * u * u, 1.0)
        dim = np.minimum(t * 3.2, 1.0)
        return np.stack([r * dim, g * dim, b * dim], axis=-1)
    return np.stack([np.interp(t, _ASTRO_S, _ASTRO_C[:, j]) for j in range(3)], axis=-1)


def project_field(rho: np.ndarray, view: dict) -> np.ndarray:
    """kProjectXY (Sim.cu:2526-2537): the G^3 density summed along z (view off) or
    each cell's centre through the view rotation into its screen cell; (G, G)
    indexed [y, x]."""
    rho = np.asarray(rho, np.float64)
    G = rho.shape[0]
    if not view.get("rot_on", 0):
        return rho.sum(axis=0)
    z, y, x = np.nonzero(rho)
    c = (np.stack([x, y, z], axis=1) + 0.5) / G - np.asarray(view["center"], np.float64)
    R = np.asarray(view["rot"], np.float64).reshape(3, 3)
    ox, oy = c @ R[0] + 0.5, c @ R[1] + 0.5
    ok = (ox >= 0) & (ox < 1) & (oy >= 0) & (oy < 1)
    sx, sy = (ox[ok] * G).astype(np.int64), (oy[ok] * G).astype(np.int64)
    out = np.zeros((G, G))
    np.add.at(out, (sy, sx), rho[z[ok], y[ok], x[ok]])
    return out


def dispersion_field(pos, vel, G: int, view: dict) -> np.ndarray:
    """kScatterDispersion + kDivideInto (Sim.cu:2548-2570, 2701-2707): the rms
    speed under each screen cell, bilinear weights with edge clamping."""
    pos = np.asarray(pos, np.float64)
    vel = np.asarray(vel, np.float64)
    live = pos[:, 0] >= 0
    p, v = pos[live], vel[live]
    v2 = np.sum(v[:, :3] ** 2, axis=1)
    if view.get("rot_on", 0):
        c = p[:, :3] - np.asarray(view["center"], np.float64)
        R = np.asarray(view["rot"], np.float64).reshape(3, 3)
        ux, uy = c @ R[0] + 0.5, c @ R[1] + 0.5
        ok = (ux >= 0) & (ux < 1) & (uy >= 0) & (uy < 1)
        ux, uy, v2 = ux[ok], uy[ok], v2[ok]
    else:
        ux, uy = p[:, 0], p[:, 1]
    gx, gy = ux * G - 0.5, uy * G - 0.5
    ix, iy = np.floor(gx).astype(np.int64), np.floor(gy).astype(np.int64)
    fx, fy = gx - ix, gy - iy
    num = np.zeros((G, G))
    den = np.zeros((G, G))
    for ox in (0, 1):
        for oy in (0, 1):
            cx, cy = np.clip(ix + ox, 0, G - 1), np.clip(iy + oy, 0, G - 1)
            w = (fx if ox else 1 - fx) * (fy if oy else 1 - fy)
            np.add.at(num, (cy, cx), w * v2)
            np.add.at(den, (cy, cx), w)
    return np.where(den > 1e-6, np.sqrt(np.maximum(num / np.where(den > 1e-6, den, 1.0), 0.0)), 0.0)


def field_brightness(g: np.ndarray, n: int, brightness: float) -> float:
    """The density view's brightness factor (RenderField.cu:125-137, 930-1000):
    brightness over the value 5 % from the top of a 64-bin log histogram of the
    positive cells, interpolated in its bin (n / G^2 when nothing is positive)."""
    G = g.shape[0]
    norm = n / (G * G)
    vals = g[g > 0]
    if len(vals):
        b = np.clip(((np.log(vals) + 9.21) / (18.42 + 9.21) * 64).astype(np.int64), 0, 63)
        h = np.bincount(b, minlength=64)
        total = int(h.sum())
        want = int(total * 0.05) + 1
        acc, hit = 0, 63
        for k in range(63, -1, -1):
            acc += int(h[k])
            if acc >= want:
                hit = k
                break
        below = acc - int(h[hit])
        frac = min(max((want - below) / h[hit], 0.0), 1.0) if h[hit] > 0 else 0.5
        m = float(np.exp((hit + 1.0 - frac) / 64 * (18.42 + 9.21) - 9.21))
        if m > 1e-6:
            norm = m
    return brightness / max(norm, 1e-6)


def shade(g: np.ndarray, bright: float, view: dict, W: int, H: int) -> np.ndarray:
    """kShade (RenderField.cu:158-316) over a (G, G) field; rows bottom-up."""
    G = g.shape[0]
    y, x = np.mgrid[0:H, 0:W]
    u, v = (x + 0.5) / W, (y + 0.5) / H
    aspect = W / H
    if aspect > 1:
        u = (u - 0.5) * aspect + 0.5
    else:
        v = (v - 0.5) / aspect + 0.5
    u = (u - 0.5) / view["zoom"] + 0.5 - view["pan_x"]
    v = (v - 0.5) / view["zoom"] + 0.5 - view["pan_y"]
    inside = (u >= 0) & (u < 1) & (v >= 0) & (v < 1)
    gfx, gfy = u * G - 0.5, v * G - 0.5
    x0, y0 = np.floor(gfx).astype(np.int64), np.floor(gfy).astype(np.int64)
    tx, ty = gfx - x0, gfy - y0
    x1, y1 = np.clip(x0 + 1, 0, G - 1), np.clip(y0 + 1, 0, G - 1)
    x0, y0 = np.clip(x0, 0, G - 1), np.clip(y0, 0, G - 1)
    d = (g[y0, x0] * (1 - tx) * (1 - ty) + g[y0, x1] * tx * (1 - ty) + g[y1, x0] * (1 - tx) * ty +
         g[y1, x1] * tx * ty)
    xl = np.maximum(np.log1p(d * bright) * 0.60, 0.0)
    t = np.power(xl / (1 + xl), view["inv_gamma"])
    rgb = (_cmap(view["cmap"], t) * 255.0).astype(np.uint8)
    out = np.zeros((H, W, 4), np.uint8)
    out[..., 3] = 255
    out[..., :3] = np.where(inside[..., None], rgb, 0)
    return out[::-1]


def render_field(field: int, rho, pos, vel, G: int, view: dict, W: int, H: int) -> np.ndarray:
    """(H, W, 4) uint8 grid view: field 0 the density (rho, G^3 z-major), 1 the
    velocity dispersion of the particles."""
    if field == 0:
        g = project_field(np.asarray(rho).reshape(G, G, G), view)
        bright = field_brightness(g, len(pos) if pos is not None else 0, view["bright"])
    else:
        g = dispersion_field(pos, vel, G, view)
        bright = view["bright"] * 60.0
    return shade(g, bright, view, W, H)


def render_points(pos, vel, view: dict, W: int, H: int) -> np.ndarray:
    """(H, W, 4) uint8 image of the gas particles."""
    pos = np.asarray(pos, np.float64)
    vel = np.asarray(vel, np.float64)
    n = len(pos)
    keep = (pos[:, 0] >= 0) & (pos[:, 3] == 0)
    p, v = pos[keep], vel[keep]
    R = np.asarray(view["rot"], np.float64).reshape(3, 3)
    f = p[:, :3] - np.asarray(view["center"], np.float64)
    xc, yc, zc = f @ R[0], f @ R[1], f @ R[2]
    depth = np.ones(len(p))
    if view["fly"]:
        ok = zc >= 1e-3
        k = 0.5 / (np.where(ok, zc, 1.0) * view["tan_half_fov"])
        u, w = xc * k + 0.5, yc * k + 0.5
        depth = zc
    else:
        ok = np.ones(len(p), bool)
        u = (xc + view["pan_x"]) * view["zoom"] + 0.5
        w = (yc + view["pan_y"]) * view["zoom"] + 0.5
    aspect = W / H
    if aspect > 1:
        u = (u - 0.5) / aspect + 0.5
    else:
        w = (w - 0.5) * aspect + 0.5
    ok &= (u >= 0) & (u < 1) & (w >= 0) & (w < 1)
    x = (u * W).astype(np.int64)
    y = ((1.0 - w) * H).astype(np.int64)
    ok &= (x >= 0) & (x < W) & (y >= 0) & (y < H)
    if view["color_by"] == 0:
        base = {1: [1.0, 1.0, 1.0], 2: list(_cmap(2, np.array([0.62]))[0])}.get(view["cmap"], [0.55, 0.42, 0.85])
        c = np.tile(np.asarray(base, np.float64), (len(p), 1))
    else:
        t = np.full(len(p), 0.5)
        if view["color_by"] == 2:
            t = np.minimum(np.sqrt(np.sum(v[:, :3] ** 2, axis=1)) * 0.25, 1.0)
        c = _cmap(view["cmap"], t)
    visible = n / max(view["zoom"] ** 2, 1.0)
    cap = 0 if visible > 8.0e6 else (1 if visible > 2.0e6 else 2)
    grow = (np.minimum(0.35 / np.maximum(depth, 1e-3), 6.0) if view["fly"]
            else np.full(len(p), min(np.sqrt(max(view["zoom"], 1.0)), 4.0)))
    rr = view["size_px"] * grow
    rad = np.minimum(np.where(rr < 2.0, 0, np.where(rr < 4.0, 1, 2)), cap)
    acc = np.zeros((H, W, 3), np.int64)
    kern = {0: np.array([1.0]), 1: np.array([0.25, 0.5, 0.25]), 2: np.array([0.0625, 0.25, 0.375, 0.25, 0.0625])}
    for r in (0, 1, 2):
        sel = ok & (rad == r)
        k = kern[r]
        for dy in range(-r, r + 1):
            for dx in range(-r, r + 1):
                xx, yy = x[sel] + dx, y[sel] + dy
                inb = (xx >= 0) & (xx < W) & (yy >= 0) & (yy < H)
                q = np.rint(c[sel][inb] * (k[dy + r] * k[dx + r]) * 16777216.0).astype(np.int64)
                np.add.at(acc, (yy[inb], xx[inb]), q)
    a = acc.astype(np.float64) / 16777216.0
    lum = a.sum(axis=-1) * 0.3333
    out = np.zeros((H, W, 4), np.uint8)
    if view["use_cmap"]:
        t = np.power(np.minimum(np.log1p(lum * view["bright"]) * 0.42, 1.0), view["inv_gamma"])
        rgb = _cmap(view["cmap"], t)
    else:
        x_ = np.log1p(lum * view["bright"]) * 0.42
        tone = (np.power(np.maximum(x_, 0) / (1 + np.maximum(x_, 0)), view["inv_gamma"]) if view["reinhard"]
                else np.power(np.minimum(x_, 1.0), view["inv_gamma"]))
        s = np.where(lum > 1e-6, tone / np.maximum(lum, 1e-30), 0.0)
        rgb = np.minimum(a * s[..., None], 1.0)
    out[..., :3] = (np.minimum(rgb, 1.0) * 255.0).astype(np.uint8)
    out[..., 3] = 255
    return out
