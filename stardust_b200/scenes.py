"""Seeded initial conditions for the benchmark workloads (scene init).

All scenes live in the periodic unit box, total mass 1 (each particle 1/N),
Newtonian G = 1. Positions and velocities are float32 ``(n, 4)`` arrays; ``w``
of pos is 0 (gas) and ``w`` of vel is 0, as the reference's plain particles.

* ``disk_galaxy``: 80 % exponential disk (scale length 0.08, sech^2 scale height
  0.008), circular velocity from the enclosed mass plus 5 % Gaussian dispersion;
  20 % Plummer bulge (a = 0.03) with isotropic Jeans dispersion.
* ``two_galaxies``: two such galaxies on a parabolic orbit (separation 0.4,
  pericentre 0.1), disks inclined +30 and -60 degrees.
* ``zeldovich``: particles on an n^3 lattice displaced by the Zel'dovich
  approximation from a Gaussian field with P(k) ~ k^-2 cut at the lattice
  Nyquist frequency, rms displacement 0.5 lattice cell, velocities of the
  growing mode of a static periodic background (v = sqrt(4 pi G rho) psi).
"""
from __future__ import annotations

import numpy as np

TWO_PI = 2.0 * np.pi


def _pack(xyz: np.ndarray, v: np.ndarray):
    n = len(xyz)
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros((n, 4), np.float32)
    pos[:, :3] = np.mod(xyz, 1.0)
    # p - floor(p) can round up to exactly 1.0 in float32; keep [0, 1)
    pos[:, :3][pos[:, :3] >= 1.0] = 0.0
    vel[:, :3] = v
    return pos, vel


def _enclosed_mass(r: np.ndarray, m_each: float) -> np.ndarray:
    order = np.argsort(r, kind="stable")
    m = np.empty_like(r)
    m[order] = (np.arange(1, len(r) + 1, dtype=np.float64)) * m_each
    return m


def _rotation(incl_deg: float) -> np.ndarray:
    a = np.deg2rad(incl_deg)
    return np.array([[1.0, 0.0, 0.0], [0.0, np.cos(a), -np.sin(a)], [0.0, np.sin(a), np.cos(a)]])


def galaxy_particles(n: int, rng: np.random.Generator, mass: float = 1.0, G: float = 1.0,
                     disk_frac: float = 0.8, r_d: float = 0.08, h_z: float = 0.008, bulge_a: float = 0.03,
                     dispersion: float = 0.05, r_max: float = 0.3):
    """Relative positions and velocities of one disk + bulge galaxy (float64)."""
    n_disk = int(round(n * disk_frac))
    n_bulge = n - n_disk
    # disk: R ~ Gamma(2, r_d) (surface density exp(-R/r_d)), truncated at r_max by resampling
    R = rng.gamma(2.0, r_d, n_disk)
    bad = R > r_max
    while bad.any():
        R[bad] = rng.gamma(2.0, r_d, int(bad.sum()))
        bad = R > r_max
    th = rng.uniform(0.0, TWO_PI, n_disk)
    z = h_z * np.arctanh(np.clip(rng.uniform(-1.0, 1.0, n_disk), -0.999999, 0.999999))
    disk = np.stack([R * np.cos(th), R * np.sin(th), z], axis=1)
    # bulge: Plummer radius from the inverse CDF, truncated at r_max
    u = rng.uniform(1e-6, 1.0, n_bulge)
    rb = bulge_a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
    bad = rb > r_max
    while bad.any():
        uu = rng.uniform(1e-6, 1.0, int(bad.sum()))
        rb[bad] = bulge_a / np.sqrt(uu ** (-2.0 / 3.0) - 1.0)
        bad = rb > r_max
    dirs = rng.normal(size=(n_bulge, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    bulge = dirs * rb[:, None]
    xyz = np.concatenate([disk, bulge], axis=0)
    m_each = mass / n
    r = np.linalg.norm(xyz, axis=1)
    menc = _enclosed_mass(r, m_each)
    v = np.zeros_like(xyz)
    # disk: circular velocity from the spherical enclosed mass, 5 % dispersion
    rd = np.maximum(r[:n_disk], 1e-4)
    vc = np.sqrt(G * menc[:n_disk] / rd)
    tang = np.stack([-np.sin(th), np.cos(th), np.zeros(n_disk)], axis=1)
    v[:n_disk] = tang * vc[:, None] + rng.normal(size=(n_disk, 3)) * (dispersion * vc)[:, None]
    # bulge: isotropic Plummer Jeans dispersion sigma^2 = G M_b / (6 sqrt(r^2 + a^2)) + disk pull
    m_b = mass * (1.0 - disk_frac)
    sig = np.sqrt(G * m_b / (6.0 * np.sqrt(rb ** 2 + bulge_a ** 2)) + G * menc[n_disk:] / (6.0 * np.maximum(rb, bulge_a)))
    v[n_disk:] = rng.normal(size=(n_bulge, 3)) * sig[:, None]
    return xyz, v


def disk_galaxy(n: int = 262_144, seed: int = 0):
    """A single disk galaxy at the box centre, total mass 1."""
    rng = np.random.default_rng(seed)
    xyz, v = galaxy_particles(n, rng)
    v -= v.mean(axis=0)
    return _pack(xyz + 0.5, v)


def two_galaxies(n: int = 4_194_304, seed: int = 1, separation: float = 0.4, pericentre: float = 0.1,
                 incl=(30.0, -60.0)):
    """Two equal galaxies on a parabolic orbit (each half the mass)."""
    rng = np.random.default_rng(seed)
    n1 = n // 2
    n2 = n - n1
    G, M = 1.0, 1.0
    # parabolic relative orbit: v^2 = 2 G M / r, specific angular momentum sqrt(2 G M q)
    v_rel = np.sqrt(2.0 * G * M / separation)
    v_t = np.sqrt(2.0 * G * M * pericentre) / separation
    v_r = -np.sqrt(max(v_rel ** 2 - v_t ** 2, 0.0))
    rel_x = np.array([separation, 0.0, 0.0])
    rel_v = np.array([v_r, v_t, 0.0])
    parts = []
    for k, (nk, inc) in enumerate(((n1, incl[0]), (n2, incl[1]))):
        xyz, v = galaxy_particles(nk, rng, mass=0.5 * nk / (0.5 * n))
        Rm = _rotation(inc)
        xyz = xyz @ Rm.T
        v = v @ Rm.T
        sgn = 0.5 if k == 0 else -0.5
        parts.append((xyz + 0.5 + sgn * rel_x, v + sgn * rel_v))
    xyz = np.concatenate([p[0] for p in parts])
    v = np.concatenate([p[1] for p in parts])
    v -= v.mean(axis=0)
    return _pack(xyz, v)


def zeldovich(n_side: int = 256, seed: int = 2, rms_cells: float = 0.5, G: float = 1.0):
    """n_side^3 particles displaced from a lattice by the Zel'dovich approximation."""
    rng = np.random.default_rng(seed)
    n = n_side
    kf = np.fft.fftfreq(n, d=1.0 / n).astype(np.float32)
    kr = np.arange(n // 2 + 1, dtype=np.float32)
    white = rng.standard_normal((n, n, n), dtype=np.float32)
    wk = np.fft.rfftn(white).astype(np.complex64)
    del white
    kz = kf[:, None, None]
    ky = kf[None, :, None]
    kx = kr[None, None, :]
    k2 = kz * kz + ky * ky + kx * kx
    k2[0, 0, 0] = 1.0
    # delta_k = sqrt(P(k)) * white_k,  P ~ k^-2, cut at the lattice Nyquist (|k_i| <= n/2)
    amp = (1.0 / np.sqrt(k2)).astype(np.float32)
    amp[0, 0, 0] = 0.0
    delta = wk * amp
    del wk, amp
    # psi_k = i k / k^2 delta_k  (so that div psi = -delta)
    psi = np.empty((n, n, n, 3), np.float32)
    for j, kk in enumerate((kx, ky, kz)):
        comp = (1j * (kk / k2) * delta).astype(np.complex64)
        psi[..., j] = np.fft.irfftn(comp, s=(n, n, n), axes=(0, 1, 2)).astype(np.float32)
        del comp
    del delta
    rms = float(np.sqrt(np.mean(np.sum(psi.astype(np.float64) ** 2, axis=-1))))
    psi *= np.float32(rms_cells / n / rms)
    q = (np.arange(n, dtype=np.float32) + 0.5) / n
    zz, yy, xx = np.meshgrid(q, q, q, indexing="ij")
    lattice = np.stack([xx, yy, zz], axis=-1)
    xyz = (lattice + psi).reshape(-1, 3).astype(np.float64)
    # growing mode of a static background with mean density 1: rate sqrt(4 pi G rho)
    v = psi.reshape(-1, 3).astype(np.float64) * np.sqrt(4.0 * np.pi * G)
    return _pack(xyz, v)


def ensemble_members(count: int = 64, seed: int = 4, n_min: int = 16_384, n_max: int = 1_048_576):
    """Recipes of the batched ensemble: per scene (kind, n, grid, seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
        kind = "disk" if rng.integers(0, 2) == 0 else "zeldovich"
        if kind == "zeldovich":
            side = max(8, int(round(n ** (1.0 / 3.0))))
            n = side ** 3
        grid = 32 if n < 65_536 else (64 if n < 524_288 else 128)
        out.append({"kind": kind, "n": n, "grid": grid, "seed": int(seed * 1000 + i)})
    return out


def make_member(m: dict):
    if m["kind"] == "disk":
        return disk_galaxy(m["n"], m["seed"])
    side = int(round(m["n"] ** (1.0 / 3.0)))
    return zeldovich(side, m["seed"])


def workload(name: str):
    """Named benchmark workloads: (pos, vel, grid, dt, steps)."""
    if name == "disk_64":
        p, v = disk_galaxy(262_144, 0)
        return p, v, 64, 1e-3, 10
    if name == "two_galaxy_256":
        p, v = two_galaxies(4_194_304, 1)
        return p, v, 256, 5e-4, 100
    if name == "cosmic_web_512":
        p, v = zeldovich(256, 2)
        return p, v, 512, 1e-3, 50
    if name == "learned_128":
        p, v = zeldovich(128, 3)
        return p, v, 128, 1e-3, 10
    raise KeyError(name)
