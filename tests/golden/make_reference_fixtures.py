"""Generate golden fixtures by running the unmodified reference on a GPU.

Usage (on a machine with a CUDA GPU and the prebuilt oracle/_ref/libsimref.so):
    python tests/golden/make_reference_fixtures.py OUTDIR [CASE ...]

With CASE names, only those cases are written (e.g. ``disk_g64 fields_g32``).
``reference_disk_g64.npz`` holds no inputs: the test rebuilds them from the seeded
scene and checks them against the stored digest. ``reference_fields_g32.npz`` holds
the screen grids of Sim::fieldDevicePtr (density projection, velocity dispersion).

For each step case it writes ``reference_<name>.npz`` holding the seeded input
particles, the reference's density after Sim::loadState (deposit of the loaded
positions), and the particles after one Sim::step() (sort + deposit + cuFFT
Poisson + gradient + kick/drift + momentum zeroing). Velocities carry a particle
id in ``w`` (the reference copies w through the sort and the integrator), so the
reference's sort permutation can be read back. For each preset case it writes
``reference_preset_<name>.npz``: the particles Sim::init lays down (reset():
kPlace, spin, Hubble flow, dispersion, centre-of-mass stop) for the given
settings. The cases are small so the committed files stay small.
"""
from __future__ import annotations

import ctypes
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from stardust_b200 import scenes  # noqa: E402

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libsimref.so")


def load_ref():
    L = ctypes.CDLL(REF_LIB)
    P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    L.ref_create.restype = P
    L.ref_destroy.argtypes = [P]
    L.ref_load.argtypes = [P, P, P, I, I, F, F, F, I, ctypes.c_char_p]
    L.ref_load_b.argtypes = [P, P, P, I, I, F, F, F, I, I, ctypes.c_char_p]
    L.ref_step.argtypes = [P]
    L.ref_steps.argtypes = [P, I]
    L.ref_get.argtypes = [P, P, P, I]
    L.ref_density.argtypes = [P, P, I]
    L.ref_timings.argtypes = [P, P]
    L.ref_init_preset.argtypes = [P, I, I, I, I, F, F, F, F, F]
    L.ref_set_hydro.argtypes = [P, I, F, I, F]
    L.ref_fail_message.restype = ctypes.c_char_p
    L.ref_sim_time.argtypes = [P]
    L.ref_sim_time.restype = ctypes.c_double
    return L


def run_case(L, pos, vel, G, gravity, soft, dt, tmpdir, boundary=1):
    """boundary: 1 periodic, 0 isolated (Sim.h's Boundary enum)."""
    n = len(pos)
    h = L.ref_create()
    try:
        path = os.path.join(tmpdir, "in.stardust").encode()
        # timeScale = dt / 0.0016 gives dt = 0.0016 * dtScaleFor(timeScale) (Sim.h:89-93)
        ts = np.float32(dt) / np.float32(0.0016)
        rc = L.ref_load_b(h, pos.ctypes.data, vel.ctypes.data, n, G, gravity, soft, float(ts), 1, boundary, path)
        if rc != 0:
            raise RuntimeError(f"ref_load failed: {rc} {L.ref_fail_message()}")
        side = G if boundary == 1 else 2 * G  # the isolated density lives in the 2G box
        rho = np.empty(side ** 3, np.float32)
        L.ref_density(h, rho.ctypes.data, side)
        rho = rho.reshape(side, side, side)[:G, :G, :G].copy()
        rc = L.ref_step(h)
        if rc != 0:
            raise RuntimeError(f"ref_step failed: {L.ref_fail_message()}")
        p1 = np.empty_like(pos)
        v1 = np.empty_like(vel)
        L.ref_get(h, p1.ctypes.data, v1.ctypes.data, n)
        t = np.empty(6, np.float32)
        L.ref_timings(h, t.ctypes.data)
        return rho, p1, v1, float(t[4])
    finally:
        L.ref_destroy(h)


def cases():
    rng = np.random.default_rng(20240)
    n = 4096
    c = rng.random((6, 3))
    xyz = (c[rng.integers(0, 6, n)] + rng.normal(scale=0.05, size=(n, 3))) % 1.0
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = xyz
    pos[:, :3][pos[:, :3] >= 1.0] = 0.0
    vel = np.zeros((n, 4), np.float32)
    vel[:, :3] = rng.normal(scale=0.2, size=(n, 3))
    yield "clustered_g16", pos, vel, 16, float(4 * np.pi * 16 ** 3), 1.0, 1e-3, 1
    p, v = scenes.disk_galaxy(8192, 7)
    yield "disk_g32", p, v, 32, float(4 * np.pi * 32 ** 3), 1.0, 1e-3, 1
    # isolated boundary (the reference's default): a disk galaxy, a few particles
    # against the walls moving into them; gravity G = Newton's G = 1 for -1/r in cells
    p, v = scenes.disk_galaxy(8192, 11)
    p[:4, 0] = [0.0015, 0.0025, 0.9975, 0.9985]
    v[:4, 0] = [-1.0, -2.0, 2.0, 1.0]
    yield "isolated_g32", p, v, 32, 32.0, 1.5, 1e-3, 0


def hydro_cases():
    """Steps with pressure and cooling on: name, particles, grid, gravity, softening,
    dt, steps, pressure_k, cooling_rate."""
    rng = np.random.default_rng(777)
    n = 6000
    c = rng.random((5, 3))
    xyz = (c[rng.integers(0, 5, n)] + rng.normal(scale=0.06, size=(n, 3))) % 1.0
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = xyz
    pos[:, :3][pos[:, :3] >= 1.0] = 0.0
    vel = np.zeros((n, 4), np.float32)
    vel[:, :3] = rng.normal(scale=0.3, size=(n, 3))
    yield "hydro_g16", pos, vel, 16, float(4 * np.pi * 16 ** 3), 1.0, 1e-3, 3, 0.45, 0.08


def preset_cases():
    # name, n, G, preset, dark fraction, shrink, spin, hubble, dispersion
    yield "filament_all", 6000, 32, 0, 0.25, 0.9, 0.7, 0.4, 0.05
    yield "filament_plain", 4096, 16, 0, 0.0, 0.0, 0.0, 0.0, 0.0
    yield "empty_dark", 3000, 16, 1, 0.3, 0.0, 0.5, 0.0, 0.1


def compact_step_cases():
    """Steps stored without their inputs, which the test regenerates from the same
    seeded scene: name, (scene kind, n, seed), grid, gravity, softening, dt, sampled
    output slots."""
    yield "disk_g64", ("disk", 262_144, 0), 64, float(4 * np.pi * 64 ** 3), 1.0, 1e-3, 16384


def scene_inputs(kind, n, seed):
    p, v = scenes.disk_galaxy(n, seed) if kind == "disk" else scenes.two_galaxies(n, seed)
    p = np.ascontiguousarray(p, np.float32)
    v = np.ascontiguousarray(v, np.float32)
    v[:, 3] = np.arange(n, dtype=np.float32)  # ids through the reference's sort
    return p, v


def input_digest(pos, vel) -> str:
    import hashlib

    return hashlib.sha256(pos.tobytes() + vel.tobytes()).hexdigest()


def field_cases():
    """Screen grids of Sim::fieldDevicePtr: name, (scene kind, n, seed), grid, view rotation."""
    c, s_ = np.cos(0.6), np.sin(0.6)
    rx = np.array([[1, 0, 0], [0, c, -s_], [0, s_, c]])
    ry = np.array([[np.cos(0.35), 0, np.sin(0.35)], [0, 1, 0], [-np.sin(0.35), 0, np.cos(0.35)]])
    rot = (ry @ rx).astype(np.float32).reshape(9)
    yield "fields_g32", ("disk", 8192, 13), 32, rot


def main(outdir: str, only=()) -> int:
    os.makedirs(outdir, exist_ok=True)
    L = load_ref()
    L.ref_field.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]

    def want(name):
        return not only or name in only

    with tempfile.TemporaryDirectory() as tmp:
        for name, (kind, n, seed), G, grav, soft, dt, sample in compact_step_cases():
            if not want(name):
                continue
            pos, vel = scene_inputs(kind, n, seed)
            rho, p1, v1, dt_used = run_case(L, pos, vel, G, grav, soft, dt, tmp)
            slots = np.sort(np.random.default_rng(5).choice(n, sample, replace=False)).astype(np.int32)
            np.savez_compressed(os.path.join(outdir, f"reference_{name}.npz"), scene=np.array([kind]), n=n, seed=seed,
                                digest=np.array([input_digest(pos, vel)]), rho_loaded=rho,
                                ids_out=v1[:, 3].astype(np.int32), slots=slots, pos_out=p1[slots], vel_out=v1[slots],
                                grid=G, gravity=grav, soft=soft, dt=np.float32(dt_used))
            print(name, "dt_used", dt_used, "mass", float(rho.sum()))
        for name, (kind, n, seed), G, rot in field_cases():
            if not want(name):
                continue
            pos, vel = scene_inputs(kind, n, seed)
            h = L.ref_create()
            try:
                path = os.path.join(tmp, "f.stardust").encode()
                if L.ref_load(h, pos.ctypes.data, vel.ctypes.data, n, G, 1.0, 1.0, 1.0, 1, path) != 0:
                    raise RuntimeError(f"ref_load failed: {L.ref_fail_message()}")
                rho = np.empty(G ** 3, np.float32)
                L.ref_density(h, rho.ctypes.data, G)
                grids = {}
                for field, fname in ((0, "density"), (1, "dispersion")):
                    for r, rname in ((None, "top"), (rot, "rot")):
                        out = np.empty(G * G, np.float32)
                        rp = None if r is None else np.ascontiguousarray(r, np.float32)
                        if L.ref_field(h, field, None if rp is None else rp.ctypes.data, out.ctypes.data, G) != 0:
                            raise RuntimeError(f"ref_field failed: {L.ref_fail_message()}")
                        grids[f"{fname}_{rname}"] = out.reshape(G, G)
            finally:
                L.ref_destroy(h)
            np.savez_compressed(os.path.join(outdir, f"reference_{name}.npz"), pos=pos, vel=vel, grid=G, rot=rot,
                                rho_loaded=rho.reshape(G, G, G), **grids)
            print(name, {k: float(v.sum()) for k, v in grids.items()})
    if only:
        return 0
    for name, pos, vel, G, grav, soft, dt, steps, pk, rate in hydro_cases():
        pos = np.ascontiguousarray(pos, np.float32)
        vel = np.ascontiguousarray(vel, np.float32)
        vel[:, 3] = np.arange(len(vel), dtype=np.float32)  # ids (>= 0: gas, not dark matter)
        n = len(pos)
        h = L.ref_create()
        try:
            with tempfile.TemporaryDirectory() as tmp:
                path = os.path.join(tmp, "in.stardust").encode()
                ts = np.float32(dt) / np.float32(0.0016)
                if L.ref_load_b(h, pos.ctypes.data, vel.ctypes.data, n, G, grav, soft, float(ts), 1, 1, path) != 0:
                    raise RuntimeError(f"ref_load failed: {L.ref_fail_message()}")
            if L.ref_set_hydro(h, 1, pk, 1, rate) != 0:
                raise RuntimeError(f"ref_set_hydro failed: {L.ref_fail_message()}")
            ps, vs, dts = [], [], []
            for _ in range(steps):
                if L.ref_step(h) != 0:
                    raise RuntimeError(f"ref_step failed: {L.ref_fail_message()}")
                p1, v1 = np.empty_like(pos), np.empty_like(vel)
                L.ref_get(h, p1.ctypes.data, v1.ctypes.data, n)
                t = np.empty(6, np.float32)
                L.ref_timings(h, t.ctypes.data)
                ps.append(p1)
                vs.append(v1)
                dts.append(t[4])
        finally:
            L.ref_destroy(h)
        np.savez_compressed(os.path.join(outdir, f"reference_{name}.npz"), pos_in=pos, vel_in=vel,
                            pos_steps=np.stack(ps), vel_steps=np.stack(vs), dt_used=np.array(dts, np.float32),
                            grid=G, gravity=grav, soft=soft, pressure_k=np.float32(pk), cooling_rate=np.float32(rate))
        print(name, "dt_used", dts)
    for name, n, G, preset, dark, shrink, spin, hubble, disp in preset_cases():
        h = L.ref_create()
        try:
            rc = L.ref_init_preset(h, n, G, 1, preset, dark, shrink, spin, hubble, disp)
            if rc != 0:
                raise RuntimeError(f"ref_init_preset failed: {rc} {L.ref_fail_message()}")
            p = np.empty((n, 4), np.float32)
            v = np.empty((n, 4), np.float32)
            L.ref_get(h, p.ctypes.data, v.ctypes.data, n)
        finally:
            L.ref_destroy(h)
        np.savez_compressed(os.path.join(outdir, f"reference_preset_{name}.npz"), pos=p, vel=v, n=n, grid=G,
                            preset=preset, dark_matter_fraction=np.float32(dark), big_bang_shrink=np.float32(shrink),
                            spin=np.float32(spin), hubble=np.float32(hubble), vel_dispersion=np.float32(disp))
        print(name, "live", int((p[:, 0] >= 0).sum()), "dark", int((v[:, 3] == -100).sum()))
    with tempfile.TemporaryDirectory() as tmp:
        for name, pos, vel, G, grav, soft, dt, boundary in cases():
            pos = np.ascontiguousarray(pos, np.float32)
            vel = np.ascontiguousarray(vel, np.float32)
            vel[:, 3] = np.arange(len(vel), dtype=np.float32)  # id through the reference's sort
            rho, p1, v1, dt_used = run_case(L, pos, vel, G, grav, soft, dt, tmp, boundary)
            np.savez_compressed(os.path.join(outdir, f"reference_{name}.npz"), pos_in=pos, vel_in=vel,
                                rho_loaded=rho, pos_out=p1, vel_out=v1, grid=G, gravity=grav, soft=soft,
                                dt=np.float32(dt_used), boundary=boundary)
            print(name, "dt_used", dt_used, "mass", float(rho.sum()))
    return 0


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit(__doc__)
    sys.exit(main(sys.argv[1], tuple(sys.argv[2:])))
