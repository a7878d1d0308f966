"""Run a few PM steps (or one stage) for profiling with an external profiler.

    python -m stardust_b200.profile --workload cosmic_web_512 --steps 2
    python -m stardust_b200.profile --stage poisson --grid 512
    python -m stardust_b200.profile --stage mlp --steps 3
    python -m stardust_b200.profile --workload zeldovich --lattice 128 --grid 512 --order 0

--stage mlp runs the learned correction's inference (sd_mlp_infer) on the
learned configuration's scene: 2,097,152 particles (Zel'dovich field, 128^3
lattice, seed 1) on a 128^3 grid, random weights.

Steps run eagerly (no CUDA graph) so each kernel appears as its own launch.
Prints per-phase device times of the last step.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import sys

import numpy as np


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="cosmic_web_512")
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--stage", choices=["step", "poisson", "mlp"], default="step")
    ap.add_argument("--grid", type=int, default=512)
    ap.add_argument("--order", type=int, default=2)
    ap.add_argument("--lattice", type=int, default=0,
                    help="with --workload zeldovich: the Zel'dovich field on this lattice (seed 2) on --grid")
    a = ap.parse_args(argv)

    import torch

    from . import _lib as L
    from . import scenes
    from .sim import Sim, SimConfig

    if a.stage == "poisson":
        G = a.grid
        rng = np.random.default_rng(0)
        rho = torch.from_numpy(rng.random((G, G, G), dtype=np.float32)).cuda()
        phi = torch.empty_like(rho)
        lib = L.lib()
        ws = torch.empty(int(lib.sd_poisson_workspace_bytes(G)), dtype=torch.uint8, device="cuda")
        for _ in range(max(1, a.steps)):
            L.check(lib.sd_poisson(rho.data_ptr(), G, ctypes.c_float(1.0), phi.data_ptr(), ws.data_ptr(),
                                   ws.numel(), None), "sd_poisson")
        torch.cuda.synchronize()
        print(json.dumps({"stage": "poisson", "grid": G}))
        return 0

    if a.stage == "mlp":
        pos, _ = scenes.zeldovich(128, 1)
        n, G = len(pos), 128
        rng = np.random.default_rng(0)
        rho = torch.from_numpy(rng.random(G ** 3, dtype=np.float32) * 3).cuda()
        params = torch.from_numpy((rng.standard_normal(int(L.lib().sd_mlp_param_count())) * 0.2).astype(np.float32)).cuda()
        pd = torch.from_numpy(pos).cuda()
        out = torch.empty((n, 4), dtype=torch.float32, device="cuda")
        for _ in range(max(1, a.steps)):
            L.check(L.lib().sd_mlp_infer(params.data_ptr(), pd.data_ptr(), None, n, rho.data_ptr(), G,
                                         ctypes.c_float(1.0), ctypes.c_float(1.0), out.data_ptr(), None),
                    "sd_mlp_infer")
        torch.cuda.synchronize()
        print(json.dumps({"stage": "mlp", "particles": n, "grid": G,
                          "wait_timeouts": int(L.lib().sd_mlp_wait_timeouts())}))
        return 0

    if a.workload == "zeldovich":
        pos, vel = scenes.zeldovich(a.lattice or 128, 2)
        G, dt = a.grid, 1e-3
    elif a.workload == "cosmic_web_512":
        pos, vel = scenes.zeldovich(256, 2)
        G, dt = 512, 1e-3
    elif a.workload == "two_galaxy_256":
        pos, vel = scenes.two_galaxies(4_194_304, 1)
        G, dt = 256, 5e-4
    else:
        pos, vel = scenes.disk_galaxy(262_144, 0)
        G, dt = 64, 1e-3
    with Sim(0) as s:
        s.init(SimConfig(particle_count=len(pos), grid_size=G, gravity=1.0, units=L.SD_UNITS_NEWTON,
                         softening_cells=1.0, order=a.order, keep_density=0))
        s.set_particles(pos, vel)
        for _ in range(a.steps):
            s.step(dt)
        print(json.dumps(s.timings()))
    return 0


if __name__ == "__main__":
    sys.exit(main())
