"""Batched ensemble: many independent scenes advanced together, one CUDA graph
launch per step (sd_ensemble_*). The reference has no counterpart: it runs one
``Sim`` per scene.

Each scene is a full simulation handle owned by the ensemble; ``scene(i)``
returns a ``Sim`` view of it, so every per-scene query (particles, density,
accelerations, state files) works unchanged. ``autotune`` picks, per scene, the
deposit path and gather grid that run fastest on this GPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from .sim import Sim, SimConfig, _host_f4


class _SceneView(Sim):
    """A Sim over a handle the ensemble owns (never destroyed from here)."""

    def __init__(self, handle: int, device: int):
        self._h = ctypes.c_void_p(handle)
        self.device = device

    def close(self) -> None:
        self._h = ctypes.c_void_p()


class Ensemble:
    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        L.check(L.lib().sd_ensemble_create(ctypes.byref(self._h), device), "sd_ensemble_create")
        self.device = device

    def close(self) -> None:
        if self._h:
            L.lib().sd_ensemble_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add(self, cfg: SimConfig, pos, vel) -> int:
        """Add a scene with its initial particles; returns its index."""
        c = cfg.to_c()
        if hasattr(pos, "is_cuda") and pos.is_cuda:
            rc = L.lib().sd_ensemble_add(self._h, ctypes.byref(c), pos.data_ptr(), vel.data_ptr(),
                                         int(pos.shape[0]), L.SD_DEVICE)
        else:
            p, v = _host_f4(pos), _host_f4(vel)
            rc = L.lib().sd_ensemble_add(self._h, ctypes.byref(c), p.ctypes.data, v.ctypes.data, len(p), L.SD_HOST)
        if rc < 0:
            L.check(rc, "sd_ensemble_add")
        return rc

    def __len__(self) -> int:
        return int(L.lib().sd_ensemble_size(self._h))

    def scene(self, i: int) -> Sim:
        h = L.lib().sd_ensemble_scene(self._h, i)
        if not h:
            raise IndexError(i)
        return _SceneView(h, self.device)

    def autotune(self, dt: float, reps: int = 3) -> list[dict]:
        L.check(L.lib().sd_ensemble_autotune(self._h, float(dt), int(reps)), "sd_ensemble_autotune")
        return [self.tuning(i) for i in range(len(self))]

    def tuning(self, i: int) -> dict:
        t = L.SdSceneTuning()
        L.check(L.lib().sd_ensemble_get_tuning(self._h, i, ctypes.byref(t)), "sd_ensemble_get_tuning")
        return {"order": ["rowmajor", "morton", "tiled"][t.order], "gather_blocks": t.gather_blocks,
                "step_ms": t.step_ms, "deposit_split": t.deposit_split}

    def steps(self, dt: float, n: int) -> None:
        L.check(L.lib().sd_ensemble_steps(self._h, float(dt), int(n)), "sd_ensemble_steps")

    def synchronize(self) -> None:
        L.check(L.lib().sd_ensemble_synchronize(self._h), "sd_ensemble_synchronize")

    @property
    def stream_handle(self) -> int:
        return int(L.lib().sd_ensemble_stream(self._h) or 0)

    def graph_kernels(self) -> int:
        return int(L.lib().sd_ensemble_graph_kernels(self._h))


def member_config(m: dict, softening_cells: float = 1.0, keep_density: int = 0) -> SimConfig:
    """Newtonian periodic configuration of one ensemble member recipe."""
    return SimConfig(particle_count=m["n"], grid_size=m["grid"], gravity=1.0, softening_cells=softening_cells,
                     units=L.SD_UNITS_NEWTON, order=L.SD_ORDER_TILED, sort_interval=1, keep_density=keep_density)


def partition(members: list[dict], ranks: int) -> list[list[int]]:
    """Longest-processing-time assignment of scenes to ranks, cost ~ bytes of a
    step (184 N + 40 G^3): each scene goes to the least-loaded rank."""
    order = sorted(range(len(members)), key=lambda i: -(184 * members[i]["n"] + 40 * members[i]["grid"] ** 3))
    load = [0.0] * ranks
    out: list[list[int]] = [[] for _ in range(ranks)]
    for i in order:
        r = int(np.argmin(load))
        out[r].append(i)
        load[r] += 184 * members[i]["n"] + 40 * members[i]["grid"] ** 3
    return [sorted(o) for o in out]
