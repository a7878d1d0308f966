"""Python mirror of the reference's ``Sim`` class over the C ABI.

Method names follow the reference (src/sim/Sim.h:854-1135), in snake_case:
``init``, ``reconfigure``, ``reset``, ``step``, ``timings``, ``sim_time``,
``grid_size``, ``particle_count``, ``active_count``, ``save_state``,
``load_state``, ``measure_total_grid_mass`` ... plus ``step(dt)`` with an explicit
time step and ``set_particles`` / ``get_particles`` for scene init. Errors raise
``SdError`` carrying the library's status code and first-failure message (the
reference's sticky ``Sim::failed()`` / ``failMessage()``, Sim.cu:52-75).

Particle arrays are float32 ``(n, 4)``: host numpy arrays, or CUDA torch tensors
(passed by device pointer, no host copy).
"""
from __future__ import annotations

import ctypes
from dataclasses import asdict, dataclass, fields

import numpy as np

from . import _lib as L


@dataclass
class SimConfig:
    """Plain-PM fields of the reference's SimConfig (Sim.h:157-796)."""

    particle_count: int = 2_000_000      # Sim.h:166
    grid_size: int = 128                 # Sim.h:167
    boundary: int = L.SD_BOUNDARY_PERIODIC
    gravity: float = 1.0                 # Sim.h:280
    softening_cells: float = 3.0         # Sim.h:315
    time_scale: float = 1.0              # Sim.h:316
    sort_interval: int = 1               # Sim.h:317
    length_scale: float = 1.0            # Sim.h:172
    time_unit_scale: float = 1.0         # Sim.h:180
    order: int = L.SD_ORDER_ROWMAJOR
    integrator: int = L.SD_INT_KD
    units: int = L.SD_UNITS_REFERENCE
    diagnostics: int = 0
    keep_density: int = 1
    # initial conditions of init / reset (Sim::reset, Sim.cu:4160-4238)
    preset: int = L.SD_PRESET_FILAMENT   # Sim.h:277
    dark_matter_fraction: float = 0.0    # Sim.h:536
    big_bang_shrink: float = 0.0         # Sim.h:214
    spin: float = 0.0                    # Sim.h:766
    hubble: float = 0.0                  # Sim.h:196
    vel_dispersion: float = 0.0          # Sim.h:263
    # grid hydrodynamics add-ons (off unless set; the reference's defaults are on)
    pressure_enabled: int = 0            # Sim.h:319
    pressure_k: float = 0.45             # Sim.h:320
    cooling_enabled: int = 0             # Sim.h:327
    cooling_rate: float = 0.08           # Sim.h:345
    full_sort: int = 0                   # 1: always the full sort; 0: merge when worthwhile; -1: merge always

    def to_c(self) -> L.SdConfig:
        c = L.SdConfig()
        for f in fields(self):
            setattr(c, f.name, getattr(self, f.name))
        return c

    @classmethod
    def from_c(cls, c: L.SdConfig) -> "SimConfig":
        return cls(**{f.name: getattr(c, f.name) for f in fields(cls)})

    def as_dict(self) -> dict:
        return asdict(self)


def _is_torch_cuda(a) -> bool:
    return hasattr(a, "is_cuda") and bool(a.is_cuda)


def _host_f4(a) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    if a.ndim != 2 or a.shape[1] != 4:
        raise ValueError("particle arrays must be float32 of shape (n, 4)")
    return a


class Sim:
    """One PM simulation on one GPU (the reference's Sim, Sim.h:854)."""

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        L.check(L.lib().sd_create(ctypes.byref(self._h), device), "sd_create")
        self.device = device

    # ---- lifetime ------------------------------------------------------------
    def close(self) -> None:
        if self._h:
            L.lib().sd_destroy(self._h)
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

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def set_stream(self, stream) -> None:
        """Run this simulation's work on ``stream`` (a CUDA stream handle as an
        int, or a torch stream), so that it is ordered with other work there."""
        ptr = getattr(stream, "cuda_stream", stream)
        L.check(L.lib().sd_set_stream(self._h, ctypes.c_void_p(int(ptr))), "sd_set_stream")

    # ---- static queries --------------------------------------------------------
    @staticmethod
    def device_available() -> bool:
        return bool(L.lib().sd_device_available())

    @staticmethod
    def failed() -> bool:
        return bool(L.lib().sd_failed())

    @staticmethod
    def fail_message() -> str:
        return L.last_error()

    @staticmethod
    def max_grid_size(boundary: int = L.SD_BOUNDARY_PERIODIC) -> int:
        return int(L.lib().sd_max_grid_size(boundary))

    @staticmethod
    def estimate_bytes(particle_count: int, grid_size: int, boundary: int = L.SD_BOUNDARY_PERIODIC) -> int:
        return int(L.lib().sd_estimate_bytes(particle_count, grid_size, boundary))

    @staticmethod
    def max_particles_for(grid_size: int, boundary: int, free_bytes: int) -> int:
        """Sim::maxParticlesFor (Sim.cu:4057-4066)."""
        return int(L.lib().sd_max_particles_for(grid_size, boundary, free_bytes))

    @staticmethod
    def estimate_step_ms(particle_count: int, grid_size: int, boundary: int = L.SD_BOUNDARY_PERIODIC) -> float:
        """Sim::estimateStepMs (Sim.cu:4022-4055); 0 without a device."""
        return float(L.lib().sd_estimate_step_ms(particle_count, grid_size, boundary))

    @staticmethod
    def device_free_bytes() -> int:
        return int(L.lib().sd_device_free_bytes())

    @staticmethod
    def device_bandwidth_gbs() -> float:
        return float(L.lib().sd_device_bandwidth_gbs())

    @staticmethod
    def device_multiprocessors() -> int:
        return int(L.lib().sd_device_multiprocessors())

    @staticmethod
    def device_name() -> str:
        buf = ctypes.create_string_buffer(256)
        L.check(L.lib().sd_device_name(buf, 256), "sd_device_name")
        return buf.value.decode()

    @staticmethod
    def device_driver() -> str:
        buf = ctypes.create_string_buffer(64)
        L.check(L.lib().sd_device_driver(buf, 64), "sd_device_driver")
        return buf.value.decode()

    # ---- configuration -----------------------------------------------------------
    def init(self, cfg: SimConfig) -> None:
        c = cfg.to_c()
        L.check(L.lib().sd_init(self._h, ctypes.byref(c)), "sd_init")

    def reconfigure(self, cfg: SimConfig) -> None:
        c = cfg.to_c()
        L.check(L.lib().sd_reconfigure(self._h, ctypes.byref(c)), "sd_reconfigure")

    def reset(self) -> None:
        L.check(L.lib().sd_reset(self._h), "sd_reset")

    def config(self) -> SimConfig:
        c = L.SdConfig()
        L.check(L.lib().sd_get_config(self._h, ctypes.byref(c)), "sd_get_config")
        return SimConfig.from_c(c)

    # ---- particles --------------------------------------------------------------
    def set_particles(self, pos, vel) -> None:
        if _is_torch_cuda(pos):
            n = int(pos.shape[0])
            L.check(L.lib().sd_set_particles(self._h, pos.data_ptr(), vel.data_ptr(), n, L.SD_DEVICE),
                    "sd_set_particles")
            return
        p, v = _host_f4(pos), _host_f4(vel)
        L.check(L.lib().sd_set_particles(self._h, p.ctypes.data, v.ctypes.data, len(p), L.SD_HOST),
                "sd_set_particles")

    def get_particles(self, n: int | None = None):
        n = self.particle_count() if n is None else n
        p = np.empty((n, 4), np.float32)
        v = np.empty((n, 4), np.float32)
        L.check(L.lib().sd_get_particles(self._h, p.ctypes.data, v.ctypes.data, n, L.SD_HOST), "sd_get_particles")
        return p, v

    def get_particles_into(self, pos_t, vel_t) -> None:
        """Copy into CUDA torch tensors (device to device)."""
        n = int(pos_t.shape[0])
        L.check(L.lib().sd_get_particles(self._h, pos_t.data_ptr(), vel_t.data_ptr(), n, L.SD_DEVICE),
                "sd_get_particles")

    def particle_pos_device_ptr(self) -> int:
        return int(L.lib().sd_particle_pos_device_ptr(self._h) or 0)

    def particle_vel_device_ptr(self) -> int:
        return int(L.lib().sd_particle_vel_device_ptr(self._h) or 0)

    def density_device_ptr(self) -> int:
        return int(L.lib().sd_density_device_ptr(self._h) or 0)

    def density(self) -> np.ndarray:
        G = self.grid_size()
        out = np.empty((G, G, G), np.float32)
        L.check(L.lib().sd_get_density(self._h, out.ctypes.data, L.SD_HOST), "sd_get_density")
        return out

    def potential(self) -> np.ndarray:
        G = self.grid_size()
        out = np.empty((G, G, G), np.float32)
        L.check(L.lib().sd_get_potential(self._h, out.ctypes.data, L.SD_HOST), "sd_get_potential")
        return out

    def accel(self, n: int | None = None) -> np.ndarray:
        n = self.particle_count() if n is None else n
        out = np.empty((n, 4), np.float32)
        L.check(L.lib().sd_get_accel(self._h, out.ctypes.data, n, L.SD_HOST), "sd_get_accel")
        return out

    def set_correction(self, correction) -> None:
        """Add a learned sub-grid correction (``learned.Correction``) to every
        step's acceleration; ``None`` restores the plain PM step."""
        from .learned import set_correction

        set_correction(self, correction)

    # ---- stepping -----------------------------------------------------------------
    def step_host(self, pos, vel, dt: float, out=None):
        """One offload step on host arrays (sd_step_host): upload, step, download.
        ``pos``/``vel``: float32 (n, 4) numpy arrays or CPU tensors (pinned for full
        copy speed); ``out``: optional (pos, vel) arrays to write. Returns them."""
        def ptr(a):
            return a.data_ptr() if hasattr(a, "data_ptr") else _host_f4(a).ctypes.data

        n = int(pos.shape[0])
        if out is None:
            out = (np.empty((n, 4), np.float32), np.empty((n, 4), np.float32))
        L.check(L.lib().sd_step_host(self._h, ptr(pos), ptr(vel), n, float(dt), ptr(out[0]), ptr(out[1])),
                "sd_step_host")
        return out

    def step_host_async(self, pos, vel, dt: float, out) -> None:
        """Queue one offload step (sd_step_host_async): ``pos``/``vel`` pinned CPU
        tensors, ``out`` = (pos, vel) pinned CPU tensors written by the time
        ``step_host_wait`` returns. Consecutive calls overlap their copies."""
        L.check(L.lib().sd_step_host_async(self._h, pos.data_ptr(), vel.data_ptr(), int(pos.shape[0]), float(dt),
                                           out[0].data_ptr(), out[1].data_ptr()), "sd_step_host_async")

    def step_host_wait(self) -> None:
        L.check(L.lib().sd_step_host_wait(self._h), "sd_step_host_wait")

    def step(self, dt: float | None = None) -> None:
        """``step()`` is the reference's CFL-clamped step; ``step(dt)`` advances by dt."""
        if dt is None:
            L.check(L.lib().sd_step_auto(self._h), "sd_step_auto")
        else:
            L.check(L.lib().sd_step(self._h, float(dt)), "sd_step")

    def steps(self, dt: float, n: int) -> None:
        L.check(L.lib().sd_steps(self._h, float(dt), int(n)), "sd_steps")

    def synchronize(self) -> None:
        L.check(L.lib().sd_synchronize(self._h), "sd_synchronize")

    def sort_only(self) -> np.ndarray:
        perm = np.empty(self.particle_count(), np.int32)
        L.check(L.lib().sd_sort_only(self._h, perm.ctypes.data, L.SD_HOST), "sd_sort_only")
        return perm

    # ---- state ----------------------------------------------------------------------
    def save_state(self, path: str) -> None:
        L.check(L.lib().sd_save_state(self._h, str(path).encode()), "sd_save_state")

    def load_state(self, path: str) -> None:
        L.check(L.lib().sd_load_state(self._h, str(path).encode()), "sd_load_state")

    # ---- queries -----------------------------------------------------------------------
    def timings(self) -> dict:
        t = L.SdTimings()
        L.check(L.lib().sd_timings_get(self._h, ctypes.byref(t)), "sd_timings_get")
        out = {f[0]: getattr(t, f[0]) for f in L.SdTimings._fields_ if f[0] != "kernel_ms"}
        out["kernel_ms"] = list(t.kernel_ms)
        return out

    def sim_time(self) -> float:
        return float(L.lib().sd_sim_time(self._h))

    def grid_size(self) -> int:
        return int(L.lib().sd_grid_size(self._h))

    def particle_count(self) -> int:
        return int(L.lib().sd_particle_count(self._h))

    def particle_capacity(self) -> int:
        return int(L.lib().sd_particle_capacity(self._h))

    def active_count(self) -> int:
        return int(L.lib().sd_active_count(self._h))

    def step_count(self) -> int:
        return int(L.lib().sd_step_count(self._h))

    def changed_fraction(self) -> float:
        """Share of keys the last merge sort found changed (-1 before the first)."""
        return float(L.lib().sd_changed_fraction(self._h))

    def merge_sorting(self) -> bool:
        return bool(L.lib().sd_merge_sorting(self._h))

    def measure_total_grid_mass(self) -> float:
        return float(L.lib().sd_measure_total_grid_mass(self._h))

    def measure_max_density(self) -> float:
        return float(L.lib().sd_measure_max_density(self._h))

    def measure_kinetic_energy(self) -> float:
        return float(L.lib().sd_measure_kinetic_energy(self._h))

    def measure_occupied_cells(self) -> int:
        return int(L.lib().sd_measure_occupied_cells(self._h))

    def measure_centroid(self) -> tuple[float, float]:
        cx, cy = ctypes.c_double(0.5), ctypes.c_double(0.5)
        L.check(L.lib().sd_measure_centroid(self._h, ctypes.byref(cx), ctypes.byref(cy)), "sd_measure_centroid")
        return cx.value, cy.value

    def diagnostics(self) -> dict:
        d = L.SdDiagnostics()
        L.check(L.lib().sd_diagnostics_get(self._h, ctypes.byref(d)), "sd_diagnostics_get")
        return {"kinetic": d.kinetic, "potential": d.potential, "momentum": list(d.momentum),
                "mean_velocity_removed": list(d.mean_velocity_removed), "live_count": d.live_count}

    def diagnostics_history(self, max_records: int = 4096) -> np.ndarray:
        """Per-step FP64 records (diagnostics = 1), oldest first: columns
        step, kinetic, potential, px, py, pz, live, |mean removed|."""
        out = np.zeros((max_records, 8), np.float64)
        k = ctypes.c_int(0)
        L.check(L.lib().sd_diagnostics_history(self._h, out.ctypes.data, max_records, ctypes.byref(k)),
                "sd_diagnostics_history")
        return out[:k.value]

    @staticmethod
    def kernel_launches() -> int:
        return int(L.lib().sd_kernel_launches(None))
