"""ctypes bindings of ``libstardust_pm.so`` (the C ABI in ``include/stardust_pm.h``).

The library is built in-tree by ``stardust_b200.build``. There is no fallback:
if the shared library is missing, importing the bindings raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libstardust_pm.so")

SD_OK = 0
SD_E_ARG, SD_E_CUDA, SD_E_NOMEM, SD_E_STATE, SD_E_IO, SD_E_FORMAT, SD_E_UNSUPPORTED = -1, -2, -3, -4, -5, -6, -7
SD_BOUNDARY_ISOLATED, SD_BOUNDARY_PERIODIC = 0, 1
SD_ORDER_ROWMAJOR, SD_ORDER_MORTON, SD_ORDER_TILED = 0, 1, 2
SD_INT_KD, SD_INT_KDK = 0, 1
SD_UNITS_REFERENCE, SD_UNITS_NEWTON = 0, 1
SD_HOST, SD_DEVICE = 0, 1
SD_PRESET_FILAMENT, SD_PRESET_EMPTY = 0, 1
SD_FIELD_DENSITY, SD_FIELD_DISPERSION = 0, 1


class SdConfig(ctypes.Structure):
    _fields_ = [
        ("particle_count", ctypes.c_int32),
        ("grid_size", ctypes.c_int32),
        ("boundary", ctypes.c_int32),
        ("gravity", ctypes.c_float),
        ("softening_cells", ctypes.c_float),
        ("time_scale", ctypes.c_float),
        ("sort_interval", ctypes.c_int32),
        ("length_scale", ctypes.c_float),
        ("time_unit_scale", ctypes.c_float),
        ("order", ctypes.c_int32),
        ("integrator", ctypes.c_int32),
        ("units", ctypes.c_int32),
        ("diagnostics", ctypes.c_int32),
        ("keep_density", ctypes.c_int32),
        ("preset", ctypes.c_int32),
        ("dark_matter_fraction", ctypes.c_float),
        ("big_bang_shrink", ctypes.c_float),
        ("spin", ctypes.c_float),
        ("hubble", ctypes.c_float),
        ("vel_dispersion", ctypes.c_float),
        ("pressure_enabled", ctypes.c_int32),
        ("pressure_k", ctypes.c_float),
        ("cooling_enabled", ctypes.c_int32),
        ("cooling_rate", ctypes.c_float),
        ("full_sort", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 7),
    ]


class SdTimings(ctypes.Structure):
    _fields_ = [
        ("sort_ms", ctypes.c_float),
        ("deposit_ms", ctypes.c_float),
        ("poisson_ms", ctypes.c_float),
        ("gather_ms", ctypes.c_float),
        ("total_ms", ctypes.c_float),
        ("dt_used", ctypes.c_float),
        ("max_speed", ctypes.c_float),
        ("steps", ctypes.c_int32),
        ("kernel_ms", ctypes.c_float * 8),
    ]


class SdView(ctypes.Structure):
    _fields_ = [("rot", ctypes.c_float * 9), ("center", ctypes.c_float * 3), ("fly", ctypes.c_int32),
                ("tan_half_fov", ctypes.c_float), ("zoom", ctypes.c_float), ("pan_x", ctypes.c_float),
                ("pan_y", ctypes.c_float), ("size_px", ctypes.c_float), ("color_by", ctypes.c_int32),
                ("cmap", ctypes.c_int32), ("bright", ctypes.c_float), ("inv_gamma", ctypes.c_float),
                ("use_cmap", ctypes.c_int32), ("reinhard", ctypes.c_int32), ("rot_on", ctypes.c_int32),
                ("reserved", ctypes.c_int32 * 3)]


class SdSceneTuning(ctypes.Structure):
    _fields_ = [("order", ctypes.c_int32), ("gather_blocks", ctypes.c_int32), ("step_ms", ctypes.c_float),
                ("deposit_split", ctypes.c_int32)]


class SdDiagnostics(ctypes.Structure):
    _fields_ = [
        ("kinetic", ctypes.c_double),
        ("potential", ctypes.c_double),
        ("momentum", ctypes.c_double * 3),
        ("mean_velocity_removed", ctypes.c_double * 3),
        ("live_count", ctypes.c_double),
    ]


# (name, restype, argtypes) for every symbol the header declares.
_P, _I, _F, _D, _S = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_size_t
_LL = ctypes.c_longlong
SIGNATURES = [
    ("sd_abi_version", _I, []),
    ("sd_device_available", _I, []),
    ("sd_failed", _I, []),
    ("sd_last_error", ctypes.c_char_p, []),
    ("sd_clear_error", None, []),
    ("sd_config_default", _I, [ctypes.POINTER(SdConfig)]),
    ("sd_max_grid_size", _I, [_I]),
    ("sd_estimate_bytes", _S, [_I, _I, _I]),
    ("sd_max_particles_for", _I, [_I, _I, _S]),
    ("sd_estimate_step_ms", _D, [_I, _I, _I]),
    ("sd_device_free_bytes", _S, []),
    ("sd_set_device_free_bytes_override", None, [_S]),
    ("sd_device_bandwidth_gbs", _D, []),
    ("sd_device_multiprocessors", _I, []),
    ("sd_device_name", _I, [ctypes.c_char_p, _I]),
    ("sd_device_driver", _I, [ctypes.c_char_p, _I]),
    ("sd_create", _I, [ctypes.POINTER(_P), _I]),
    ("sd_destroy", _I, [_P]),
    ("sd_set_stream", _I, [_P, _P]),
    ("sd_init", _I, [_P, ctypes.POINTER(SdConfig)]),
    ("sd_reconfigure", _I, [_P, ctypes.POINTER(SdConfig)]),
    ("sd_reset", _I, [_P]),
    ("sd_get_config", _I, [_P, ctypes.POINTER(SdConfig)]),
    ("sd_set_particles", _I, [_P, _P, _P, _I, _I]),
    ("sd_get_particles", _I, [_P, _P, _P, _I, _I]),
    ("sd_particle_pos_device_ptr", _P, [_P]),
    ("sd_particle_vel_device_ptr", _P, [_P]),
    ("sd_density_device_ptr", _P, [_P]),
    ("sd_get_density", _I, [_P, _P, _I]),
    ("sd_get_potential", _I, [_P, _P, _I]),
    ("sd_get_accel", _I, [_P, _P, _I, _I]),
    ("sd_step", _I, [_P, _F]),
    ("sd_step_auto", _I, [_P]),
    ("sd_step_host", _I, [_P, _P, _P, _I, _F, _P, _P]),
    ("sd_step_host_async", _I, [_P, _P, _P, _I, _F, _P, _P]),
    ("sd_step_host_wait", _I, [_P]),
    ("sd_steps", _I, [_P, _F, _I]),
    ("sd_synchronize", _I, [_P]),
    ("sd_sort_only", _I, [_P, _P, _I]),
    ("sd_save_state", _I, [_P, ctypes.c_char_p]),
    ("sd_load_state", _I, [_P, ctypes.c_char_p]),
    ("sd_timings_get", _I, [_P, ctypes.POINTER(SdTimings)]),
    ("sd_sim_time", _D, [_P]),
    ("sd_grid_size", _I, [_P]),
    ("sd_particle_count", _I, [_P]),
    ("sd_particle_capacity", _I, [_P]),
    ("sd_active_count", _I, [_P]),
    ("sd_step_count", _I, [_P]),
    ("sd_changed_fraction", _D, [_P]),
    ("sd_merge_sorting", _I, [_P]),
    ("sd_measure_total_grid_mass", _D, [_P]),
    ("sd_measure_max_density", _D, [_P]),
    ("sd_measure_kinetic_energy", _D, [_P]),
    ("sd_measure_occupied_cells", _I, [_P]),
    ("sd_measure_centroid", _I, [_P, _P, _P]),
    ("sd_diagnostics_get", _I, [_P, ctypes.POINTER(SdDiagnostics)]),
    ("sd_kernel_launches", _LL, [_P]),
    ("sd_cell_keys", _I, [_P, _I, _I, _I, _P, _P]),
    ("sd_key_bits", _I, [_I, _I]),
    ("sd_sort_workspace_bytes", _S, [_I]),
    ("sd_sort_pairs", _I, [_P, _P, _P, _P, _P, _P, _I, _I, _P, _S, _P]),
    ("sd_reorder", _I, [_P, _P, _P, _P, _P, _I, _P]),
    ("sd_deposit_workspace_bytes", _S, [_I]),
    ("sd_deposit", _I, [_P, _I, _I, _P, _P, _S, _P]),
    ("sd_poisson_workspace_bytes", _S, [_I]),
    ("sd_poisson", _I, [_P, _I, _F, _P, _P, _S, _P]),
    ("sd_poisson_noalloc", _I, [_P, _I, _F, _P, _P]),
    ("sd_gather_kick_drift", _I, [_P, _I, _F, _P, _P, _I, _F, _F, _F, _P, _P, _P, _S, _P]),
    ("sd_gather_workspace_bytes", _S, [_I]),
    ("sd_interpolate_accel", _I, [_P, _I, _F, _P, _P, _I, _P]),
    ("sd_diagnostics_history", _I, [_P, _P, _I, _P]),
    ("sd_mlp_param_count", _I, []),
    ("sd_mlp_features", _I, [_P, _P, _I, _P, _I, _F, _P, _P]),
    ("sd_mlp_infer", _I, [_P, _P, _P, _I, _P, _I, _F, _F, _P, _P]),
    ("sd_mlp_wait_timeouts", _I, []),
    ("sd_mlp_train_workspace_bytes", _S, [_I]),
    ("sd_mlp_loss_grad", _I, [_P, _P, _P, _I, _P, _P, _P, _S, _P]),
    ("sd_mlp_adam", _I, [_P, _P, _P, _P, _I, _F, _F, _F, _F, _P]),
    ("sd_set_mlp", _I, [_P, _P, _F]),
    ("sd_ensemble_create", _I, [_P, _I]),
    ("sd_ensemble_destroy", _I, [_P]),
    ("sd_ensemble_add", _I, [_P, _P, _P, _P, _I, _I]),
    ("sd_ensemble_size", _I, [_P]),
    ("sd_ensemble_scene", _P, [_P, _I]),
    ("sd_ensemble_autotune", _I, [_P, _F, _I]),
    ("sd_ensemble_get_tuning", _I, [_P, _I, _P]),
    ("sd_ensemble_steps", _I, [_P, _F, _I]),
    ("sd_ensemble_synchronize", _I, [_P]),
    ("sd_ensemble_stream", _P, [_P]),
    ("sd_ensemble_graph_kernels", _LL, [_P]),
    ("sd_view_default", None, [_P]),
    ("sd_render_workspace_bytes", _S, [_I, _I]),
    ("sd_render_points", _I, [_P, _P, _I, _P, _I, _I, _P, _S, _P, _P]),
    ("sd_render_field_workspace_bytes", _S, [_I]),
    ("sd_render_field", _I, [_I, _P, _I, _P, _P, _I, _P, _I, _I, _P, _S, _P, _P]),
    ("sd_ewald_modes", _I, [_I]),
    ("sd_ewald_workspace_bytes", _S, [_I]),
    ("sd_ewald_forces", _I, [_P, _I, _P, _I, _D, _D, _I, _P, _P, _S, _P]),
]

_lib = None


class SdError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        super().__init__(f"{what} failed with status {code}: {last_error()}")


def lib() -> ctypes.CDLL:
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m stardust_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    m = lib().sd_last_error()
    return m.decode() if m else ""


def check(rc: int, what: str) -> None:
    if rc != SD_OK:
        raise SdError(rc, what)
