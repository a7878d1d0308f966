"""CPU checks of the C ABI: the library loads, exports every symbol the header
declares, and validates arguments without touching a GPU."""
import ctypes
import os
import re

import pytest

from stardust_b200 import _lib as L

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "stardust_pm.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sd_[a-z0-9_]+)\s*\(", text)))


def test_header_and_bindings_agree(lib):
    declared = declared_symbols()
    bound = sorted(name for name, _, _ in L.SIGNATURES)
    assert declared == bound


def test_every_declared_symbol_is_exported(lib):
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_struct_sizes_match_header(lib):
    assert ctypes.sizeof(L.SdConfig) == 32 * 4
    assert ctypes.sizeof(L.SdTimings) == 16 * 4


def test_defaults_follow_reference_simconfig(lib):
    c = L.SdConfig()
    assert lib.sd_config_default(ctypes.byref(c)) == 0
    assert c.particle_count == 2_000_000 and c.grid_size == 128       # Sim.h:166-167
    assert c.softening_cells == 3.0 and c.time_scale == 1.0          # Sim.h:315-316
    assert c.length_scale == 1.0 and c.time_unit_scale == 1.0
    assert c.boundary == L.SD_BOUNDARY_PERIODIC and c.sort_interval == 1


def test_static_queries(lib):
    assert lib.sd_abi_version() == 2
    assert lib.sd_max_grid_size(L.SD_BOUNDARY_PERIODIC) == 512       # Sim.cu:4158
    assert lib.sd_max_grid_size(L.SD_BOUNDARY_ISOLATED) == 256
    # key bits of key+1: G^3 + 1 values for row-major / Morton; tile rows: G^2 values
    assert lib.sd_key_bits(64, L.SD_ORDER_ROWMAJOR) == 19
    assert lib.sd_key_bits(512, L.SD_ORDER_ROWMAJOR) == 28
    assert lib.sd_key_bits(512, L.SD_ORDER_TILED) == 18
    small = lib.sd_estimate_bytes(1000, 64, L.SD_BOUNDARY_PERIODIC)
    big = lib.sd_estimate_bytes(1000, 128, L.SD_BOUNDARY_PERIODIC)
    assert 0 < small < big
    assert lib.sd_sort_workspace_bytes(1 << 20) >= 256 * 512 * 4


def test_argument_validation_needs_no_gpu(lib):
    lib.sd_clear_error()
    assert lib.sd_create(None, 0) == L.SD_E_ARG
    assert lib.sd_failed() == 1 and "null" in L.last_error()
    lib.sd_clear_error()
    assert lib.sd_failed() == 0
    assert lib.sd_init(None, None) == L.SD_E_ARG
    assert lib.sd_step(None, ctypes.c_float(1e-3)) == L.SD_E_ARG
    assert lib.sd_cell_keys(None, 10, 64, 0, None, None) == L.SD_E_ARG
    assert lib.sd_cell_keys(None, 10, 48, 0, None, None) == L.SD_E_ARG  # not a power of two
    assert lib.sd_deposit(None, 10, 64, None, None, 0, None) == L.SD_E_ARG
    assert lib.sd_sort_pairs(None, None, None, None, None, None, 10, 20, None, 0, None) == L.SD_E_ARG
    assert lib.sd_sort_pairs(None, None, None, None, None, None, 10, 40, None, 0, None) == L.SD_E_ARG
    lib.sd_clear_error()


def test_first_failure_is_sticky(lib):
    lib.sd_clear_error()
    lib.sd_init(None, None)
    first = L.last_error()
    lib.sd_cell_keys(None, 10, 64, 0, None, None)
    assert L.last_error() == first
    lib.sd_clear_error()


def test_create_without_device_reports_cuda_error(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    h = ctypes.c_void_p()
    assert lib.sd_create(ctypes.byref(h), 0) == L.SD_E_CUDA
    assert lib.sd_device_available() == 0
    lib.sd_clear_error()


def test_max_particles_for_fits_the_memory(lib):
    """Sim::maxParticlesFor (Sim.cu:4057-4066): the grid's share first, 80 % of the
    rest for particles; the allocation model of that many particles fits."""
    for G, b in ((64, L.SD_BOUNDARY_PERIODIC), (512, L.SD_BOUNDARY_PERIODIC), (256, L.SD_BOUNDARY_ISOLATED)):
        grid = lib.sd_estimate_bytes(1, G, b)
        assert lib.sd_max_particles_for(G, b, grid) == 0          # nothing left for particles
        assert lib.sd_max_particles_for(G, b, grid // 2) == 0
        free = grid + (1 << 30)
        n = lib.sd_max_particles_for(G, b, free)
        assert 1000 < n
        assert lib.sd_estimate_bytes(n, G, b) <= free
        # 80 % of the room: the model of 1.3 n particles no longer fits in it
        assert lib.sd_estimate_bytes(int(n * 1.3), G, b) > free
    assert lib.sd_max_particles_for(512, L.SD_BOUNDARY_PERIODIC, 1 << 62) == 400_000_000
    assert lib.sd_max_particles_for(64, 7, 1 << 40) == 0


def test_device_queries_without_a_device(lib):
    """Without a GPU the device queries answer 0 or empty, as the reference's do."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    assert lib.sd_estimate_step_ms(1 << 20, 128, L.SD_BOUNDARY_PERIODIC) == 0.0
    assert lib.sd_device_bandwidth_gbs() == 0.0
    buf = ctypes.create_string_buffer(64)
    assert lib.sd_device_name(buf, 64) == 0 and buf.value == b"unknown"
