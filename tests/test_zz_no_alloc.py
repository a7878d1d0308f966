"""The allocation-free Poisson entry point, checked against the regular one.

sd_poisson_noalloc serves callers that cannot allocate device memory (no
cudaMalloc and no caller workspace on their path): it keeps its spectrum in
fixed device storage of the library, limited to grids of up to 128^3. This file
is collected last on purpose, so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

from stardust_b200 import _lib as L

pytestmark = pytest.mark.gpu

RTOL = 2e-5  # relative to the potential's range, the Poisson tolerance of the stage tests


def _solve_regular(cuda, lib, rho_d, G, soft):
    phi = cuda.empty(G ** 3, dtype=cuda.float32, device="cuda")
    ws = cuda.empty(int(lib.sd_poisson_workspace_bytes(G)), dtype=cuda.uint8, device="cuda")
    L.check(lib.sd_poisson(rho_d.data_ptr(), G, ctypes.c_float(soft), phi.data_ptr(), ws.data_ptr(), ws.numel(),
                           None), "sd_poisson")
    cuda.cuda.synchronize()
    return phi.cpu().numpy()


def _solve_noalloc(cuda, lib, rho_d, G, soft, stream=None):
    phi = cuda.empty(G ** 3, dtype=cuda.float32, device="cuda")
    handle = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
    L.check(lib.sd_poisson_noalloc(rho_d.data_ptr(), G, ctypes.c_float(soft), phi.data_ptr(), handle),
            "sd_poisson_noalloc")
    cuda.cuda.synchronize()
    return phi.cpu().numpy()


@pytest.mark.parametrize("on_stream", [False, True], ids=["default-stream", "caller-stream"])
@pytest.mark.parametrize("G", [16, 64, 128])
def test_noalloc_matches_regular_entry_point_twice(cuda, lib, oracle, G, on_stream):
    rng = np.random.default_rng(G)
    stream = cuda.cuda.Stream() if on_stream else None
    # two different inputs in a row: the shared workspace keeps the previous
    # call's contents, which must not leak into the next result
    for call, soft in enumerate((1.0, 2.5)):
        rho = rng.random((G, G, G), dtype=np.float32) * (1 + call)
        rho[rng.integers(0, G, 8), rng.integers(0, G, 8), rng.integers(0, G, 8)] += 50.0
        rho_d = cuda.from_numpy(rho).cuda()
        ref = _solve_regular(cuda, lib, rho_d, G, soft)
        got = _solve_noalloc(cuda, lib, rho_d, G, soft, stream)
        # the same kernels and the same tables as sd_poisson: the same bits
        assert np.array_equal(got.view(np.int32), ref.view(np.int32)), (G, call)
        # and the FP64 solve, within the Poisson tolerance of the stage tests
        exact = oracle.poisson_periodic_f64(rho.astype(np.float64), soft).reshape(-1)
        span = float(exact.max() - exact.min())
        assert np.abs(got - exact).max() <= RTOL * span, (G, call)


def test_noalloc_rejects_grids_beyond_its_workspace(cuda, lib):
    rho = cuda.zeros(256 ** 3, dtype=cuda.float32, device="cuda")
    phi = cuda.empty_like(rho)
    lib.sd_clear_error()
    rc = lib.sd_poisson_noalloc(rho.data_ptr(), 256, ctypes.c_float(1.0), phi.data_ptr(), None)
    assert rc == L.SD_E_ARG
    assert "128" in L.last_error()
    lib.sd_clear_error()
    assert lib.sd_poisson_noalloc(rho.data_ptr(), 48, ctypes.c_float(1.0), phi.data_ptr(), None) == L.SD_E_ARG
    lib.sd_clear_error()
