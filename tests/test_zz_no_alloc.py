"""fdtd_gradient_noalloc through the C ABI (needs a B200).

Some callers cannot let the library call cudaMalloc or cudaFree while they run: those calls can
synchronize the whole device and stall everything else on it, and a process whose device memory is
held by a caching allocator may have none to give. fdtd_gradient_noalloc serves them from a fixed
static pool. Here its gradient must equal fdtd_gradient's on two calls in a row, and a run too large
for the pool must be refused before any work. This file is collected last; it also passes alone in
a fresh process."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
from conftest import load_golden

from acoustic_spaces_b200 import B200WaveSolver, _abi

pytestmark = pytest.mark.gpu

_F64 = ctypes.POINTER(ctypes.c_double)


def _noalloc(solver, signal, dloss, segment):
    signal = np.ascontiguousarray(signal, np.float32)
    dloss = np.ascontiguousarray(dloss, np.float64)
    info = solver.info()
    out = {k: np.zeros(int(n)) for k, n in (("coef_b", info.special_cells), ("coef_inv", info.special_cells),
                                              ("now", info.branch_states), ("before", info.branch_states),
                                              ("gain", info.branch_states))}  # fmt: skip
    lib = _abi.load_library()
    status = lib.fdtd_gradient_noalloc(solver._handle, signal.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                       len(signal), dloss.ctypes.data_as(_F64), segment,
                                       *(a.ctypes.data_as(_F64) for a in out.values()))  # fmt: skip
    return status, out


@pytest.mark.parametrize("name,precision,rtol", [("resonant7", "fp64", 1e-12), ("fitted_closed", "fp32", 1e-6)])
def test_the_static_pool_gives_fdtd_gradients_result_twice(name, precision, rtol):
    layout, signal, _ = load_golden(name)
    signal = signal[:200]
    solver = B200WaveSolver(layout, precision=precision)
    y = solver.run(signal)
    dloss = 2.0 * (y - 0.7 * y)
    solver.reset()
    expected = solver.gradient(signal, dloss, segment=64)
    held = solver.info().device_bytes
    for _ in range(2):
        status, got = _noalloc(solver, signal, dloss, 64)
        assert status == _abi.FDTD_OK, _abi.load_library().fdtd_last_error(solver._handle)
        # the handle took no device memory for it, and kept none
        assert solver.info().device_bytes == held
        for key in expected:
            scale = np.max(np.abs(expected[key])) if expected[key].size else 0.0
            np.testing.assert_allclose(got[key], expected[key], rtol=rtol, atol=rtol * scale, err_msg=key)
    solver.close()


def test_a_run_beyond_the_pool_is_refused_before_any_work():
    layout, signal, _ = load_golden("resonant7")
    solver = B200WaveSolver(layout, precision="fp64")
    # a state a gradient would change: a gradient resets the grid and steps it from rest
    solver.run(signal[:37])
    before = solver.state()
    held = solver.info().device_bytes
    steps = 1_000_000  # dL/dy alone takes probes x 8 MB, beyond the 16 MiB pool
    status, _ = _noalloc(solver, np.zeros(steps, np.float32), np.zeros((solver.probes, steps)), 0)
    assert status == _abi.FDTD_EINVAL
    message = _abi.load_library().fdtd_last_error(solver._handle).decode()
    assert "static pool holds 16777216" in message
    after = solver.state()
    for key in before:
        np.testing.assert_array_equal(after[key], before[key], err_msg=key)
    assert solver.info().steps_done == 37
    assert solver.info().device_bytes == held
    solver.close()
