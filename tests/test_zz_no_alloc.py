"""The allocation-free cell sort (mpm_cell_sort_static) against the solver's.

Callers that cannot call cudaMalloc (an embedding host that owns the GPU
memory budget, a frame loop that must not stall on an allocation, a thin
foreign-function host without an allocator) use mpm_cell_sort_static, whose
scratch is a static array inside the library.  Its keys, permutation and cell
starts must equal those of the solver's own sort (mpm_probe_sort) and the
stable argsort of the keys bit for bit, on two calls in a row (the second call
reuses the array the first call left behind); the calls must not take device
memory (free memory, read with cudaMemGetInfo, stays within one allocation
granule), and sizes beyond its fixed maximum must be refused.

This file is collected last so that a run that stops at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

from mpm_b200 import _lib, create_mpm_mls_gpu_solver
from mpm_b200.layout import validate_mpm_mls_gpu_input
from mpm_b200.scenes import create_si_tank_scene

pytestmark = pytest.mark.gpu


def _static_sort(lib, cells_x, cells_y, cell_size, positions):
    count = positions.shape[0]
    keys = np.zeros(count, dtype=np.uint32)
    perm = np.zeros(count, dtype=np.uint32)
    starts = np.zeros((cells_x + 3) * (cells_y + 3) + 1, dtype=np.uint32)
    error = ctypes.create_string_buffer(256)
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    rc = lib.mpm_cell_sort_static(0, cells_x, cells_y, ctypes.c_float(cell_size), _lib.ptr(pos), count,
                                  _lib.ptr(keys), _lib.ptr(perm), _lib.ptr(starts), error, 256)
    return rc, keys, perm, starts, error.value.decode()


def _free_device_bytes():
    runtime = ctypes.CDLL("libcudart.so.12")
    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    assert runtime.cudaMemGetInfo(ctypes.byref(free), ctypes.byref(total)) == 0
    return free.value


def _library():
    lib = _lib.load_library()
    fn = lib.mpm_cell_sort_static
    fn.argtypes = [ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, ctypes.c_void_p,
                   ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p,
                   ctypes.c_uint32]
    fn.restype = ctypes.c_int32
    return lib


@pytest.mark.parametrize("seed", [7, 8])
def test_static_sort_matches_the_solver_sort_on_two_calls(seed):
    lib = _library()
    particles, config = create_si_tank_scene(seed=seed)
    solver = create_mpm_mls_gpu_solver(particles, config)
    try:
        keys_ref, perm_ref, starts_ref = solver.probe_sort(1e-4)
    finally:
        solver.dispose()
    positions = validate_mpm_mls_gpu_input(particles, config).packed_particles[:, 0:2]
    grid = config["grid"]
    # the stable counting sort, stated directly: keys of the base cells, the
    # stable argsort, the cell starts
    dx = np.float32(grid["cellSize"])
    base = np.floor((positions / dx).astype(np.float32) - np.float32(0.5)).astype(np.int64)
    keys_np = (base[:, 1] + 1) * (grid["cellsX"] + 3) + (base[:, 0] + 1)
    perm_np = np.argsort(keys_np, kind="stable")
    counts = np.bincount(keys_np, minlength=(grid["cellsX"] + 3) * (grid["cellsY"] + 3))
    starts_np = np.concatenate(([0], np.cumsum(counts)))
    free_before = None
    for call in range(3):
        rc, keys, perm, starts, message = _static_sort(lib, grid["cellsX"], grid["cellsY"], dx, positions)
        assert rc == 0, message
        assert np.array_equal(keys, keys_ref) and np.array_equal(keys.astype(np.int64), keys_np)
        assert np.array_equal(perm, perm_ref) and np.array_equal(perm.astype(np.int64), perm_np)
        assert np.array_equal(starts, starts_ref) and np.array_equal(starts.astype(np.int64), starts_np)
        if call == 0:
            free_before = _free_device_bytes()  # after the first call's one-time set-up
    assert free_before - _free_device_bytes() < 2 * 1024 * 1024


def test_static_sort_refuses_sizes_beyond_its_maximum():
    lib = _library()
    too_many = np.zeros((65537, 2), dtype=np.float32) + 1.0
    rc, _, _, _, message = _static_sort(lib, 16, 16, 1.0, too_many)
    assert rc == _lib.MPM_ERR_INVALID_ARGUMENT
    assert "65536" in message
    rc, _, _, _, message = _static_sort(lib, 1024, 1024, 1.0, np.ones((4, 2), dtype=np.float32))
    assert rc == _lib.MPM_ERR_INVALID_ARGUMENT
    assert "262144" in message
