"""The GPU free-surface field (gatherSurfaceOccupancy, shaders.ts:700-806,
through mpm_gather_surface_occupancy) against the FP64 current-area oracle
(occupancy.ts:70-128; the GPU field is the display area, twice it):

* a two-liquid dam break, before and after 8 substeps, and the Gate 4 scene
  (water, oil, pebbles, fracture particles: only the liquids count), every
  node within 3 max(cellsX, cellsY) 2^-24 of the largest value plus 1e-5
  relative: the device divides position by cellSize in float32 as the
  reference's shader does, so a stencil fraction carries up to an ulp of the
  grid coordinate, and a weight (slope at most 1.5) twice that;
* the water and oil sums conserve 2 V det F over the liquid particles;
* repeated gathers are bit-identical (fixed-point sums).
"""
import numpy as np
import pytest

from mpm_b200 import create_mpm_mls_gpu_solver
from mpm_b200.scenes import (create_dam_break_scene, create_mpm_gate4_scene,
                             create_mpm_gate4_step_config)
from oracle import current_area_fp64

pytestmark = pytest.mark.gpu

WATER_MODEL, OIL_MODEL = 2, 3


def _oracle_display(solver, config):
    packed, _ = solver.read_particles_packed()
    pk = packed.astype(np.float64)
    model = packed[:, 13].view(np.uint32)
    phase = np.where(model == WATER_MODEL, 0, np.where(model == OIL_MODEL, 1, 2))
    g = config["grid"]
    field = current_area_fp64(pk[:, 0], pk[:, 1], pk[:, 8:12], pk[:, 17], phase, g["cellsX"], g["cellsY"],
                              float(np.float32(g["cellSize"])))
    liquid = phase < 2
    det = pk[:, 8] * pk[:, 11] - pk[:, 9] * pk[:, 10]
    totals = [2 * np.sum(pk[liquid & (phase == k), 17] * det[liquid & (phase == k)]) for k in (0, 1)]
    return 2 * field, totals


def _check(solver, config):
    gpu = solver.gather_surface_occupancy().astype(np.float64)
    want, totals = _oracle_display(solver, config)
    scale = np.abs(want).max()
    assert scale > 0
    err = np.abs(gpu - want)
    g = config["grid"]
    atol = 3 * max(g["cellsX"], g["cellsY"]) * 2.0 ** -24 * scale
    assert np.all(err <= atol + 1e-5 * np.abs(want)), float(err.max() / scale)
    cell = float(np.float32(config["grid"]["cellSize"])) ** 2
    for k in (0, 1):
        assert abs(gpu[..., k].sum() * cell - totals[k]) <= 1e-5 * max(totals[k], 1e-30)
    again = solver.gather_surface_occupancy()
    assert np.array_equal(again, gpu.astype(np.float32))
    return gpu


def test_dam_break_surface_field_matches_the_oracle():
    grid = {"cellsX": 256, "cellsY": 256, "cellSize": 10}
    p, config = create_dam_break_scene(particles_per_phase=20_000, columns=200, grid=grid)
    solver = create_mpm_mls_gpu_solver(p, config)
    try:
        before = _check(solver, config)
        assert before[..., 0].sum() > 0 and before[..., 1].sum() > 0
        solver.step_batch(8, 5e-4, {"x": 0.0, "y": 90.0})
        solver.check_numerical_status()
        _check(solver, config)
        ptr, w, h = solver.surface_field_device()
        assert ptr != 0 and (w, h) == (259, 259)
    finally:
        solver.dispose()


def test_gate4_counts_only_the_liquids():
    p, bonds, _ = create_mpm_gate4_scene()
    for a in (p.px, p.py, p.vx, p.vy):
        a[:] = a.astype(np.float32)
    config = create_mpm_gate4_step_config(fracture_bonds=bonds)
    solver = create_mpm_mls_gpu_solver(p, config)
    try:
        _check(solver, config)
        solver.step_batch(4, 2e-4, config["gravity"])
        solver.check_numerical_status()
        _check(solver, config)
    finally:
        solver.dispose()
