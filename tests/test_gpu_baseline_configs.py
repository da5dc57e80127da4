"""The CUDA path at the benchmark configurations, against the FP64 oracle.

* C3, the 1,000,000-particle water/oil dam break (1024x2048 cells): 5 CFL
  microsteps of its 1/240 s macrostep through both P2G paths (gather, and
  fixed point at 2^16: the reference's 2^24 overflows at these sums);
  positions within 1e-3 cell sizes, velocities within 1e-3 (1 + |v|).
* C2, the enlarged multi-material Gate 4 scene of
  src/lib/mpm/kernels/README.md:116-135 (220x600 grid, liquid area 1,600,
  +4,500 in y; 2,000 water, 1,500 oil, 50 bonded pebbles, a fractured
  24-particle solid): 4 CFL microsteps through both paths within the
  reference's own CPU-vs-GPU bounds (src/routes/labs/mpm/kernels/
  +page.svelte:120-122: position 0.02, velocity 0.025 + 5e-4 |v|) and the
  fracture damage within 1e-3.
* C1, the SI tank over its full 600 macrosteps of 1/120 s (about 1.4e5
  microsteps): the trajectories of float32 and float64 runs part long before
  that (the flow is a collapsing column), so the check is statistical: the
  water diagnostics of src/lib/mpm/experiments/si-performance.ts:19-56 every
  60 macrosteps against the oracle's (tests/golden/si_tank_long_fp64.json),
  within the bounds of LONG_HORIZON_BOUNDS.
"""
import json
import os

import numpy as np
import pytest

from helpers import oracle_columns, packed_columns
from mpm_b200 import (calculate_mpm_cfl_microsteps, create_experimental_mpm_mls_atomic_gpu_solver,
                      create_mpm_mls_gpu_solver)
from mpm_b200.diagnostics import summarize_si_water
from mpm_b200.scenes import (DAM_BREAK_FIXED_STEP_SECONDS, DAM_BREAK_GRAVITY, GATE4_FIXED_STEP_SECONDS,
                              SI_TANK_GRAVITY, create_dam_break_scene, create_mpm_gate4_scene,
                              create_mpm_gate4_step_config, create_si_tank_scene)
from oracle import OracleState

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))

# |GPU - oracle| per diagnostic at each checkpoint of the 600-macrostep run:
# (absolute, relative to the oracle's value).  The oracle's own values over
# the run: area drift -0.013 to -0.017 %, density-error p95 1.1-1.3 %,
# det F in [0.947, 1.063], maximum speed 0.01-0.06 m/s.
LONG_HORIZON_BOUNDS = {
    "areaDriftPercent": (0.05, 0.0),
    "densityErrorPercentP95": (0.1, 0.1),
    "determinantMin": (0.01, 0.0),
    "determinantMax": (0.01, 0.0),
    "maximumSpeed": (0.01, 0.25),
}


def _factory(variant):
    if variant == "gather":
        return create_mpm_mls_gpu_solver
    return lambda p, c: create_experimental_mpm_mls_atomic_gpu_solver(p, c, fixed_point_shift=16)


@pytest.mark.parametrize("variant", ["gather", "fixed16"])
def test_dam_break_1m_matches_the_oracle(variant):
    p, config = create_dam_break_scene()
    assert len(p.px) == 1_000_000
    solver = _factory(variant)(p, config)
    try:
        bounds = solver.cfl_bounds
        plan = calculate_mpm_cfl_microsteps(DAM_BREAK_FIXED_STEP_SECONDS, config["grid"]["cellSize"],
                                            bounds["waveSpeedBound"], 5.0, 64)
        steps = 5
        solver.step_batch(steps, plan["microDt"], DAM_BREAK_GRAVITY)
        solver.check_numerical_status()
        packed, _ = solver.read_particles_packed()
    finally:
        solver.dispose()
    dt32 = float(np.float32(plan["microDt"]))
    cfg = dict(config, dt=dt32, gravity=DAM_BREAK_GRAVITY)
    state = OracleState(p, cfg)
    state.run(cfg, steps)
    gpu, ref = packed_columns(packed), oracle_columns(state)
    dx = config["grid"]["cellSize"]
    pos_err = float(np.max(np.abs(gpu["position"] - ref["position"])))
    vel_err = float(np.max(np.abs(gpu["velocity"] - ref["velocity"]) / (1 + np.abs(ref["velocity"]))))
    assert pos_err <= 1e-3 * dx, pos_err
    assert vel_err <= 1e-3, vel_err
    # the scene moved: gravity acted over the five microsteps
    assert float(np.max(np.abs(ref["velocity"]))) > 0.1


@pytest.mark.parametrize("variant", ["gather", "fixed16"])
def test_enlarged_gate4_scene_matches_the_oracle(variant):
    p, bonds, _ = create_mpm_gate4_scene(liquid_particle_area=1600, y_shift=4500)
    for a in (p.px, p.py, p.vx, p.vy):
        a[:] = a.astype(np.float32)
    grid = {"cellsX": 220, "cellsY": 600, "cellSize": 10}
    config = create_mpm_gate4_step_config(fracture_bonds=bonds, grid=grid)
    assert len(p.px) == 3_674
    dt = GATE4_FIXED_STEP_SECONDS / 5
    steps = 4
    gravity = config["gravity"]
    solver = _factory(variant)(p, config)
    try:
        solver.step_batch(steps, dt, gravity)
        solver.check_numerical_status()
        packed, _ = solver.read_particles_packed()
    finally:
        solver.dispose()
    cfg = dict(config, dt=float(np.float32(dt)))
    state = OracleState(p, cfg)
    state.run(cfg, steps)
    gpu, ref = packed_columns(packed), oracle_columns(state)
    assert np.max(np.abs(gpu["position"] - ref["position"])) <= 0.02
    excess = np.abs(gpu["velocity"] - ref["velocity"]) - (0.025 + 5e-4 * np.abs(ref["velocity"]))
    assert np.max(excess) <= 0.0, np.max(excess)
    solids = np.nonzero(p.material == 2)[0]
    assert np.max(np.abs(packed[solids, 18] - state.particles["damage"][solids])) <= 1e-3


def test_si_tank_600_macrosteps_water_diagnostics_match_the_oracle():
    with open(os.path.join(HERE, "golden", "si_tank_long_fp64.json")) as f:
        golden = json.load(f)
    p, config = create_si_tank_scene(seed=1)
    solver = create_mpm_mls_gpu_solver(p, config)
    steps = golden["microstepsPerMacrostep"]
    try:
        got = [summarize_si_water(solver.read_particles_packed()[0], golden["referenceArea"])]
        for macro in range(1, golden["macrosteps"] + 1):
            solver.step_batch(steps, golden["microDt"], SI_TANK_GRAVITY)
            if macro % golden["every"] == 0:
                solver.check_numerical_status()
                got.append(summarize_si_water(solver.read_particles_packed()[0], golden["referenceArea"]))
    finally:
        solver.dispose()
    assert len(got) == len(golden["diagnostics"])
    for k, (g, r) in enumerate(zip(got, golden["diagnostics"])):
        for key, (absolute, relative) in LONG_HORIZON_BOUNDS.items():
            assert abs(g[key] - r[key]) <= absolute + relative * abs(r[key]), (k * golden["every"], key, g[key], r[key])
