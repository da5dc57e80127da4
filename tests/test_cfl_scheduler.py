"""Host CFL policy and scheduler: the reference's known answers.

Cases from src/lib/mpm/kernels/cfl.spec.ts, cfl-bounds.spec.ts and
step-scheduler.spec.ts (7korobi/powder-play).
"""
import math
import sys

import numpy as np
import pytest

from mpm_b200 import (RangeError, calculate_mpm_cfl_microsteps, calculate_mpm_cfl_safe_dt,
                      calculate_mpm_cfl_velocity_limit, calculate_mpm_step_batch, derive_mpm_mls_gpu_cfl_bounds,
                      particles_from_dicts)
from mpm_b200.layout import fround
from mpm_b200.scenes import (GATE4_GRID, GATE4_PARTICLE_AREA, GATE4_SOLID_PARTICLE_MASS, create_mpm_gate4_scene,
                             create_si_fluid_scene)

BASE = dict(macroDt=0.025, cellSize=0.1, waveSpeedBound=2, velocityBound=1, maxMicrosteps=3)


def test_safe_dt():
    # cfl.spec.ts:19-25
    assert calculate_mpm_cfl_safe_dt(0.1, 2, 1) == pytest.approx(0.3 * 0.1 / 3)


def test_default_plan():
    # cfl.spec.ts:27-36
    plan = calculate_mpm_cfl_microsteps(**BASE)
    assert plan["stepCount"] == 3
    assert plan["safeDt"] == pytest.approx(0.3 * 0.1 / 3)
    assert plan["microDt"] == pytest.approx(0.025 / 3)
    assert plan["microDt"] <= plan["safeDt"]


def test_certified_minimum_count():
    # cfl.spec.ts:38-53
    plan = calculate_mpm_cfl_microsteps(**dict(BASE, maxMicrosteps=6), minimumStepCount=5)
    assert plan["stepCount"] == 5
    with pytest.raises(RangeError, match=r"required microstep count .* exceeds maxMicrosteps"):
        calculate_mpm_cfl_microsteps(**dict(BASE, maxMicrosteps=4), minimumStepCount=5)


def test_custom_courant_limit_exact_plan():
    # cfl.spec.ts:55-70: exact {3, 0.25/3, 0.1}
    plan = calculate_mpm_cfl_microsteps(0.25, 1, 2, 3, 3, courantLimit=0.5)
    assert plan == {"stepCount": 3, "microDt": 0.25 / 3, "safeDt": 0.1}


def test_float32_micro_dt_within_safe_dt():
    # cfl.spec.ts:72-84
    plan = calculate_mpm_cfl_microsteps(1, 1, 4, 6, 11, courantLimit=1)
    assert plan["stepCount"] == 11
    assert fround(plan["microDt"]) <= plan["safeDt"]


def test_velocity_limit():
    # cfl.spec.ts:86-99
    limit = calculate_mpm_cfl_velocity_limit(10, 1400, 0.001, 0.3)
    assert fround(limit) == limit
    assert (limit + fround(1400)) * fround(0.001) <= 0.3 * fround(10)
    assert limit > 1599


def test_velocity_limit_rejections():
    # cfl.spec.ts:101-131
    with pytest.raises(RangeError, match="no finite non-negative CFL velocity allowance"):
        calculate_mpm_cfl_velocity_limit(10, 400, 0.01)
    for args in ((0, 1, 0.01), (10, math.inf, 0.01), (10, 1, 0)):
        with pytest.raises(RangeError):
            calculate_mpm_cfl_velocity_limit(*args)


def test_zero_speed_bounds_use_one_step():
    # cfl.spec.ts:133-146
    plan = calculate_mpm_cfl_microsteps(**dict(BASE, macroDt=0.1, waveSpeedBound=0, velocityBound=0, maxMicrosteps=1))
    assert plan == {"stepCount": 1, "microDt": 0.1, "safeDt": math.inf}


def test_required_count_beyond_limit_throws():
    # cfl.spec.ts:148-156
    with pytest.raises(RangeError, match=r"required microstep count .* exceeds maxMicrosteps"):
        calculate_mpm_cfl_microsteps(**dict(BASE, maxMicrosteps=2))


def test_overflowing_intermediates():
    # cfl.spec.ts:158-178
    s = calculate_mpm_cfl_microsteps(0.1, sys.float_info.max, sys.float_info.max, sys.float_info.max, 1)
    p = calculate_mpm_cfl_microsteps(1e30, sys.float_info.max, 1, 1, 1, courantLimit=2)
    assert s["safeDt"] == pytest.approx(0.15, abs=1e-14)
    assert s["microDt"] <= s["safeDt"]
    assert p["safeDt"] == sys.float_info.max
    assert p["microDt"] <= p["safeDt"]


def test_unrepresentable_float32_microsteps():
    # cfl.spec.ts:180-190
    with pytest.raises(RangeError, match=r"required float32 microstep count .* exceeds maxMicrosteps"):
        calculate_mpm_cfl_microsteps(sys.float_info.max, 1, 0, 0, 2 ** 53 - 1)


@pytest.mark.parametrize("overrides", [
    {"macroDt": 0}, {"macroDt": math.nan}, {"macroDt": math.inf}, {"cellSize": 0}, {"cellSize": math.nan},
    {"waveSpeedBound": -1}, {"waveSpeedBound": math.inf}, {"velocityBound": -1}, {"velocityBound": math.nan},
    {"courantLimit": 0}, {"courantLimit": math.inf}, {"maxMicrosteps": 0}, {"maxMicrosteps": 1.5},
    {"maxMicrosteps": 2 ** 53},
])
def test_invalid_inputs(overrides):
    # cfl.spec.ts:192-217
    with pytest.raises(RangeError):
        calculate_mpm_cfl_microsteps(**dict(BASE, **overrides))


def test_scheduler_plans_complete_microsteps():
    # step-scheduler.spec.ts:12-34
    b = calculate_mpm_step_batch(0, 0.05, 1, 0.025, 0.1, 2, 1, 6)
    assert b["macroStepCount"] == 2 and b["microstepPlan"]["stepCount"] == 3 and b["microStepCount"] == 6
    assert b["simulatedSeconds"] == 0.05
    assert b["remainderSeconds"] == pytest.approx(0)


@pytest.mark.parametrize("speed,expected", [(0.5, 2), (1, 4), (2, 8), (4, 16)])
def test_scheduler_acceleration(speed, expected):
    # step-scheduler.spec.ts:36-56
    b = calculate_mpm_step_batch(0, 1 / 60, speed, 1 / 240, 0.1, 20, 1, 64)
    assert b["macroStepCount"] == expected and b["microstepPlan"]["stepCount"] == 3
    assert b["microStepCount"] == expected * 3


def test_scheduler_keeps_fractional_time():
    # step-scheduler.spec.ts:58-84
    half = 0.025 / 2
    first = calculate_mpm_step_batch(0, half, 1, 0.025, 0.1, 2, 1, 6)
    second = calculate_mpm_step_batch(first["remainderSeconds"], half, 1, 0.025, 0.1, 2, 1, 6)
    assert first["macroStepCount"] == 0 and first["microStepCount"] == 0
    assert first["remainderSeconds"] == pytest.approx(half)
    assert second["macroStepCount"] == 1 and second["microStepCount"] == 3
    assert second["remainderSeconds"] == pytest.approx(0)


def test_gate4_wave_speed_bound_from_the_seeded_scene():
    # cfl-bounds.spec.ts:21-38
    p, _, _ = create_mpm_gate4_scene(0x4C414234)
    config = {"particleMass": GATE4_SOLID_PARTICLE_MASS, "particleVolume": GATE4_PARTICLE_AREA,
              "material": {"lambda": 20, "mu": 10, "model": "neo-hookean"}}
    bounds = derive_mpm_mls_gpu_cfl_bounds(p, config)
    speed = float(np.max(np.hypot(p.vx.astype(np.float32), p.vy.astype(np.float32))))
    assert bounds["waveSpeedBound"] >= math.sqrt(160_000 / 0.02)
    assert bounds["waveSpeedBound"] == pytest.approx(math.sqrt(160_000 / 0.02), abs=5e-3)
    assert speed <= bounds["velocityBound"] < speed + 0.01


def test_neo_hookean_and_tait_bounds():
    # cfl-bounds.spec.ts:40-86
    config = {"particleMass": 4, "particleVolume": 100, "material": {"lambda": 20, "mu": 10, "model": "neo-hookean"}}
    base = {"position": {"x": 1, "y": 1}, "velocity": {"x": 0, "y": 0},
            "C": {"m00": 0, "m01": 0, "m10": 0, "m11": 0}, "F": {"m00": 1, "m01": 0, "m10": 0, "m11": 1}}
    ref = derive_mpm_mls_gpu_cfl_bounds(particles_from_dicts([base]), config)
    stretched = derive_mpm_mls_gpu_cfl_bounds(particles_from_dicts([dict(base, F={"m00": 2, "m01": 0, "m10": 0,
                                                                                  "m11": 1})]), config)
    assert ref["waveSpeedBound"] == pytest.approx(math.sqrt(40 / 0.04), abs=5e-5)
    assert stretched["waveSpeedBound"] > ref["waveSpeedBound"]
    water = {"lambda": ((998.2 * 400) / 7.15) * 0.02, "mu": 0, "model": "water", "density": 998.2 * 0.02,
             "equationOfState": {"model": "tait", "exponent": 7.15}}
    tref = derive_mpm_mls_gpu_cfl_bounds(particles_from_dicts([dict(base, material=water)]), config)
    tcomp = derive_mpm_mls_gpu_cfl_bounds(particles_from_dicts([dict(base, material=water, F={
        "m00": 0.9, "m01": 0, "m10": 0, "m11": 1})]), config)
    assert tref["waveSpeedBound"] == pytest.approx(20, abs=5e-3)
    assert tcomp["waveSpeedBound"] > tref["waveSpeedBound"]


def test_unsupported_models_have_no_bound():
    # cfl-bounds.spec.ts:88-110
    config = {"particleMass": 4, "particleVolume": 100,
              "material": {"lambda": 4, "mu": 2, "model": "powder", "frictionCoefficient": 0.5}}
    assert derive_mpm_mls_gpu_cfl_bounds([], config) == {"waveSpeedBound": 0.0, "velocityBound": 0.0}
    p = {"position": {"x": 0, "y": 0}, "velocity": {"x": 0, "y": 0},
         "C": {"m00": 0, "m01": 0, "m10": 0, "m11": 0}, "F": {"m00": 1, "m01": 0, "m10": 0, "m11": 1}}
    assert derive_mpm_mls_gpu_cfl_bounds(particles_from_dicts([p]), config) is None


def test_si_fluid_scene_layout():
    # si-fluid.spec.ts:14-38: 80x20 = 1,600 particles, first at (1.25 mm, 151.25 mm)
    p, config = create_si_fluid_scene()
    assert len(p) == 1600
    assert p.px[0] == pytest.approx(0.00125) and p.py[0] == pytest.approx(0.15125)
    assert config["grid"] == {"cellsX": 40, "cellsY": 40, "cellSize": 0.005}
    assert config["material"]["equationOfState"]["exponent"] == 7.15


def test_gate4_scene_counts_and_probes():
    # gate4.spec.ts: 3,674 particles, 53 fracture bonds, probe indices
    p, bonds, probes = create_mpm_gate4_scene()
    assert len(p) == 3674 and len(bonds) == 53
    assert probes == [25, 3475, 3586]
    assert GATE4_GRID == {"cellsX": 220, "cellsY": 150, "cellSize": 10}
