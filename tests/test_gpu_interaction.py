"""Interaction ops of the GPU solver (appendParticles, removeParticlesInOutlet,
pick, clone, drag; src/lib/mpm/kernels/solver.ts:2108-2940):

* the op itself: appended particles read back as emitted (float32), an outlet
  removes exactly the liquid particles inside it and they read back with the
  removed model, pick returns the nearest particle (lowest index among equally
  near ones), a clone reads back as its source moved by the offset;
* the state after the op steps on like the FP64 oracle started from it
  (positions within 1e-3 cell sizes over 8 substeps).
"""
import numpy as np
import pytest

from mpm_b200 import RangeError, create_mpm_mls_gpu_solver, particles_from_dicts
from mpm_b200.scenes import (SI_TANK_GRAVITY, create_mpm_emitter_particles, create_si_tank_scene)
from oracle import OracleState

pytestmark = pytest.mark.gpu

STEPS = 8


def _solver(extra_capacity=600):
    particles, config = create_si_tank_scene(seed=3)
    config = dict(config, capacity=len(particles) + extra_capacity)
    return create_mpm_mls_gpu_solver(particles, config), particles, config


def _dt(solver):
    return float(np.float32(2e-5))


def _steps_like_the_oracle(solver, config):
    """Steps the solver and the oracle started from its current state."""
    dicts = solver.read_particles()
    dt = _dt(solver)
    state = OracleState(particles_from_dicts(dicts), dict(config, dt=dt, gravity=SI_TANK_GRAVITY))
    solver.step_batch(STEPS, dt, SI_TANK_GRAVITY)
    state.run(dict(config, dt=dt, gravity=SI_TANK_GRAVITY), STEPS)
    after = solver.read_particles()
    got = np.array([[p["position"]["x"], p["position"]["y"]] for p in after])
    err = float(np.max(np.abs(got - state.positions())))
    assert err <= 1e-3 * config["grid"]["cellSize"], err


def _emitter(config, count=300, center=(0.12, 0.15), shape="rectangle"):
    return create_mpm_emitter_particles({
        "count": count, "seed": 11, "center": {"x": center[0], "y": center[1]}, "shape": shape, "spacing": 0.00125,
        "velocity": {"x": 0.05, "y": 0.0}, "material": "water", "particleVolume": config["particleVolume"],
        "grid": config["grid"]})


def test_appended_particles_read_back_and_step_like_the_oracle():
    solver, particles, config = _solver()
    try:
        emitted = _emitter(config)
        # the emitter's water takes the scene's Tait material
        for p in emitted:
            p["material"] = dict(config["material"])
        before = solver.particle_count
        result = solver.append_particles(emitted)
        assert result["accepted"] == 300 and result["refused"] == 0 and result["dropped"] == 0
        assert solver.particle_count == before + 300 == solver.allocated_particle_count
        packed, ids = solver.read_particles_packed()
        new = packed[before:]
        want = np.array([[p["position"]["x"], p["position"]["y"]] for p in emitted], dtype=np.float32)
        assert np.array_equal(new[:, 0:2], want)
        assert len(set(ids[before:].tolist())) == 1 and ids[before] not in set(ids[:before].tolist())
        _steps_like_the_oracle(solver, config)
        # capacity: the rest is dropped
        more = solver.append_particles(_emitter(config, count=400, center=(0.15, 0.15)))
        assert more["accepted"] == 300 and more["dropped"] == 100 and "capacity" in more["reason"]
    finally:
        solver.dispose()


def test_outlet_removes_the_liquid_inside_and_the_rest_steps_on():
    solver, particles, config = _solver()
    try:
        packed, _ = solver.read_particles_packed()
        bounds = {"minX": 0.0, "minY": 0.0, "maxX": 0.02, "maxY": 0.05}
        inside = ((packed[:, 0] >= 0) & (packed[:, 0] <= 0.02) & (packed[:, 1] >= 0) & (packed[:, 1] <= 0.05))
        removed = solver.remove_particles_in_outlet(bounds)
        assert removed == int(inside.sum()) > 0
        assert solver.particle_count == len(particles) - removed
        assert solver.allocated_particle_count == len(particles)
        after, _ = solver.read_particles_packed()
        model = after[:, 13].view(np.uint32)
        assert np.array_equal(model == 0xFFFFFFFF, inside)
        assert np.array_equal(after[inside, 0:2], packed[inside, 0:2])  # their last state
        assert len(solver.read_particles()) == len(particles) - removed
        with pytest.raises(RangeError):
            solver.remove_particles_in_outlet({"minX": 0.1, "minY": 0.0, "maxX": 0.05, "maxY": 0.05})
        # the kept particles step like the oracle started from them
        kept = solver.read_particles()
        dt = _dt(solver)
        state = OracleState(particles_from_dicts(kept), dict(config, dt=dt, gravity=SI_TANK_GRAVITY))
        solver.step_batch(STEPS, dt, SI_TANK_GRAVITY)
        state.run(dict(config, dt=dt, gravity=SI_TANK_GRAVITY), STEPS)
        got = np.array([[p["position"]["x"], p["position"]["y"]] for p in solver.read_particles()])
        assert float(np.max(np.abs(got - state.positions()))) <= 1e-3 * config["grid"]["cellSize"]
        # a removal blocks clones
        sel = solver.pick({"x": 0.04, "y": 0.04}, 0.01)
        assert sel is not None and solver.clone(sel, {"x": 0.05, "y": 0.05}) is False
    finally:
        solver.dispose()


def test_pick_returns_the_nearest_particle():
    solver, particles, config = _solver()
    try:
        packed, ids = solver.read_particles_packed()
        for point in ((0.01, 0.01), (0.025, 0.03), (0.049, 0.002)):
            d2 = (packed[:, 0] - np.float32(point[0])) ** 2 + (packed[:, 1] - np.float32(point[1])) ** 2
            want = int(np.argmin(d2))
            sel = solver.pick({"x": point[0], "y": point[1]}, 0.01)
            assert sel["particleIndex"] == want
            assert sel["objectId"] == int(ids[want])
            assert sel["anchor"] == {"x": float(packed[want, 0]), "y": float(packed[want, 1])}
        assert solver.pick({"x": 0.19, "y": 0.19}, 0.001) is None
    finally:
        solver.dispose()


def test_clone_copies_the_object_and_steps_like_the_oracle():
    solver, particles, config = _solver(extra_capacity=1600)
    try:
        sel = solver.pick({"x": 0.025, "y": 0.025}, 0.01)
        before, _ = solver.read_particles_packed()
        assert solver.clone(sel, {"x": 0.1, "y": 0.12}) is True
        n = len(particles)
        assert solver.allocated_particle_count == solver.particle_count == 2 * n
        after, ids = solver.read_particles_packed()
        domain = config["grid"]["cellsX"] * config["grid"]["cellSize"]
        want = np.clip(before[:, 0:2] + np.array([0.1, 0.12], dtype=np.float32), 0, np.float32(domain))
        assert np.array_equal(after[n:, 0:2], want.astype(np.float32))
        assert np.array_equal(after[n:, 2:12], before[:, 2:12])
        assert len(set(ids[n:].tolist())) == 1 and ids[n] != ids[0]
        assert solver.clone(sel, {"x": 0.0, "y": 0.0}) is False  # no capacity left
        _steps_like_the_oracle(solver, config)
    finally:
        solver.dispose()


def test_drag_pulls_toward_the_target():
    solver, particles, config = _solver()
    try:
        sel = solver.pick({"x": 0.045, "y": 0.045}, 0.01)
        solver.begin_drag(sel, {"x": 0.07, "y": 0.07}, 0.05)
        solver.step_batch(20, _dt(solver), {"x": 0.0, "y": 0.0})
        solver.end_drag()
        packed, _ = solver.read_particles_packed()
        assert float(packed[sel["particleIndex"], 2]) > 0 and float(packed[sel["particleIndex"], 3]) > 0
    finally:
        solver.dispose()
