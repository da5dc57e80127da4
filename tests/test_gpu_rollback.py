"""The whole-microstep rollback, pinned bit for bit (commitParticles,
src/lib/mpm/kernels/shaders.ts:3067-3080).

A water block falls freely under gravity g, so after k microsteps every
particle moves at k g dt (to rounding).  A CFL guard whose velocity limit
lies halfway between (done) g dt and (done + 1) g dt makes microstep
done + 1 fail, deterministically.  The state the solver keeps afterwards must
equal, bit for bit, the state of a guard-free run of exactly `done`
microsteps -- for an odd and an even `done` (the ping-pong buffers end on
different sides), in the single-scene and the batched solver -- and stepping
on from it must equal the guard-free run stepping on.
"""
import numpy as np
import pytest

from mpm_b200 import create_mpm_batched_gpu_solver, create_mpm_mls_gpu_solver
from mpm_b200.layout import ParticleArrays

pytestmark = pytest.mark.gpu

DT = 1e-3
GRAVITY = {"x": 0.0, "y": -100.0}
STEP_SPEED = 100.0 * DT  # speed gained per microstep
BATCH = 8


def _falling_block(offset=0.0, side=16):
    n = side * side
    r, c = np.divmod(np.arange(n), side)
    p = ParticleArrays.empty(n)
    p.px[:] = 28.25 + offset + 0.5 * c
    p.py[:] = 40.25 + 0.5 * r
    p.volume[:] = 0.25
    water = {"lambda": 10.0, "mu": 0.0, "model": "water", "density": 1.0}
    p.materials = [water]
    p.material[:] = 0
    config = {"grid": {"cellsX": 64, "cellsY": 64, "cellSize": 1.0}, "particleMass": 0.25, "particleVolume": 0.25,
              "material": water}
    return p, config


def _bits(packed):
    return np.ascontiguousarray(packed[:, 0:12]).view(np.uint32)


def _free_run(p, config, steps):
    solver = create_mpm_mls_gpu_solver(p, config)
    try:
        for count in steps:
            solver.step_batch(count, DT, GRAVITY)
        solver.check_numerical_status()
        return solver.read_particles_packed()[0]
    finally:
        solver.dispose()


@pytest.mark.parametrize("done", [3, 4])
def test_single_scene_rollback_equals_a_guard_free_run(done):
    p, config = _falling_block()
    limit = STEP_SPEED * (done + 0.5)
    solver = create_mpm_mls_gpu_solver(p, config)
    try:
        solver.step_batch(BATCH, DT, GRAVITY, cfl_velocity_bound=limit)
        speed, completed, status = solver._read_compact()
        assert status[0] == 16384 and status[6] == 3  # a CFL rejection with its diagnostics
        assert completed == done
        solver._clear_status()  # readParticles refuses to read while a status is raised
        rolled_back = solver.read_particles_packed()[0]
        solver.step_batch(2, DT, GRAVITY)
        solver.check_numerical_status()
        continued = solver.read_particles_packed()[0]
    finally:
        solver.dispose()
    assert np.array_equal(_bits(rolled_back), _bits(_free_run(p, config, [done])))
    assert np.array_equal(_bits(continued), _bits(_free_run(p, config, [done, 2])))
    # the rolled-back state is not the failed microstep's
    assert not np.array_equal(_bits(rolled_back), _bits(_free_run(p, config, [done + 1])))


@pytest.mark.parametrize("done", [3, 4])
def test_batched_rollback_equals_a_guard_free_run(done):
    failing = _falling_block()
    passing = _falling_block(offset=-8.0)
    batch = create_mpm_batched_gpu_solver([failing, passing])
    try:
        batch.step_batch([BATCH, BATCH], [DT, DT], GRAVITY,
                         velocity_limits=[STEP_SPEED * (done + 0.5), STEP_SPEED * (BATCH + 4)])
        _, completed, status = batch.read_compact()
        assert status[0][0] == 16384 and int(completed[0]) == done
        assert status[1][0] == 0 and int(completed[1]) == BATCH
        scene0 = batch.read_particles_packed(0)[0]
        scene1 = batch.read_particles_packed(1)[0]
        batch.clear_status()
        batch.step_batch([2, 0], [DT, DT], GRAVITY)
        assert all(e is None for e in batch.check_numerical_status())
        scene0_on = batch.read_particles_packed(0)[0]
    finally:
        batch.dispose()
    assert np.array_equal(_bits(scene0), _bits(_free_run(*failing, [done])))
    assert np.array_equal(_bits(scene1), _bits(_free_run(*passing, [BATCH])))
    assert np.array_equal(_bits(scene0_on), _bits(_free_run(*failing, [done, 2])))
