"""The batched solver (many scenes in one handle, mpmb_* of the C ABI)
against single-scene solvers stepping the same scenes with the same dt
sequence.

A scene's tiles, sums and G2P are the same computation whether it runs alone
or inside a batch (its tile list entries only move), so positions,
velocities, C and F must agree bit for bit; so must the rollback of a scene
that fails its CFL guard, while the other scenes of the batch go on.
"""
import math

import numpy as np
import pytest

from mpm_b200 import (calculate_mpm_cfl_microsteps, calculate_mpm_cfl_velocity_limit, create_mpm_batched_gpu_solver,
                      create_mpm_mls_gpu_solver, derive_mpm_mls_gpu_cfl_bounds)
from mpm_b200.scenes import BATCHED_TANK_GRAVITY, create_batched_tank_scenes

pytestmark = pytest.mark.gpu

STATE_WORDS = slice(0, 12)  # x, v, C, F of the packed 20-word record


def _small_scenes(count=6, seed=7):
    return create_batched_tank_scenes(count, seed=seed, particles=(300, 3000), sides=(20, 96))


def _micro_dt(bounds, config, velocity, macro_dt=1 / 240):
    return calculate_mpm_cfl_microsteps(macro_dt, config["grid"]["cellSize"], bounds["waveSpeedBound"], velocity,
                                        4096)["microDt"]


def _bits(packed):
    return np.ascontiguousarray(packed[:, STATE_WORDS]).view(np.uint32)


def _wide_bounds(particles, config):
    """CFL bounds with 4x the derived wave-speed bound (the jittered lattice
    compresses some particles at once)."""
    b = derive_mpm_mls_gpu_cfl_bounds(particles, config)
    return dict(b, waveSpeedBound=4 * b["waveSpeedBound"])


def _solo_state(particles, config, submits, guard_limits=None, bounds=None):
    """Runs the scene alone: submits = [(steps, dt), ...].  Returns its packed
    particles, the status of the first failing submit (zeros if none) and
    the committed microsteps of the last guarded submit."""
    solo = create_mpm_mls_gpu_solver(particles, config, cfl_bounds=bounds)
    try:
        completed = 0
        for j, (steps, dt) in enumerate(submits):
            if steps == 0:
                continue
            limit = None if guard_limits is None else guard_limits[j]
            solo.step_batch(steps, dt, BATCHED_TANK_GRAVITY, cfl_velocity_bound=limit)
            _, completed, status = solo._read_compact()
            if status[0] != 0:
                solo._clear_status()
                return solo.read_particles_packed()[0], status, completed
        return solo.read_particles_packed()[0], np.zeros(8, np.uint32), completed
    finally:
        solo.dispose()


def test_batched_scenes_match_solo_runs_bit_for_bit():
    scenes = _small_scenes()
    batch = create_mpm_batched_gpu_solver(scenes)
    try:
        s = batch.scene_count
        dts = [_micro_dt(batch.cfl_bounds[k], scenes[k][1], 0.5) for k in range(s)]
        submits = [[(3 + k, dts[k]) for k in range(s)],
                   [(0 if k % 3 == 0 else 2 * k + 1, dts[k]) for k in range(s)],
                   [(5, dts[k] * 0.75) for k in range(s)]]
        for sub in submits:
            batch.step_batch([st for st, _ in sub], [dt for _, dt in sub], BATCHED_TANK_GRAVITY)
        assert all(e is None for e in batch.check_numerical_status())
        for k, (particles, config) in enumerate(scenes):
            got, _ = batch.read_particles_packed(k)
            want, status, _ = _solo_state(particles, config, [sub[k] for sub in submits])
            assert status[0] == 0
            assert np.array_equal(_bits(got), _bits(want)), f"scene {k} differs from its solo run"
    finally:
        batch.dispose()


def test_tiny_scenes_among_larger_ones_match_solo_runs_bit_for_bit():
    # scenes of 2 to 4 particles (a few lanes of one warp, one tile each)
    # between tanks of hundreds, some sitting a batch out
    tiny = create_batched_tank_scenes(4, seed=3, particles=(1, 40), sides=(16, 24))
    scenes = [tiny[0]] + _small_scenes(2, seed=9) + tiny[1:3] + _small_scenes(1, seed=11) + [tiny[3]]
    batch = create_mpm_batched_gpu_solver(scenes)
    try:
        s = batch.scene_count
        dts = [_micro_dt(batch.cfl_bounds[k], scenes[k][1], 0.5) for k in range(s)]
        submits = [[(2 + k % 3, dts[k]) for k in range(s)],
                   [(0 if k % 2 else 3, dts[k]) for k in range(s)]]
        for sub in submits:
            batch.step_batch([st for st, _ in sub], [dt for _, dt in sub], BATCHED_TANK_GRAVITY)
        assert all(e is None for e in batch.check_numerical_status())
        for k, (particles, config) in enumerate(scenes):
            got, _ = batch.read_particles_packed(k)
            want, status, _ = _solo_state(particles, config, [sub[k] for sub in submits])
            assert status[0] == 0
            assert np.array_equal(_bits(got), _bits(want)), f"scene {k} differs from its solo run"
    finally:
        batch.dispose()


def test_a_failing_scene_rolls_back_alone():
    scenes = _small_scenes(5, seed=11)
    bounds = [_wide_bounds(p, c) for p, c in scenes]
    batch = create_mpm_batched_gpu_solver(scenes, cfl_bounds=bounds)
    try:
        s = batch.scene_count
        dts = [_micro_dt(batch.cfl_bounds[k], scenes[k][1], 0.5) for k in range(s)]
        steps = [12, 9, 12, 7, 12]
        bad = 2
        # the guard of scene 2 trips after a few microsteps of free fall
        limits = [1e3] * s
        limits[bad] = 9.81 * dts[bad] * 3.5
        batch.step_batch(steps, dts, BATCHED_TANK_GRAVITY, limits)
        speeds, done, status = batch.read_compact()
        assert status[bad, 0] != 0 and done[bad] < steps[bad]
        # every scene, failing or not, ends exactly as it does alone
        for k, (particles, config) in enumerate(scenes):
            got, _ = batch.read_particles_packed(k)
            want, solo_status, solo_done = _solo_state(particles, config, [(steps[k], dts[k])], [limits[k]],
                                                       bounds[k])
            # flags and diagnostic kind; which failing particle claims the
            # diagnostic words is first come, first served, as in the reference
            assert status[k, 0] == solo_status[0] and status[k, 6] == solo_status[6]
            assert done[k] == solo_done
            assert np.array_equal(_bits(got), _bits(want)), f"scene {k} differs from its solo run"
        # the failed scene was rolled back to the start of its failed
        # microstep: after clearing the status it steps on like the others
        assert sum(int(status[k, 0] == 0) for k in range(s)) == s - 1
        batch.clear_status()
        batch.step_batch([2] * s, dts, BATCHED_TANK_GRAVITY)
        assert all(e is None for e in batch.check_numerical_status())
    finally:
        batch.dispose()


def test_adaptive_macrosteps_commit_each_scene_its_own_plan():
    scenes = _small_scenes(8, seed=3)
    batch = create_mpm_batched_gpu_solver(scenes)
    try:
        s = batch.scene_count
        velocity = [batch.cfl_bounds[k]["velocityBound"] for k in range(s)]
        for _ in range(3):
            results = batch.step_cfl_batch_adaptive(1 / 240, velocity, 4096, BATCHED_TANK_GRAVITY)
            velocity = [r["recommendedVelocityBound"] for r in results]
            for r in results:
                assert r["remainingDuration"] == 0.0
                assert r["committedMicroStepCount"] >= 1
                assert math.isfinite(r["maximumSpeed"])
            assert len({r["committedMicroStepCount"] for r in results}) > 1  # uneven grids, uneven plans
        for k, (particles, config) in enumerate(scenes):
            got, _ = batch.read_particles_packed(k)
            assert np.isfinite(got[:, STATE_WORDS]).all()
            size = config["grid"]["cellsX"] * config["grid"]["cellSize"]
            assert (got[:, 0] >= 0).all() and (got[:, 0] <= size).all()
            assert (got[:, 1] >= 0).all() and (got[:, 1] <= size).all()
            assert got[:, 1].mean() < particles.py.mean()  # the water falls
    finally:
        batch.dispose()


def _run_policy(scenes, factor, margin, macrosteps=3):
    """The adaptive loop under a recovery factor and a planning margin (the
    bench's policy study): returns the results of each macrostep and the
    final particles of each scene."""
    from bench import _batched_bound
    batch = create_mpm_batched_gpu_solver(scenes)
    try:
        batch.recovery_bound_factor = factor
        velocity = [batch.cfl_bounds[k]["velocityBound"] for k in range(batch.scene_count)]
        history = []
        for _ in range(macrosteps):
            bounds = [_batched_bound(v, 1 / 240, BATCHED_TANK_GRAVITY) * margin for v in velocity]
            results = batch.step_cfl_batch_adaptive(1 / 240, bounds, 4096, BATCHED_TANK_GRAVITY)
            velocity = [r["recommendedVelocityBound"] for r in results]
            history.append(results)
        return history, [batch.read_particles_packed(k)[0] for k in range(batch.scene_count)]
    finally:
        batch.dispose()


@pytest.mark.parametrize("factor,margin", [(1.5, 1.0), (2.0, 1.0), (1.25, 1.25)])
def test_a_recovery_policy_commits_every_macrostep(factor, margin):
    scenes = _small_scenes(8, seed=3)
    history, finals = _run_policy(scenes, factor, margin)
    reference_history, _ = _run_policy(scenes, 1.25, 1.0)
    for results in history:
        assert all(r["remainingDuration"] == 0.0 and r["committedMicroStepCount"] >= 1 for r in results)
    for (particles, config), got in zip(scenes, finals):
        size = config["grid"]["cellsX"] * config["grid"]["cellSize"]
        assert np.isfinite(got[:, STATE_WORDS]).all()
        assert (got[:, 0:2] >= 0).all() and (got[:, 0:2] <= size).all()
        assert got[:, 1].mean() < particles.py.mean()
    # the first macrostep starts from the same state: a scene without a retry
    # in either run plans at least as many microsteps under a margin
    for r, q in zip(history[0], reference_history[0]):
        if r["retryCount"] == 0 and q["retryCount"] == 0:
            assert (r["committedMicroStepCount"] >= q["committedMicroStepCount"]) if margin > 1.0 else \
                (r["committedMicroStepCount"] == q["committedMicroStepCount"])


def test_a_batch_of_one_scene_matches_the_plain_solver():
    (particles, config), = _small_scenes(1, seed=5)
    batch = create_mpm_batched_gpu_solver([(particles, config)])
    try:
        dt = _micro_dt(batch.cfl_bounds[0], config, 0.5)
        limit = calculate_mpm_cfl_velocity_limit(config["grid"]["cellSize"], batch.cfl_bounds[0]["waveSpeedBound"],
                                                 dt)
        batch.step_batch([9], [dt], BATCHED_TANK_GRAVITY, [limit])
        _, done, status = batch.read_compact()
        assert status[0, 0] == 0 and done[0] == 9
        got, _ = batch.read_particles_packed(0)
        want, _, _ = _solo_state(particles, config, [(9, dt)], [limit])
        assert np.array_equal(_bits(got), _bits(want))
    finally:
        batch.dispose()


def test_crowded_scenes_match_solo_runs_bit_for_bit():
    # tens of particles per cell: tiles far above one shared-memory stage,
    # taken in chunks of whole cells, still sum in a fixed order
    scenes = create_batched_tank_scenes(3, seed=21, particles=(12_000, 20_000), sides=(20, 28))
    batch = create_mpm_batched_gpu_solver(scenes)
    try:
        dts = [_micro_dt(batch.cfl_bounds[k], scenes[k][1], 0.5) for k in range(3)]
        steps = [6, 4, 5]
        batch.step_batch(steps, dts, BATCHED_TANK_GRAVITY)
        assert all(e is None for e in batch.check_numerical_status())
        for k, (particles, config) in enumerate(scenes):
            per_cell = len(particles.px) / (config["grid"]["cellsX"] ** 2)
            assert per_cell > 10
            got, _ = batch.read_particles_packed(k)
            want, status, _ = _solo_state(particles, config, [(steps[k], dts[k])])
            assert status[0] == 0
            assert np.array_equal(_bits(got), _bits(want)), f"scene {k} differs from its solo run"
    finally:
        batch.dispose()



def test_autotuned_launch_shape_changes_no_result():
    scenes = _small_scenes(4, seed=13)
    dts = None
    results = []
    for tune in (False, True):
        batch = create_mpm_batched_gpu_solver(scenes)
        try:
            dts = [_micro_dt(batch.cfl_bounds[k], scenes[k][1], 0.5) for k in range(batch.scene_count)]
            batch.step_batch([3] * batch.scene_count, dts, BATCHED_TANK_GRAVITY)
            if tune:
                before = [batch.read_particles_packed(k)[0] for k in range(batch.scene_count)]
                shape = batch.autotune(substeps=4)
                assert shape["p2gCtas"] >= 1 and shape["g2pCtas"] >= 1
                assert batch.launch_shape()["p2gCtas"] == shape["p2gCtas"]
                # the tuner restored the state it started from
                for k in range(batch.scene_count):
                    assert np.array_equal(_bits(batch.read_particles_packed(k)[0]), _bits(before[k]))
            batch.step_batch([5] * batch.scene_count, dts, BATCHED_TANK_GRAVITY)
            results.append([batch.read_particles_packed(k)[0] for k in range(batch.scene_count)])
        finally:
            batch.dispose()
    for a, b in zip(*results):
        assert np.array_equal(_bits(a), _bits(b))
