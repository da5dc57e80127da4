"""CUDA path vs the oracle, through the C ABI (libmpm_b200.so).

Tolerances:
* the 45-particle, 5-model transfer fixture: max |GPU - FP64 oracle| <= 1e-3
  over 8 steps, the bound of src/lib/mpm/experiments/transfer-regression.ts:29;
  batch-of-8 vs 8 single steps identical (:80-91);
* sort, indexing and fixed-point P2G integers: bit-exact;
* scenes: positions within 1e-3 cell sizes and velocities within
  1e-3 * (1 + |v|) (in cell sizes per step-time units, see each test) of the
  FP64 oracle stepping the same microDt sequence.
"""
import math

import numpy as np
import pytest

from helpers import (max_abs_difference, oracle_columns, packed_columns, transfer_regression_fixture)
from mpm_b200 import (MpmMlsGpuNumericalError, calculate_mpm_cfl_microsteps, create_experimental_mpm_mls_atomic_gpu_solver,
                      create_mpm_mls_gpu_solver, particles_from_dicts)
from mpm_b200.cfl_bounds import calculate_mpm_cfl_velocity_bound
from mpm_b200.layout import ParticleArrays, validate_mpm_mls_gpu_input
from mpm_b200.scenes import (DAM_BREAK_GRAVITY, GATE4_FIXED_STEP_SECONDS, create_dam_break_scene,
                              create_mpm_gate4_scene, create_mpm_gate4_step_config, create_si_fluid_scene,
                              create_si_tank_scene)
from oracle import OracleState, emulate_fixed_point_scatter

pytestmark = pytest.mark.gpu

FACTORIES = {"gather": create_mpm_mls_gpu_solver, "atomic": create_experimental_mpm_mls_atomic_gpu_solver}


@pytest.mark.parametrize("variant", ["gather", "atomic"])
def test_transfer_regression_fixture_matches_the_oracle(variant):
    particles, config = transfer_regression_fixture()
    dt, gravity = 0.001, {"x": 0, "y": 0}
    state = OracleState(particles_from_dicts(particles), dict(config, dt=dt, gravity=gravity))
    for _ in range(8):
        state.step(dict(config, dt=dt, gravity=gravity))
    factory = FACTORIES[variant]
    batched = factory(particles, config)
    try:
        batched.step_batch(8, dt, gravity)
        packed_batch, _ = batched.read_particles_packed()
    finally:
        batched.dispose()
    singles = factory(particles, config)
    try:
        for _ in range(8):
            singles.step(dt, gravity)
        packed_single, _ = singles.read_particles_packed()
    finally:
        singles.dispose()
    err = max_abs_difference(oracle_columns(state), packed_columns(packed_batch))
    assert err <= 1e-3, f"{variant}: GPU vs FP64 oracle {err}"
    assert np.array_equal(packed_batch.view(np.uint32), packed_single.view(np.uint32))


def test_cell_sort_is_a_bit_exact_stable_counting_sort():
    p, config = create_si_tank_scene(seed=7)
    solver = create_mpm_mls_gpu_solver(p, config)
    try:
        keys, perm, starts = solver.probe_sort(1e-4)
        state = validate_mpm_mls_gpu_input(p, config)
    finally:
        solver.dispose()
    pos = state.packed_particles[:, 0:2]
    dx = np.float32(config["grid"]["cellSize"])
    g = (pos / dx).astype(np.float32)
    base = np.floor((g - np.float32(0.5)).astype(np.float32)).astype(np.int64)
    width = config["grid"]["cellsX"] + 3
    expected_keys = (base[:, 1] + 1) * width + (base[:, 0] + 1)
    assert np.array_equal(keys.astype(np.int64), expected_keys)
    expected_perm = np.argsort(expected_keys, kind="stable")
    assert np.array_equal(perm.astype(np.int64), expected_perm)
    counts = np.bincount(expected_keys, minlength=starts.size - 1)
    assert np.array_equal(starts.astype(np.int64), np.concatenate(([0], np.cumsum(counts))))


def test_cell_sort_stays_canonical_after_steps():
    # after the slots have been re-sorted by several substeps, the sort is still
    # the stable counting sort of the particles in their original order
    p, config = create_si_tank_scene(seed=9)
    solver = create_mpm_mls_gpu_solver(p, config)
    try:
        solver.step_batch(7, 2e-4, {"x": 0.0, "y": -9.81})
        packed, _ = solver.read_particles_packed()
        keys, perm, starts = solver.probe_sort(2e-4)
    finally:
        solver.dispose()
    dx = np.float32(config["grid"]["cellSize"])
    g = (packed[:, 0:2] / dx).astype(np.float32)
    base = np.floor((g - np.float32(0.5)).astype(np.float32)).astype(np.int64)
    expected_keys = (base[:, 1] + 1) * (config["grid"]["cellsX"] + 3) + (base[:, 0] + 1)
    assert np.array_equal(keys.astype(np.int64), expected_keys)
    assert np.array_equal(perm.astype(np.int64), np.argsort(expected_keys, kind="stable"))


def _mixed_liquid_scene(seed=3, n_side=48):
    rng = np.random.default_rng(seed)
    n = n_side * n_side
    p = ParticleArrays.empty(n)
    r, c = np.divmod(np.arange(n), n_side)
    p.px[:] = 40 + c * 5.0 + rng.uniform(-1, 1, n)
    p.py[:] = 40 + r * 5.0 + rng.uniform(-1, 1, n)
    p.vx[:] = rng.uniform(-3, 3, n)
    p.vy[:] = rng.uniform(-3, 3, n)
    p.C[:] = rng.uniform(-0.05, 0.05, (n, 4))
    p.volume[:] = 25.0
    water = {"lambda": 160_000, "mu": 0, "model": "water", "density": 0.02}
    oil = {"lambda": 120_000, "mu": 0, "model": "oil", "density": 0.016}
    p.materials = [water, oil]
    p.material[:] = (r >= n_side // 2).astype(np.int32)
    config = {"grid": {"cellsX": 40, "cellsY": 40, "cellSize": 10}, "particleMass": 0.5, "particleVolume": 25,
              "material": water}
    return p, config


def test_fixed_point_integers_match_the_cpu_emulation_bit_for_bit():
    p, config = _mixed_liquid_scene()
    solver = create_experimental_mpm_mls_atomic_gpu_solver(p, config, fixed_point_shift=20)
    try:
        words, affine = solver.probe_fixed_point(1e-4)
        state = validate_mpm_mls_gpu_input(p, config)
    finally:
        solver.dispose()
    expected, flags = emulate_fixed_point_scatter(state.packed_particles, affine, state.cell_size_f32,
                                                  state.particle_mass_f32, state.particle_volume_f32, 40, 40, 20)
    assert flags == 0
    assert np.count_nonzero(words) > 0
    assert np.array_equal(words, expected)


@pytest.mark.parametrize("contribution_overflow", [False, True])
def test_fixed_point_overflow_sets_65536_and_rolls_back_bitwise(contribution_overflow):
    # runMpmAtomicOverflowRegression, transfer-regression.ts:97-170
    p, config = create_si_fluid_scene()
    count = 1 if contribution_overflow else 512
    base = p.take([0] * count)
    base.px[:] = 0.1
    base.py[:] = 0.1
    base.vx[:] = 1e7 if contribution_overflow else 0.0
    solver = create_experimental_mpm_mls_atomic_gpu_solver(base, config)
    try:
        state = validate_mpm_mls_gpu_input(base, config)
        solver.step(1e-5, {"x": 0, "y": 0})
        for _ in range(2):
            with pytest.raises(MpmMlsGpuNumericalError) as info:
                solver.check_numerical_status()
            assert info.value.flags == 65536
        status = solver.read_status_words()
        assert status[0] == 65536
        # the rolled-back state equals the uploaded state bit for bit (read
        # through the C ABI directly: readParticles rejects while status != 0)
        from mpm_b200 import _lib
        packed = np.zeros((count, 20), dtype=np.float32)
        ids = np.zeros(count, dtype=np.uint32)
        rc = solver._lib.mpm_read_particles(solver._handle, None, count, _lib.ptr(packed), _lib.ptr(ids))
        assert rc == 0
        assert np.array_equal(packed.view(np.uint32), state.packed_particles.view(np.uint32))
    finally:
        solver.dispose()


def _run_parity(p, config, gravity, micro_dt, steps, factory):
    solver = factory(p, config)
    try:
        solver.step_batch(steps, micro_dt, gravity)
        packed, _ = solver.read_particles_packed()
    finally:
        solver.dispose()
    state = OracleState(p, dict(config, dt=float(np.float32(micro_dt)), gravity=gravity))
    state.run(dict(config, dt=float(np.float32(micro_dt)), gravity=gravity), steps)
    return packed_columns(packed), oracle_columns(state)


@pytest.mark.parametrize("variant", ["gather", "atomic"])
def test_si_fluid_scene_matches_the_oracle(variant):
    p, config = create_si_fluid_scene()
    gravity = {"x": 0.0, "y": 9.81}
    plan = calculate_mpm_cfl_microsteps(1 / 120, config["grid"]["cellSize"], 20.01, 0.0, 512)
    gpu, ref = _run_parity(p, config, gravity, plan["microDt"], 40, FACTORIES[variant])
    dx = config["grid"]["cellSize"]
    pos_err = np.max(np.abs(gpu["position"] - ref["position"]))
    vel_err = np.max(np.abs(gpu["velocity"] - ref["velocity"]) / (1 + np.abs(ref["velocity"])))
    assert pos_err <= 1e-3 * dx, pos_err
    assert vel_err <= 1e-3, vel_err


def test_si_tank_scene_matches_the_oracle_and_is_deterministic():
    p, config = create_si_tank_scene(seed=1)
    gravity = {"x": 0.0, "y": -9.81}
    plan = calculate_mpm_cfl_microsteps(1 / 120, config["grid"]["cellSize"], 20.01, 0.0, 512)
    gpu, ref = _run_parity(p, config, gravity, plan["microDt"], 60, create_mpm_mls_gpu_solver)
    dx = config["grid"]["cellSize"]
    assert np.max(np.abs(gpu["position"] - ref["position"])) <= 1e-3 * dx
    again, _ = _run_parity(p, config, gravity, plan["microDt"], 60, create_mpm_mls_gpu_solver)
    for key in gpu:
        assert np.array_equal(gpu[key], again[key])


def _crowded_scene(per_side, seed=5):
    # a 16 x 8-cell block at per_side^2 particles per cell: more particles in
    # one tile than the P2G stages at once (640), and at per_side 8 more than
    # that in a single cell row
    rng = np.random.default_rng(seed)
    dx = 10.0
    spacing = dx / per_side
    nx, ny = 16 * per_side, 8 * per_side
    r, c = np.divmod(np.arange(nx * ny), nx)
    p = ParticleArrays.empty(nx * ny)
    p.px[:] = 60 + (c + 0.5) * spacing + rng.uniform(-0.1, 0.1, nx * ny) * spacing
    p.py[:] = 60 + (r + 0.5) * spacing + rng.uniform(-0.1, 0.1, nx * ny) * spacing
    p.vx[:] = rng.uniform(-2, 2, nx * ny)
    p.vy[:] = rng.uniform(-2, 2, nx * ny)
    water = {"lambda": 40_000, "mu": 0, "model": "water", "density": 0.02}
    oil = {"lambda": 30_000, "mu": 0, "model": "oil", "density": 0.016}
    p.materials = [water, oil]
    p.material[:] = (c >= nx // 2).astype(np.int32)
    p.volume[:] = spacing * spacing
    config = {"grid": {"cellsX": 40, "cellsY": 40, "cellSize": dx}, "particleMass": 0.02 * spacing * spacing,
              "particleVolume": spacing * spacing, "material": water}
    return p, config


@pytest.mark.parametrize("per_side", [5, 8])
def test_crowded_tiles_match_the_oracle(per_side):
    p, config = _crowded_scene(per_side)
    gravity = {"x": 0.0, "y": -9.81}
    gpu, ref = _run_parity(p, config, gravity, 2e-4, 12, create_mpm_mls_gpu_solver)
    dx = config["grid"]["cellSize"]
    assert np.max(np.abs(gpu["position"] - ref["position"])) <= 1e-3 * dx
    vel_err = np.max(np.abs(gpu["velocity"] - ref["velocity"]) / (1 + np.abs(ref["velocity"])))
    assert vel_err <= 1e-3, vel_err
    if per_side == 5:
        # tiles taken in chunks of whole cell rows keep a fixed summation order
        again, _ = _run_parity(p, config, gravity, 2e-4, 12, create_mpm_mls_gpu_solver)
        for key in gpu:
            assert np.array_equal(gpu[key], again[key])


def _gate4_float32():
    # the Gate 4 scene with positions and velocities already float32, so the
    # oracle and the device start from the same values
    p, bonds, probes = create_mpm_gate4_scene()
    for a in (p.px, p.py, p.vx, p.vy):
        a[:] = a.astype(np.float32)
    return p, bonds, probes


def test_triangle_field_matches_the_oracle():
    # buildTriangleField of the 50 pebbles at the start of the scene; the
    # device samples in float64 with the CPU reference's operations
    p, bonds, _ = _gate4_float32()
    config = create_mpm_gate4_step_config(fracture_bonds=bonds)
    solver = create_mpm_mls_gpu_solver(p, config)
    try:
        gpu = solver.probe_triangle_field(GATE4_FIXED_STEP_SECONDS / 16)
    finally:
        solver.dispose()
    ref = OracleState(p, config).triangle_field(config)
    near = ref["body"] >= 0
    assert near.sum() > 0
    assert np.array_equal(gpu["body"], ref["body"])  # ties included (the pebbles sit on a lattice)
    # float32 storage of the float64 samples
    assert np.max(np.abs(gpu["sd"] - ref["sd"]) / (1 + np.abs(ref["sd"]))) <= 1e-6
    assert np.max(np.abs(gpu["normal"][near] - ref["normal"][near])) <= 1e-6
    assert np.max(np.abs(gpu["bary"][near] - ref["bary"][near])) <= 1e-6


@pytest.mark.parametrize("variant", ["gather", "atomic"])
def test_gate4_pebbles_and_fracture_match_the_oracle(variant):
    # the reference's multi-material scene: 2,000 water, 1,500 oil, 50 bonded
    # triangle pebbles (fluid contact, bonded edges, pair contacts) and a
    # fractured Neo-Hookean block (53 bonds); fixed microsteps of 1/3840 s
    p, bonds, probes = _gate4_float32()
    config = create_mpm_gate4_step_config(fracture_bonds=bonds)
    # the scene's CFL microstep (about five per 1/240 s macrostep): the bonded
    # edges turn position rounding into velocity by 1/dt, and pebble contacts
    # switch on thresholds, so float32 and float64 runs part after a few
    # microsteps; compare over 4 with the reference's own CPU-vs-GPU bounds
    dt = GATE4_FIXED_STEP_SECONDS / 5
    steps = 4
    gravity = config["gravity"]
    # the reference's 2^24 fixed-point scale overflows at these velocities
    solver = (create_mpm_mls_gpu_solver(p, config) if variant == "gather"
              else create_experimental_mpm_mls_atomic_gpu_solver(p, config, fixed_point_shift=16))
    try:
        solver.step_batch(steps, dt, gravity)
        packed, _ = solver.read_particles_packed()
    finally:
        solver.dispose()
    cfg = dict(config, dt=float(np.float32(dt)))
    state = OracleState(p, cfg)
    state.run(cfg, steps)
    gpu, ref = packed_columns(packed), oracle_columns(state)
    # src/routes/labs/mpm/kernels/+page.svelte:120-122: position 0.02,
    # velocity 0.025 + 5e-4 |v|
    assert np.max(np.abs(gpu["position"] - ref["position"])) <= 0.02
    excess = np.abs(gpu["velocity"] - ref["velocity"]) - (0.025 + 5e-4 * np.abs(ref["velocity"]))
    assert np.max(excess) <= 0.0, np.max(excess)
    # fracture damage of the Neo-Hookean particles (packed word 18)
    solids = np.nonzero(p.material == 2)[0]
    assert np.max(np.abs(packed[solids, 18] - state.particles["damage"][solids])) <= 1e-3


def _fracture_block(cols=8, rows=4, spacing=5.0):
    # a bonded Neo-Hookean block whose halves move apart (updateFractureBonds /
    # applyFractureParticleDamage): bonds strain, gather damage and break
    n = cols * rows
    p = ParticleArrays.empty(n)
    r, c = np.divmod(np.arange(n), cols)
    p.px[:] = 100 + c * spacing
    p.py[:] = 100 + r * spacing
    p.vx[:] = np.where(c < cols // 2, -150.0, 150.0)
    p.object_id[:] = 1
    p.volume[:] = spacing * spacing
    p.plastic_volume[:] = 1.0
    nh = {"lambda": 2000.0, "mu": 1000.0, "model": "neo-hookean"}
    p.materials = [nh]
    p.material[:] = 0
    bonds = []
    for k in range(n):
        rr, cc = divmod(k, cols)
        if cc + 1 < cols:
            bonds.append({"firstParticle": k, "secondParticle": k + 1, "restLength": spacing, "failureStrain": 0.12})
        if rr + 1 < rows:
            bonds.append({"firstParticle": k, "secondParticle": k + cols, "restLength": spacing,
                          "failureStrain": 0.12})
    config = {"grid": {"cellsX": 40, "cellsY": 40, "cellSize": 10}, "particleMass": 0.5, "particleVolume": 25,
              "material": nh, "fractureBonds": bonds, "gravity": {"x": 0.0, "y": 0.0}}
    return p, config


def test_fracture_damage_matches_the_oracle():
    p, config = _fracture_block()
    gravity = config["gravity"]
    solver = create_mpm_mls_gpu_solver(p, config)
    try:
        solver.step_batch(60, 2e-4, gravity)
        packed, _ = solver.read_particles_packed()
    finally:
        solver.dispose()
    cfg = dict(config, dt=float(np.float32(2e-4)))
    state = OracleState(p, cfg)
    state.run(cfg, 60)
    assert int(state.bonds["broken"].sum()) > 0  # the case reaches broken bonds
    ref = state.particles["damage"]
    assert np.max(np.abs(packed[:, 18] - ref)) <= 1e-3
    gpu = packed_columns(packed)
    assert np.max(np.abs(gpu["position"] - oracle_columns(state)["position"])) <= 1e-3 * 10


def test_multi_material_models_match_the_oracle():
    # all five reference models plus fixed-corotated in one scene
    materials = [{"model": "neo-hookean", "lambda": 20, "mu": 10}, {"model": "snow", "lambda": 20, "mu": 10},
                 {"model": "water", "lambda": 8, "mu": 0, "density": 1},
                 {"model": "oil", "lambda": 6, "mu": 0, "density": 0.8,
                  "equationOfState": {"model": "tait", "exponent": 7.0}},
                 {"model": "powder", "lambda": 20, "mu": 10, "frictionCoefficient": 0.55},
                 {"model": "fixed-corotated", "lambda": 20, "mu": 10}]
    rng = np.random.default_rng(11)
    parts = []
    for group, material in enumerate(materials):
        for local in range(16):
            parts.append({"position": {"x": 4 + group * 7 + (local % 4) * 0.5 + rng.uniform(0, 0.2),
                                       "y": 4 + (local // 4) * 0.5 + rng.uniform(0, 0.2)},
                          "velocity": {"x": rng.uniform(-0.5, 0.5), "y": rng.uniform(-0.5, 0.5)},
                          "C": {"m00": 0, "m01": 0.01, "m10": 0, "m11": 0},
                          "F": {"m00": 0.99, "m01": 0.01, "m10": 0, "m11": 1.01},
                          "material": material, "objectId": group + 1, "plasticVolume": 1})
    config = {"grid": {"cellsX": 48, "cellsY": 16, "cellSize": 1}, "particleMass": 0.1, "particleVolume": 0.05,
              "material": materials[0]}
    for factory in (create_mpm_mls_gpu_solver, create_experimental_mpm_mls_atomic_gpu_solver):
        gpu, ref = _run_parity(particles_from_dicts(parts), config, {"x": 0, "y": -1}, 1e-3, 20, factory)
        assert max_abs_difference(gpu, ref) <= 1e-3


def test_cfl_adaptive_batches_commit_every_microstep():
    p, config = create_si_fluid_scene()
    gravity = {"x": 0.0, "y": 9.81}
    solver = create_mpm_mls_gpu_solver(p, config)
    try:
        velocity = solver.cfl_bounds["velocityBound"]
        for _ in range(5):
            # a recovered retry may raise the wave-speed bound: plan with the current one
            bounds = solver.cfl_bounds
            # the scheduler's velocity envelope: current bound + |g| * duration
            envelope = calculate_mpm_cfl_velocity_bound(velocity, 1 / 120, 9.81, 0, 0, 0, 0)
            plan = calculate_mpm_cfl_microsteps(1 / 120, config["grid"]["cellSize"], bounds["waveSpeedBound"],
                                                envelope, 512)
            before = solver.committed_microsteps_total
            m = solver.step_cfl_batch_adaptive(1, 1 / 120, plan, envelope, 512, gravity)
            assert m["remainingDuration"] == 0
            assert m["attemptedMicroStepCount"] >= plan["stepCount"]
            assert solver.committed_microsteps_total - before >= plan["stepCount"]
            velocity = m["recommendedVelocityBound"]
        assert 0 < velocity < 5
    finally:
        solver.dispose()


def test_cfl_violation_rolls_back_and_retries_at_a_finer_step():
    # a strong body force makes particles exceed the planned velocity bound
    p, config = create_si_fluid_scene()
    gravity = {"x": 0.0, "y": 4000.0}
    solver = create_mpm_mls_gpu_solver(p, config)
    try:
        bounds = solver.cfl_bounds
        plan = calculate_mpm_cfl_microsteps(1 / 120, config["grid"]["cellSize"], bounds["waveSpeedBound"], 0.5, 512)
        m = solver.step_cfl_batch_adaptive(1, 1 / 120, plan, 0.5, 512, gravity)
        assert m["retryCount"] >= 1
        packed, _ = solver.read_particles_packed()
        assert np.all(np.isfinite(packed[:, :12]))
    finally:
        solver.dispose()


def test_dam_break_scale_scene_runs_and_conserves_particles():
    p, config = create_dam_break_scene(particles_per_phase=125_000, columns=250)
    solver = create_mpm_mls_gpu_solver(p, config)
    try:
        bounds = solver.cfl_bounds
        plan = calculate_mpm_cfl_microsteps(1 / 240, 10, bounds["waveSpeedBound"], 5.0, 64)
        m = solver.step_cfl_batch_adaptive(1, 1 / 240, plan, 5.0, 64, DAM_BREAK_GRAVITY)
        assert m["remainingDuration"] == 0
        packed, ids = solver.read_particles_packed()
        assert packed.shape[0] == 250_000
        assert np.all(np.isfinite(packed[:, :12]))
        assert np.all(packed[:, 1] <= 20480) and np.all(packed[:, 0] >= 0)
    finally:
        solver.dispose()
