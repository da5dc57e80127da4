"""createMpmCpuParitySample (src/lib/mpm/scenes/gate4.ts:359-467) restated
in mpm_b200.scenes, checked like src/lib/mpm/scenes/gate4.spec.ts:483-593:
a local sample bigger than 110 particles and smaller than the scene with
whole bonded triangles; one FP64 CPU step of the sample reproduces the
probes' step of the full scene exactly, and three microsteps within 1e-4;
and, on the GPU, the probes of the full scene read back by index
(readParticles(indices)) against the FP64 oracle stepping only the sample,
within the reference's CPU/GPU tolerance (position 0.02, velocity
0.025 + 5e-4 |v|; src/routes/labs/mpm/kernels/+page.svelte:120-122)."""
import numpy as np
import pytest

from mpm_b200 import RangeError, create_mpm_mls_gpu_solver
from mpm_b200.scenes import (GATE4_GRID, GATE4_PARTICLE_AREA, GATE4_PEBBLE_EDGE_LENGTH, GATE4_SOLID_PARTICLE_MASS,
                             create_mpm_cpu_parity_sample, create_mpm_gate4_scene)
from oracle import OracleState


def _config(dt):
    # gate4.spec.ts:528-537 / :553-562
    return {"dt": dt, "grid": dict(GATE4_GRID), "particleMass": GATE4_SOLID_PARTICLE_MASS,
            "particleVolume": GATE4_PARTICLE_AREA, "bondRestLength": GATE4_PEBBLE_EDGE_LENGTH,
            "material": {"lambda": 20, "mu": 10, "model": "neo-hookean"}, "gravity": {"x": 0, "y": 90}}


def _values(state, index):
    p = state.particles[index]
    return np.array([p[k] for k in ("px", "py", "vx", "vy", "c00", "c01", "c10", "c11",
                                    "f00", "f01", "f10", "f11")])


@pytest.fixture(scope="module")
def scene():
    return create_mpm_gate4_scene()


def test_sample_is_local_and_keeps_whole_triangles(scene):
    particles, _, probes = scene
    sample = create_mpm_cpu_parity_sample(particles, probes, GATE4_GRID["cellSize"])
    n = len(sample["particles"])
    assert 110 < n < len(particles)
    assert len(sample["sourceIndices"]) == n and len(sample["probeSampleIndices"]) == 3
    chosen = set(sample["sourceIndices"])
    for s in sample["sourceIndices"]:
        v = int(particles.bonded_vertex[s])
        if v >= 0:
            assert {s - v, s - v + 1, s - v + 2} <= chosen
    for k, probe in enumerate(probes):
        assert sample["sourceIndices"][sample["probeSampleIndices"][k]] == probe


def test_sample_errors_match_the_reference(scene):
    particles, _, probes = scene
    with pytest.raises(RangeError, match="At least one CPU/GPU parity probe"):
        create_mpm_cpu_parity_sample(particles, [], 10)
    with pytest.raises(RangeError, match="gridCellSize"):
        create_mpm_cpu_parity_sample(particles, probes, 0)
    with pytest.raises(RangeError, match="identify input particles"):
        create_mpm_cpu_parity_sample(particles, [len(particles)], 10)


def test_one_cpu_step_of_the_sample_reproduces_the_probes(scene):
    particles, _, probes = scene
    sample = create_mpm_cpu_parity_sample(particles, probes, GATE4_GRID["cellSize"])
    config = _config(1 / 120)
    full, part = OracleState(particles, config), OracleState(sample["particles"], config)
    full.step(config)
    part.step(config)
    for k, probe in enumerate(probes):
        assert np.array_equal(_values(full, probe), _values(part, sample["probeSampleIndices"][k]))


def test_three_microsteps_keep_the_probes_within_1e4(scene):
    particles, _, probes = scene
    sample = create_mpm_cpu_parity_sample(particles, probes, GATE4_GRID["cellSize"])
    config = _config(1 / 720)
    full, part = OracleState(particles, config), OracleState(sample["particles"], config)
    for _ in range(3):
        full.step(config)
        part.step(config)
        for k, probe in enumerate(probes):
            diff = np.abs(_values(full, probe) - _values(part, sample["probeSampleIndices"][k]))
            assert diff.max() <= 1e-4


@pytest.mark.gpu
def test_gpu_probes_read_by_index_match_the_sampled_oracle(scene):
    particles, _, probes = scene
    p = particles.copy()
    for a in (p.px, p.py, p.vx, p.vy):
        a[:] = a.astype(np.float32)
    sample = create_mpm_cpu_parity_sample(p, probes, GATE4_GRID["cellSize"])
    dt = float(np.float32(1 / 720))
    config = _config(dt)
    solver = create_mpm_mls_gpu_solver(p, config)
    try:
        solver.step_batch(3, dt, config["gravity"])
        solver.check_numerical_status()
        got = solver.read_particles(list(probes))
    finally:
        solver.dispose()
    part = OracleState(sample["particles"], config)
    part.run(config, 3)
    for k, g in enumerate(got):
        want = _values(part, sample["probeSampleIndices"][k])
        assert abs(g["position"]["x"] - want[0]) <= 0.02 and abs(g["position"]["y"] - want[1]) <= 0.02
        for gv, wv in ((g["velocity"]["x"], want[2]), (g["velocity"]["y"], want[3])):
            assert abs(gv - wv) <= 0.025 + 5e-4 * abs(wv)
