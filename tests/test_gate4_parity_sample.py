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
from mpm_b200.scenes import (GATE4_FIXED_STEP_SECONDS, GATE4_GRID, GATE4_LIQUID_PARTICLE_AREA, GATE4_PARTICLE_AREA,
                             GATE4_PEBBLE_EDGE_LENGTH, GATE4_SOLID_PARTICLE_MASS, create_mpm_cpu_parity_sample,
                             create_mpm_gate4_scene, create_mpm_gate4_step_config)
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


def test_the_scene_is_the_shared_workload(scene):
    """src/lib/mpm/reference/cpu-simulation.spec.ts:20-34: 50x40 water,
    50x30 oil, 50 three-particle pebbles and a 6x4 fractured solid with its
    horizontal, vertical and diagonal bonds; every liquid particle carries
    the liquid area."""
    particles, bonds, _ = scene
    assert len(particles) == 50 * 40 + 50 * 30 + 50 * 3 + 6 * 4 == 3_674
    assert np.count_nonzero(particles.material == 0) == 2_000  # water
    assert np.count_nonzero(particles.material == 1) == 1_500  # oil
    assert np.count_nonzero(particles.bonded_vertex >= 0) == 150
    assert len(np.unique(particles.object_id[particles.bonded_vertex >= 0])) == 50
    assert len(bonds) == 5 * 4 + 3 * 6 + 5 * 3
    liquid = particles.material <= 1
    assert np.all(particles.volume[liquid] == GATE4_LIQUID_PARTICLE_AREA)


def test_stepping_carries_the_fracture_state(scene):
    """src/lib/mpm/reference/cpu-simulation.spec.ts:93-116: a second step from
    the first step's particles and bonds equals two steps in one run.  The
    scene's bonds stay intact over the first steps, so one enters broken and
    one partly damaged, and both must come out the same way."""
    particles, bonds, _ = scene
    bonds = [dict(bonds[0], broken=True, damage=1.0), dict(bonds[1], damage=0.3)] + list(bonds[2:])
    config = dict(create_mpm_gate4_step_config(fracture_bonds=bonds), dt=GATE4_FIXED_STEP_SECONDS / 8)
    stepped = OracleState(particles, config)
    stepped.step(config)
    stepped.step(config)
    ran = OracleState(particles, config)
    ran.run(config, 2)
    assert np.array_equal(stepped.particles, ran.particles)
    assert np.array_equal(stepped.bonds, ran.bonds)
    assert len(stepped.bonds) == len(bonds)
    assert stepped.bonds["broken"][0] == 1 and stepped.bonds["damage"][1] == 0.3
    ends = [bonds[0]["firstParticle"], bonds[0]["secondParticle"]]
    assert np.all(stepped.particles["damage"][ends] == 1.0)


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
