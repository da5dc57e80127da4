"""The reference CPU solver's property cases (src/lib/mpm/reference/solver.spec.ts)
run through the CUDA path (gather and fixed-point P2G, via the C ABI), each
against the FP64 oracle on the same input: an empty particle set, a lone
particle on a sparse 2000x2000 grid, each domain wall, wall friction, a
velocity gradient that needs deformation substeps, and ragged particle
counts (1 to 257, not multiples of a warp or a tile).

Tolerances: wall and rest positions exact (the confinement clamps to the
wall); otherwise 1e-4 absolute for the single-particle cases and, for the
ragged sets, positions within 1e-3 cell sizes and velocities within
1e-3 * (1 + |v|).
"""
import numpy as np
import pytest

from helpers import make_config, make_particle, oracle_columns, oracle_run, packed_columns
from mpm_b200 import create_experimental_mpm_mls_atomic_gpu_solver, create_mpm_mls_gpu_solver
from mpm_b200.layout import ParticleArrays

pytestmark = pytest.mark.gpu

FACTORIES = {"gather": create_mpm_mls_gpu_solver, "atomic": create_experimental_mpm_mls_atomic_gpu_solver}


def _gpu(particles, config, variant, steps=1):
    solver = FACTORIES[variant](particles, config)
    try:
        solver.step_batch(steps, config["dt"], config["gravity"])
        packed, _ = solver.read_particles_packed()
    finally:
        solver.dispose()
    return packed_columns(packed)


@pytest.mark.parametrize("variant", sorted(FACTORIES))
def test_empty_particle_set_steps(variant):
    # solver.spec.ts:63-75
    out = _gpu([], make_config(), variant, steps=3)
    assert out["position"].shape == (0, 2)


@pytest.mark.parametrize("variant", sorted(FACTORIES))
def test_lone_particle_rests_on_a_sparse_2000_grid(variant):
    # solver.spec.ts:77-88
    config = make_config(grid={"cellsX": 2000, "cellsY": 2000, "cellSize": 1})
    out = _gpu([make_particle(position={"x": 8, "y": 8})], config, variant)
    assert tuple(out["position"][0]) == (8.0, 8.0)
    assert tuple(out["velocity"][0]) == (0.0, 0.0)


@pytest.mark.parametrize("variant", sorted(FACTORIES))
def test_each_domain_wall_stops_the_particle_on_it(variant):
    # solver.spec.ts:213-252
    cases = [((0, 4), (-10, 0), (0, 4)), ((8, 4), (10, 0), (8, 4)), ((4, 0), (0, -10), (4, 0)),
             ((4, 8), (0, 10), (4, 8))]
    config = make_config(dt=0.1, grid={"cellsX": 8, "cellsY": 8, "cellSize": 1})
    for (px, py), (vx, vy), expected in cases:
        particle = make_particle(position={"x": px, "y": py}, velocity={"x": vx, "y": vy})
        out = _gpu([particle], config, variant)
        ref, _ = oracle_run([particle], dict(config, dt=float(np.float32(config["dt"]))))
        assert tuple(out["position"][0]) == expected == tuple(ref.positions()[0])
        assert tuple(out["velocity"][0]) == (0.0, 0.0)


@pytest.mark.parametrize("variant", sorted(FACTORIES))
def test_wall_friction_damps_the_tangential_velocity(variant):
    # solver.spec.ts:254-268
    particle = make_particle(position={"x": 0, "y": 4}, velocity={"x": 0, "y": 10})
    config = make_config(dt=0.1, grid={"cellsX": 8, "cellsY": 8, "cellSize": 1})
    free = _gpu([particle], config, variant)
    stuck = _gpu([particle], dict(config, wallFriction=1), variant)
    assert free["velocity"][0, 1] > 0
    assert stuck["velocity"][0, 1] < free["velocity"][0, 1]
    for cfg, out in ((config, free), (dict(config, wallFriction=1), stuck)):
        ref, _ = oracle_run([particle], dict(cfg, dt=float(np.float32(cfg["dt"]))))
        assert np.max(np.abs(out["velocity"] - ref.velocities())) <= 1e-4
        assert np.max(np.abs(out["position"] - ref.positions())) <= 1e-4


@pytest.mark.parametrize("variant", sorted(FACTORIES))
def test_a_large_velocity_gradient_keeps_det_f_positive(variant):
    # solver.spec.ts:199-211: the F update is split into substeps
    particle = make_particle(C={"m00": 0, "m01": 0, "m10": 0, "m11": -100})
    config = make_config(dt=0.1)
    out = _gpu([particle], config, variant)
    F = out["F"][0]
    assert F[0] * F[3] - F[1] * F[2] > 0
    ref, _ = oracle_run([particle], dict(config, dt=float(np.float32(config["dt"]))))
    assert np.max(np.abs(out["F"] - ref.deformation())) <= 1e-4
    assert np.max(np.abs(out["C"] - ref.affine())) <= 1e-4 * 100


@pytest.mark.parametrize("variant", sorted(FACTORIES))
@pytest.mark.parametrize("count", [1, 31, 33, 129, 257])
def test_ragged_particle_counts_match_the_oracle(count, variant):
    rng = np.random.default_rng(count)
    p = ParticleArrays.empty(count)
    p.px[:] = rng.uniform(3, 29, count).astype(np.float32)
    p.py[:] = rng.uniform(3, 29, count).astype(np.float32)
    p.vx[:] = rng.uniform(-1, 1, count).astype(np.float32)
    p.vy[:] = rng.uniform(-1, 1, count).astype(np.float32)
    water = {"lambda": 8, "mu": 0, "model": "water", "density": 1}
    solid = {"lambda": 20, "mu": 10}
    p.materials = [water, solid]
    p.material[:] = rng.integers(0, 2, count)
    p.volume[:] = 0.05
    config = {"grid": {"cellsX": 32, "cellsY": 32, "cellSize": 1}, "particleMass": 0.1, "particleVolume": 0.05,
              "material": solid, "dt": float(np.float32(1e-3)), "gravity": {"x": 0.0, "y": -1.0}}
    out = _gpu(p, config, variant, steps=6)
    ref, _ = oracle_run(p, config, steps=6)
    ref = oracle_columns(ref)
    assert np.max(np.abs(out["position"] - ref["position"])) <= 1e-3
    assert np.max(np.abs(out["velocity"] - ref["velocity"]) / (1 + np.abs(ref["velocity"]))) <= 1e-3
