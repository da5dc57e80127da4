"""The reference CPU solver's own property tests, re-run against the C oracle.

Each test restates one case of src/lib/mpm/reference/solver.spec.ts
(7korobi/powder-play) with the reference's inputs, assertions and
tolerances; together they pin the FP64 restatement (the reference ships no
stored trajectories).
"""
import numpy as np
import pytest

from helpers import make_config, make_particle, oracle_run
from oracle import OracleError


def det(F):
    return F[..., 0] * F[..., 3] - F[..., 1] * F[..., 2]


def test_empty_particle_set_has_zero_diagnostics():
    # solver.spec.ts:63-75
    state, diag = oracle_run([], make_config())
    assert len(state.particles) == 0
    assert diag == {k: 0.0 for k in diag}


def test_sparse_sized_grid_keeps_a_resting_particle_and_its_mass():
    # solver.spec.ts:77-88 (2000x2000 grid)
    particle = make_particle(position={"x": 8, "y": 8})
    state, d = oracle_run([particle], make_config(grid={"cellsX": 2000, "cellsY": 2000, "cellSize": 1}))
    assert tuple(state.positions()[0]) == (8.0, 8.0)
    assert abs(d["grid_mass"] - 0.1) < 1e-9


def test_substeps_a_large_velocity_gradient():
    # solver.spec.ts:199-211
    state, _ = oracle_run([make_particle(C={"m00": 0, "m01": 0, "m10": 0, "m11": -100})], make_config(dt=0.1))
    assert det(state.deformation()[0]) > 0


def test_collides_with_each_domain_wall_without_leaving_the_domain():
    # solver.spec.ts:213-252
    cases = [((0, 4), (-10, 0), (0, 4)), ((8, 4), (10, 0), (8, 4)), ((4, 0), (0, -10), (4, 0)),
             ((4, 8), (0, 10), (4, 8))]
    config = make_config(dt=0.1, grid={"cellsX": 8, "cellsY": 8, "cellSize": 1})
    for (px, py), (vx, vy), expected in cases:
        state, _ = oracle_run([make_particle(position={"x": px, "y": py}, velocity={"x": vx, "y": vy})], config)
        assert tuple(state.positions()[0]) == expected
        assert tuple(state.velocities()[0]) == (0.0, 0.0)


def test_wall_friction_damps_tangential_velocity_only_when_configured():
    # solver.spec.ts:254-268
    particle = make_particle(position={"x": 0, "y": 4}, velocity={"x": 0, "y": 10})
    config = make_config(dt=0.1, grid={"cellsX": 8, "cellsY": 8, "cellSize": 1})
    free, _ = oracle_run([particle], config)
    stuck, _ = oracle_run([particle], dict(config, wallFriction=1))
    assert free.velocities()[0, 1] > 0
    assert stuck.velocities()[0, 1] < free.velocities()[0, 1]


def test_tait_pressure_holds_volume_better_than_the_linear_profile():
    # solver.spec.ts:270-302
    tait = {"lambda": 1000, "mu": 0, "model": "water", "density": 20,
            "equationOfState": {"model": "tait", "exponent": 7.15}}
    linear = {"lambda": 1000, "mu": 0, "model": "water", "density": 20}
    particle = make_particle(position={"x": 4, "y": 4}, F={"m00": 0.975, "m01": 0, "m10": 0, "m11": 0.975},
                             volume=0.04)
    config = make_config(dt=0.00001, grid={"cellsX": 8, "cellsY": 8, "cellSize": 1}, particleMass=0.8,
                         particleVolume=0.04, material=tait)
    t, _ = oracle_run([particle], config)
    lin, _ = oracle_run([particle], dict(config, material=linear))
    assert det(t.deformation()[0]) > det(lin.deformation()[0])


@pytest.mark.parametrize("material", [
    {"lambda": 8, "mu": 0, "model": "water", "density": 0.04},
    {"lambda": 6, "mu": 0, "model": "oil", "density": 0.032},
    {"lambda": 20, "mu": 10, "model": "powder", "frictionCoefficient": 0.55},
])
def test_all_materials_stay_inside_the_domain_under_wall_impacts(material):
    # solver.spec.ts:304-352 (480 steps of sustained acceleration into each wall)
    collisions = [(8.2, 15.2, {"x": -90, "y": 0}), (23.2, 15.2, {"x": 90, "y": 0}),
                  (15.2, 8.2, {"x": 0, "y": -90}), (15.2, 23.2, {"x": 0, "y": 90})]
    for sx, sy, gravity in collisions:
        particles = [make_particle(position={"x": sx + (i % 3) * 0.4, "y": sy + (i // 3) * 0.4}, material=material)
                     for i in range(9)]
        config = make_config(dt=1 / 240, grid={"cellsX": 32, "cellsY": 32, "cellSize": 1}, particleVolume=0.16,
                             material=material, gravity=gravity)
        state, _ = oracle_run(particles, config, steps=480)
        assert np.all(det(state.deformation()) > 0)
        pos = state.positions()
        assert np.all(pos >= 0) and np.all(pos <= 32)


def test_conserves_mass_and_momentum_away_from_gravity_and_boundaries():
    # solver.spec.ts:354-390: mass 1e-12, momentum 1e-10
    particles = [
        make_particle(position={"x": 24.2, "y": 21.7}, velocity={"x": 0.5, "y": -0.2}),
        make_particle(position={"x": 25.1, "y": 21.9}, velocity={"x": -0.1, "y": 0.4}),
        make_particle(position={"x": 24.6, "y": 22.8}, velocity={"x": 0.2, "y": 0.1}),
    ]
    config = make_config(dt=0.001, grid={"cellsX": 64, "cellsY": 64, "cellSize": 1}, particleMass=0.1)
    mx = sum(0.1 * p["velocity"]["x"] for p in particles)
    my = sum(0.1 * p["velocity"]["y"] for p in particles)
    _, d = oracle_run(particles, config)
    assert abs(d["grid_mass"] - d["input_mass"]) <= 1e-12
    assert abs(d["output_mass"] - d["input_mass"]) <= 1e-12
    assert abs(d["grid_mx"] - mx) <= 1e-10 and abs(d["grid_my"] - my) <= 1e-10
    assert abs(d["output_mx"] - mx) <= 1e-10 and abs(d["output_my"] - my) <= 1e-10


def test_fracture_is_localised_and_conserves_mass_and_momentum():
    # solver.spec.ts:392-445
    particles = [make_particle(position={"x": 10, "y": 20}, velocity={"x": 1, "y": 0}, objectId=4),
                 make_particle(position={"x": 25, "y": 20}, velocity={"x": -1, "y": 0}, objectId=4),
                 make_particle(position={"x": 35, "y": 20}, objectId=4)]
    bonds = [{"firstParticle": 0, "secondParticle": 1, "restLength": 10, "failureStrain": 0.1}]
    config = make_config(dt=0.001, grid={"cellsX": 64, "cellsY": 64, "cellSize": 1}, particleMass=1,
                         fractureBonds=bonds)
    state, d = oracle_run(particles, config)
    assert state.bonds[0]["broken"] == 1 and state.bonds[0]["damage"] == 1.0
    damage = np.where(state.particles["has_damage"] == 1, state.particles["damage"], 0.0)
    assert list(damage) == [1.0, 1.0, 0.0]
    assert d["input_mass"] == 3 and abs(d["grid_mass"] - 3) < 1e-12 and d["output_mass"] == 3
    assert abs(d["output_mx"]) < 1e-12
    before = state.positions().copy()
    state.step(config)
    after = state.positions()
    assert after[0, 0] > before[0, 0] and after[1, 0] < before[1, 0]
    assert state.particles["has_damage"][2] == 0


def test_denser_liquid_moves_down_relative_to_the_lighter_one():
    # solver.spec.ts:585-605
    particles = [make_particle(position={"x": 8, "y": 8}, volume=1,
                               material={"lambda": 8, "mu": 0, "model": "water", "density": 2}),
                 make_particle(position={"x": 8, "y": 8}, volume=1,
                               material={"lambda": 8, "mu": 0, "model": "oil", "density": 1})]
    state, _ = oracle_run(particles, make_config(dt=0.01, gravity={"x": 0, "y": 10}))
    v, p = state.velocities(), state.positions()
    assert v[0, 1] > v[1, 1] and p[0, 1] > p[1, 1]


def test_denser_water_sinks_through_inverted_oil():
    # solver.spec.ts:607-627 (500 steps)
    particles = [make_particle(position={"x": 8, "y": 7.5}, volume=1,
                               material={"lambda": 8, "mu": 0, "model": "water", "density": 2}),
                 make_particle(position={"x": 8, "y": 8.5}, volume=1,
                               material={"lambda": 8, "mu": 0, "model": "oil", "density": 1})]
    state, _ = oracle_run(particles, make_config(dt=0.001, gravity={"x": 0, "y": 10}), steps=500)
    p = state.positions()
    assert p[0, 1] > p[1, 1]


def test_stretched_bonded_triangle_is_restored_toward_rest_length():
    # solver.spec.ts:845-878
    particles = [make_particle(position={"x": 8, "y": 8}, objectId=4, bondedTriangleVertex=0),
                 make_particle(position={"x": 10, "y": 8}, objectId=4, bondedTriangleVertex=1),
                 make_particle(position={"x": 9, "y": 9.5}, objectId=4, bondedTriangleVertex=2)]

    def edge_error(pos):
        return sum(abs(np.hypot(*(pos[(k + 1) % 3] - pos[k])) - 1) for k in range(3))

    initial = edge_error(np.array([[8, 8], [10, 8], [9, 9.5]], dtype=float))
    state, _ = oracle_run(particles, make_config(dt=0.001, bondRestLength=1, bondStiffness=1))
    assert edge_error(state.positions()) < initial
    assert list(state.particles["bonded_vertex"]) == [0, 1, 2]


def test_invalid_inputs_raise_the_reference_errors():
    # solver.spec.ts:130-162 (a subset of the rejected inputs)
    with pytest.raises(OracleError, match="dt must be greater than zero"):
        oracle_run([make_particle()], make_config(dt=-1))
    with pytest.raises(OracleError, match=r"particles\[0\]\.position must be inside the grid domain"):
        oracle_run([make_particle(position={"x": 17, "y": 1})], make_config())
    with pytest.raises(OracleError, match=r"particles\[0\]\.F must have a finite positive determinant"):
        oracle_run([make_particle(F={"m00": 1, "m01": 0, "m10": 0, "m11": -1})], make_config())
