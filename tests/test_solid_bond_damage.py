"""Fracture-bond damage, restating src/lib/mpm/reference/solid-bonds.spec.ts
against the oracle, the host validation and (under -m gpu) the CUDA path.

updateMpmSolidBondDamage (src/lib/mpm/reference/solid-bonds.ts:72-109) runs at
the end of every stepMpm on the advected positions.  The spec calls it on
particles at rest, so these tests take one step of a scene in which nothing
moves: zero gravity, zero velocity, F = I (no stress), particles far from the
walls.  Positions after the step are then the spec's positions exactly, and
the damage the step writes is the spec's.

The spec's three particles sit on y = 20 at x = 10, 20, 30 (unstrained) or
10, 22, 32 (the first bond stretched by 2 over its rest length 10: strain
0.2, the failure strain, so it breaks).
"""
import numpy as np
import pytest

from mpm_b200 import RangeError, create_mpm_mls_gpu_solver
from mpm_b200.layout import particles_from_dicts, validate_mpm_mls_gpu_input
from oracle import OracleError, OracleState

ZERO = {"m00": 0.0, "m01": 0.0, "m10": 0.0, "m11": 0.0}
IDENTITY = {"m00": 1.0, "m01": 0.0, "m10": 0.0, "m11": 1.0}
SOLID = {"lambda": 20.0, "mu": 10.0, "model": "neo-hookean"}
WATER = {"lambda": 10.0, "mu": 0.0, "model": "water", "density": 1.0}


def _particle(x, velocity_x=0.0, **extra):
    p = {"position": {"x": float(x), "y": 20.0}, "velocity": {"x": float(velocity_x), "y": 0.0},
         "C": dict(ZERO), "F": dict(IDENTITY), "objectId": 4, "material": SOLID}
    p.update(extra)
    return p


def _bond(first, second, **extra):
    b = {"firstParticle": first, "secondParticle": second, "restLength": 10.0, "failureStrain": 0.2}
    b.update(extra)
    return b


def _config(bonds):
    return {"grid": {"cellsX": 64, "cellsY": 64, "cellSize": 1.0}, "particleMass": 1.0, "particleVolume": 1.0,
            "material": SOLID, "gravity": {"x": 0.0, "y": 0.0}, "dt": 1e-3, "fractureBonds": bonds}


def _oracle_step(particles, bonds):
    config = _config(bonds)
    state = OracleState(particles_from_dicts(particles), config)
    state.step(config)
    damage = np.where(state.particles["has_damage"] != 0, state.particles["damage"], 0.0)
    return state, damage


def test_unstrained_bonds_leave_no_damage():
    state, damage = _oracle_step([_particle(10), _particle(20), _particle(30)], [_bond(0, 1), _bond(1, 2)])
    assert list(state.bonds["damage"]) == [0.0, 0.0]
    assert list(state.bonds["broken"]) == [0, 0]
    assert list(damage) == [0.0, 0.0, 0.0]
    assert list(state.particles["px"]) == [10.0, 20.0, 30.0]


def test_tensile_damage_reaches_the_threshold_and_stays_on_incident_particles():
    state, damage = _oracle_step([_particle(10), _particle(22), _particle(32)], [_bond(0, 1), _bond(1, 2)])
    assert (state.bonds["damage"][0], state.bonds["broken"][0]) == (1.0, 1)
    assert (state.bonds["damage"][1], state.bonds["broken"][1]) == (0.0, 0)
    assert list(damage) == [1.0, 1.0, 0.0]


def test_partial_strain_accumulates_proportional_damage():
    # strain 0.1 of 0.2: damage 0.5, not broken; a later, smaller strain keeps the maximum
    state, damage = _oracle_step([_particle(10), _particle(21), _particle(31)], [_bond(0, 1), _bond(1, 2)])
    assert state.bonds["damage"][0] == pytest.approx(0.5, abs=1e-12) and state.bonds["broken"][0] == 0
    assert list(damage[:2]) == pytest.approx([0.5, 0.5], abs=1e-12) and damage[2] == 0.0
    config = _config([dict(_bond(0, 1), damage=0.5), _bond(1, 2)])
    relaxed = OracleState(particles_from_dicts([_particle(10), _particle(20.5), _particle(30.5)]), config)
    relaxed.step(config)
    assert relaxed.bonds["damage"][0] == pytest.approx(0.5, abs=1e-12)


def test_broken_bonds_stay_broken_after_unloading_and_momentum_is_kept():
    initial = [_particle(10, 2.0), _particle(20, -2.0), _particle(30, 0.0)]
    initial_momentum = sum(p["velocity"]["x"] for p in initial)
    state, damage = _oracle_step([_particle(10), _particle(10.1), _particle(30)],
                                 [_bond(0, 1, broken=True, damage=1.0), _bond(1, 2)])
    assert (state.bonds["broken"][0], state.bonds["damage"][0]) == (1, 1.0)
    assert damage[0] == 1.0
    # the second bond spans 19.9 over its rest length 10: it breaks as well
    assert state.bonds["broken"][1] == 1 and list(damage) == [1.0, 1.0, 1.0]
    assert len(state.particles) == len(initial)
    assert float(np.sum(state.particles["vx"])) == initial_momentum


REJECTIONS = [
    ([_particle(10)], [_bond(0, 1)], "existing particle"),
    ([_particle(10), _particle(20)], [_bond(0, 1), _bond(1, 0)], "duplicates"),
    ([_particle(10), _particle(20, objectId=5)], [_bond(0, 1)], "one object"),
    ([_particle(10), _particle(20, material=WATER)], [_bond(0, 1)], "neo-hookean solids"),
]


@pytest.mark.parametrize("particles,bonds,message", REJECTIONS, ids=[r[2] for r in REJECTIONS])
def test_the_oracle_rejects_invalid_bond_graphs(particles, bonds, message):
    config = _config(bonds)
    with pytest.raises(OracleError, match=message):
        OracleState(particles_from_dicts(particles), config).step(config)


@pytest.mark.parametrize("particles,bonds,message", REJECTIONS, ids=[r[2] for r in REJECTIONS])
def test_the_host_rejects_invalid_bond_graphs_before_any_device_work(particles, bonds, message):
    with pytest.raises(RangeError, match=message):
        validate_mpm_mls_gpu_input(particles, _config(bonds))


@pytest.mark.gpu
@pytest.mark.parametrize("xs,expected", [((10, 20, 30), [0.0, 0.0, 0.0]), ((10, 22, 32), [1.0, 1.0, 0.0]),
                                         ((10, 21, 31), [0.5, 0.5, 0.0])])
def test_the_cuda_path_writes_the_same_particle_damage(xs, expected):
    particles = [_particle(x) for x in xs]
    bonds = [_bond(0, 1), _bond(1, 2)]
    solver = create_mpm_mls_gpu_solver(particles, _config(bonds))
    try:
        solver.step(1e-3, {"x": 0.0, "y": 0.0})
        solver.check_numerical_status()
        packed, _ = solver.read_particles_packed()
    finally:
        solver.dispose()
    _, oracle_damage = _oracle_step(particles, bonds)
    assert list(packed[:, 0]) == [float(x) for x in xs]
    assert np.allclose(packed[:, 18], expected, atol=1e-6)
    assert np.allclose(packed[:, 18], oracle_damage, atol=1e-6)


@pytest.mark.gpu
def test_the_cuda_path_keeps_broken_bonds_broken():
    particles = [_particle(10), _particle(10.1), _particle(30)]
    bonds = [_bond(0, 1, broken=True, damage=1.0), _bond(1, 2)]
    solver = create_mpm_mls_gpu_solver(particles, _config(bonds))
    try:
        for _ in range(3):
            solver.step(1e-3, {"x": 0.0, "y": 0.0})
        solver.check_numerical_status()
        packed, _ = solver.read_particles_packed()
    finally:
        solver.dispose()
    assert list(packed[:, 18]) == [1.0, 1.0, 1.0]
    assert float(np.sum(packed[:, 2])) == 0.0
