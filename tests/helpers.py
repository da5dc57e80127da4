"""Shared fixtures: reference-shaped particles/configs and oracle helpers."""
from __future__ import annotations

import numpy as np

from mpm_b200.layout import ParticleArrays, particles_from_dicts
from oracle import OracleState

ZERO = {"m00": 0.0, "m01": 0.0, "m10": 0.0, "m11": 0.0}
IDENTITY = {"m00": 1.0, "m01": 0.0, "m10": 0.0, "m11": 1.0}


def make_config(**overrides) -> dict:
    """makeConfig of src/lib/mpm/reference/solver.spec.ts:14-24."""
    cfg = {"dt": 0.001, "grid": {"cellsX": 16, "cellsY": 16, "cellSize": 1}, "particleMass": 0.1,
           "particleVolume": 0.01, "material": {"lambda": 20, "mu": 10}, "gravity": {"x": 0, "y": 0}}
    cfg.update(overrides)
    return cfg


def make_particle(**overrides) -> dict:
    """makeParticle of src/lib/mpm/reference/solver.spec.ts:26-34."""
    p = {"position": {"x": 8, "y": 8}, "velocity": {"x": 0, "y": 0}, "C": dict(ZERO), "F": dict(IDENTITY)}
    p.update(overrides)
    return p


def oracle_run(particles, config: dict, steps: int = 1):
    arrays = particles if isinstance(particles, ParticleArrays) else particles_from_dicts(particles)
    state = OracleState(arrays, config)
    diag = None
    for _ in range(steps):
        diag = state.step(config)
    return state, diag


def transfer_regression_fixture():
    """runMpmTransferRegression's 45 particles: src/lib/mpm/experiments/transfer-regression.ts:33-58."""
    materials = [
        {"model": "neo-hookean", "lambda": 20, "mu": 10},
        {"model": "snow", "lambda": 20, "mu": 10},
        {"model": "water", "lambda": 8, "mu": 0, "density": 1},
        {"model": "oil", "lambda": 6, "mu": 0, "density": 0.8},
        {"model": "powder", "lambda": 20, "mu": 10, "frictionCoefficient": 0.55},
    ]
    particles = []
    for group, material in enumerate(materials):
        for local in range(9):
            particles.append({
                "position": {"x": 4 + group * 8 + local % 3, "y": 4 + local // 3},
                "velocity": {"x": 0.03 * group, "y": -0.02},
                "C": {"m00": 0, "m01": 0.001, "m10": 0, "m11": 0},
                "F": {"m00": 0.98, "m01": 0.01, "m10": 0, "m11": 0.99},
                "material": material, "objectId": group + 1, "plasticVolume": 1,
            })
    config = {"grid": {"cellsX": 48, "cellsY": 16, "cellSize": 1}, "particleMass": 0.1, "particleVolume": 0.05,
              "material": materials[0], "capacity": 54}
    return particles, config


def packed_columns(packed: np.ndarray) -> dict:
    p = packed.astype(np.float64)
    return {"position": p[:, 0:2], "velocity": p[:, 2:4], "C": p[:, 4:8], "F": p[:, 8:12], "plastic": p[:, 12]}


def oracle_columns(state: OracleState) -> dict:
    return {"position": state.positions(), "velocity": state.velocities(), "C": state.affine(),
            "F": state.deformation(), "plastic": state.particles["plastic_volume"].copy()}


def max_abs_difference(a: dict, b: dict, fields=("position", "velocity", "C", "F", "plastic")) -> float:
    return max(float(np.max(np.abs(np.asarray(a[k]) - np.asarray(b[k])))) if np.size(a[k]) else 0.0 for k in fields)
