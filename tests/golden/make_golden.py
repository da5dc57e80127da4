"""Golden fixtures of the substep path: the FP64 oracle's end states for small
seeded cases, each with a digest of its validated input.

The reference (TypeScript + WebGPU) has no runtime on this image, so these
are the oracle's outputs; the oracle itself is pinned by the reference's own
property tests and known answers (tests/test_oracle_reference_properties.py).
The fixtures freeze it: tests/test_golden.py checks on the CPU that the oracle
still reproduces them bit for bit, and on the GPU compares the CUDA path with
them without running the oracle.

Cases (inputs are rebuilt from the seeded generators below; the digest
catches any drift in them):
* transfer       - the 45-particle, five-model fixture of
                   src/lib/mpm/experiments/transfer-regression.ts:33-58, 8 steps;
* multi_material - 96 particles of all six models (fixed-corotated included), 20 steps;
* si_tank        - the 1,600-particle SI Tait water tank (seed 1), 60 CFL microsteps;
* dam_break      - a 2,400-particle water/oil dam break on a 64x64 grid, 10 steps.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for _p in (os.path.join(ROOT, "powder-play_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

FIXTURE = os.path.join(HERE, "oracle_fp64.npz")
ALL_FIELDS = ("position", "velocity", "C", "F", "plastic")
MOTION_FIELDS = ("position", "velocity")


def _multi_material():
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
    return parts, config


def cases() -> dict:
    """name -> {particles, config, gravity, dt (float32-representable), steps,
    fields, tolerance}; tolerance "abs" bounds every field's absolute error,
    "scene" bounds positions by 1e-3 cell sizes and velocities by
    1e-3 * (1 + |v|)."""
    from helpers import transfer_regression_fixture
    from mpm_b200 import calculate_mpm_cfl_microsteps
    from mpm_b200.scenes import DAM_BREAK_GRAVITY, create_dam_break_scene, create_si_tank_scene

    f32 = lambda v: float(np.float32(v))
    out = {}
    parts, config = transfer_regression_fixture()
    out["transfer"] = dict(particles=parts, config=config, gravity={"x": 0.0, "y": 0.0}, dt=f32(1e-3), steps=8,
                           fields=ALL_FIELDS, tolerance="abs")
    parts, config = _multi_material()
    out["multi_material"] = dict(particles=parts, config=config, gravity={"x": 0.0, "y": -1.0}, dt=f32(1e-3),
                                 steps=20, fields=ALL_FIELDS, tolerance="abs")
    p, config = create_si_tank_scene(seed=1)
    plan = calculate_mpm_cfl_microsteps(1 / 120, config["grid"]["cellSize"], 20.01, 0.0, 512)
    out["si_tank"] = dict(particles=p, config=config, gravity={"x": 0.0, "y": -9.81}, dt=f32(plan["microDt"]),
                          steps=60, fields=MOTION_FIELDS, tolerance="scene")
    p, config = create_dam_break_scene(particles_per_phase=1200, columns=40,
                                       grid={"cellsX": 64, "cellsY": 64, "cellSize": 10})
    out["dam_break"] = dict(particles=p, config=config, gravity=dict(DAM_BREAK_GRAVITY), dt=f32(8e-4), steps=10,
                            fields=MOTION_FIELDS, tolerance="scene")
    return out


def input_digest(case: dict) -> str:
    """sha256 of the validated float32 particle records, their object ids and
    the step settings."""
    from mpm_b200.layout import validate_mpm_mls_gpu_input
    state = validate_mpm_mls_gpu_input(case["particles"], case["config"])
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(state.packed_particles, dtype=np.float32).tobytes())
    h.update(np.ascontiguousarray(state.packed_object_ids, dtype=np.uint32).tobytes())
    h.update(json.dumps([case["config"], case["gravity"], case["dt"], case["steps"]], sort_keys=True,
                        default=str).encode())
    return h.hexdigest()


def run_oracle(case: dict) -> dict:
    """The oracle's end state of the case: {field: float64 array}."""
    from helpers import oracle_columns
    from mpm_b200.layout import particles_from_dicts
    from oracle import OracleState
    particles = case["particles"]
    if isinstance(particles, list):
        particles = particles_from_dicts(particles)
    cfg = dict(case["config"], dt=case["dt"], gravity=case["gravity"])
    state = OracleState(particles, cfg)
    state.run(cfg, case["steps"])
    cols = oracle_columns(state)
    return {k: np.asarray(cols[k], dtype=np.float64) for k in case["fields"]}


def main() -> None:
    arrays = {}
    for name, case in cases().items():
        arrays[f"{name}/input_sha256"] = np.array(input_digest(case))
        for field, values in run_oracle(case).items():
            arrays[f"{name}/{field}"] = values
    np.savez_compressed(FIXTURE, **arrays)
    print(f"wrote {FIXTURE} ({os.path.getsize(FIXTURE)} bytes, {len(arrays)} arrays)")


if __name__ == "__main__":
    main()
