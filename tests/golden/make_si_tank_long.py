"""Long-horizon fixture of the SI water tank: the FP64 oracle's water
diagnostics over 600 macrosteps of 1/120 s (5 s of simulated time).

Scene: the 1,600-particle SI tank on an 80x80 grid (create_si_tank_scene,
seed 1; dx 2.5 mm, Tait gamma 7, c 20 m/s, no-slip walls), gravity
(0, -9.81).  Schedule: every macrostep takes the same CFL plan, the one the
reference's scheduler gives for the tank's wave-speed bound and a velocity
envelope of 2 m/s (calculate_mpm_cfl_microsteps with at most 512 microsteps),
so the GPU test can replay it exactly; the oracle steps the float32 microDt.
Every 60 macrosteps the diagnostics of summarizeSiWater
(src/lib/mpm/experiments/si-performance.ts:19-56) are recorded.

Run from the repository root (about a minute and a half):
    python tests/golden/make_si_tank_long.py
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for _p in (os.path.join(ROOT, "powder-play_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

from mpm_b200.cfl import calculate_mpm_cfl_microsteps  # noqa: E402
from mpm_b200.cfl_bounds import derive_mpm_mls_gpu_cfl_bounds  # noqa: E402
from mpm_b200.diagnostics import summarize_si_water  # noqa: E402
from mpm_b200.layout import validate_mpm_mls_gpu_input  # noqa: E402
from mpm_b200.scenes import SI_TANK_GRAVITY, create_si_tank_scene  # noqa: E402

FIXTURE = os.path.join(HERE, "si_tank_long_fp64.json")
MACRO_DT = 1 / 120
MACROSTEPS = 600
EVERY = 60
VELOCITY_ENVELOPE = 2.0
MAX_MICROSTEPS = 512


def schedule():
    """(particles, config, microDt, microsteps per macrostep, reference area)."""
    particles, config = create_si_tank_scene(seed=1)
    state = validate_mpm_mls_gpu_input(particles, config)
    bounds = derive_mpm_mls_gpu_cfl_bounds(particles, state.config)
    plan = calculate_mpm_cfl_microsteps(MACRO_DT, config["grid"]["cellSize"], bounds["waveSpeedBound"],
                                        VELOCITY_ENVELOPE, MAX_MICROSTEPS)
    reference_area = float(np.sum(state.packed_particles[:, 17].astype(np.float64)))
    return particles, config, plan["microDt"], plan["stepCount"], reference_area


def packed_from_oracle(state) -> np.ndarray:
    out = np.zeros((len(state.particles), 20), dtype=np.float64)
    out[:, 0:2] = state.positions()
    out[:, 2:4] = state.velocities()
    out[:, 4:8] = state.affine()
    out[:, 8:12] = state.deformation()
    out[:, 17] = state.particles["volume"]
    return out


def main():
    from oracle import OracleState

    particles, config, micro_dt, steps, reference_area = schedule()
    dt32 = float(np.float32(micro_dt))
    cfg = dict(config, dt=dt32, gravity=SI_TANK_GRAVITY)
    state = OracleState(particles, cfg)
    records = [summarize_si_water(packed_from_oracle(state), reference_area)]
    started = time.time()
    for macro in range(1, MACROSTEPS + 1):
        state.run(cfg, steps)
        if macro % EVERY == 0:
            records.append(summarize_si_water(packed_from_oracle(state), reference_area))
    data = {"microDt": micro_dt, "microstepsPerMacrostep": steps, "macrosteps": MACROSTEPS, "every": EVERY,
            "referenceArea": reference_area, "diagnostics": records}
    with open(FIXTURE, "w") as f:
        json.dump(data, f, indent=1)
    print(f"wrote {FIXTURE}: {MACROSTEPS} x {steps} microsteps of {dt32:.4e} s in {time.time() - started:.0f} s")


if __name__ == "__main__":
    main()
