"""Long-horizon fixture of the 1,000,000-particle two-phase dam break: the
FP64 oracle over 200 macrosteps of 1/240 s (the benchmark configuration's
horizon), each taken as 5 microsteps of 1/1200 s (the CFL plan gives 4-5 at
these speeds; a fixed schedule lets the GPU test replay it exactly; the
oracle steps the float32 microDt).

Recorded: every 40 macrosteps, the bulk diagnostics of each liquid
(mpm_b200.diagnostics.summarize_dam_break_phase); at the end, position and
velocity of every 1,000th particle (1,000 particles, original indices 0,
1000, ...).

Run from the repository root (about six minutes, one thread):
    python tests/golden/make_dam_break_long.py
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

from mpm_b200.diagnostics import summarize_dam_break_phase  # noqa: E402
from mpm_b200.scenes import DAM_BREAK_GRAVITY, create_dam_break_scene  # noqa: E402

FIXTURE = os.path.join(HERE, "dam_break_long_fp64.json")
MACROSTEPS = 200
MICROSTEPS = 5
MICRO_DT = 1 / 1200
EVERY = 40
SAMPLE_STRIDE = 1000


def packed_from_oracle(state) -> np.ndarray:
    out = np.zeros((len(state.particles), 20), dtype=np.float64)
    out[:, 0:2] = state.positions()
    out[:, 2:4] = state.velocities()
    out[:, 4:8] = state.affine()
    out[:, 8:12] = state.deformation()
    return out


def phases(packed: np.ndarray, half: int) -> dict:
    return {"water": summarize_dam_break_phase(packed[:half]), "oil": summarize_dam_break_phase(packed[half:])}


def main():
    from oracle import OracleState

    particles, config = create_dam_break_scene()
    half = len(particles) // 2
    dt32 = float(np.float32(MICRO_DT))
    cfg = dict(config, dt=dt32, gravity=DAM_BREAK_GRAVITY)
    state = OracleState(particles, cfg)
    records = [phases(packed_from_oracle(state), half)]
    started = time.time()
    for macro in range(1, MACROSTEPS + 1):
        state.run(cfg, MICROSTEPS)
        if macro % EVERY == 0:
            records.append(phases(packed_from_oracle(state), half))
            print(f"macrostep {macro}: {time.time() - started:.0f} s", flush=True)
    final = packed_from_oracle(state)[::SAMPLE_STRIDE, 0:4]
    data = {"microDt": MICRO_DT, "microstepsPerMacrostep": MICROSTEPS, "macrosteps": MACROSTEPS, "every": EVERY,
            "sampleStride": SAMPLE_STRIDE, "diagnostics": records, "sample": final.tolist()}
    with open(FIXTURE, "w") as f:
        json.dump(data, f)
    print(f"wrote {FIXTURE}: {MACROSTEPS} x {MICROSTEPS} microsteps of {dt32:.4e} s in {time.time() - started:.0f} s")


if __name__ == "__main__":
    main()
