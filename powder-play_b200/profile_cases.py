"""Small fixed cases of the batched and differentiable forms for kernel
profiling (ncu launch lists), each a few hundred launches:

    python powder-play_b200/profile_cases.py batched   # 512 tanks, 2 x 4 substeps
    python powder-play_b200/profile_cases.py dense     # the 64 tanks with most particles per cell
    python powder-play_b200/profile_cases.py adjoint   # 64 scenes, 2 x (40 forward + 40 backward)

Prints the device milliseconds of the last pass.
"""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import numpy as np  # noqa: E402


def batched(dense_only=False):
    from mpm_b200 import calculate_mpm_cfl_microsteps, create_mpm_batched_gpu_solver
    from mpm_b200.scenes import BATCHED_TANK_GRAVITY, create_batched_tank_scenes
    scenes = create_batched_tank_scenes()
    if dense_only:
        per_cell = np.array([len(p.px) / c["grid"]["cellsX"] ** 2 for p, c in scenes])
        scenes = [scenes[i] for i in np.argsort(per_cell)[-64:]]
    b = create_mpm_batched_gpu_solver(scenes)
    try:
        dt = min(calculate_mpm_cfl_microsteps(1 / 240, c["grid"]["cellSize"], bounds["waveSpeedBound"], 1.0,
                                              4096)["microDt"] for (_, c), bounds in zip(scenes, b.cfl_bounds))
        for _ in range(2):
            b.step_batch([4] * len(scenes), [dt] * len(scenes), BATCHED_TANK_GRAVITY)
        print(f"batched: 4 substeps of {len(scenes)} scenes", b.last_batch_device_ms(), "ms")
    finally:
        b.dispose()


def adjoint():
    from mpm_b200.adjoint import create_mpm_adjoint_engine, fixed_cfl_dt
    from mpm_b200.scenes import ADJOINT_GRAVITY, create_adjoint_scenes
    scenes = create_adjoint_scenes()
    dts = [float(np.float32(fixed_cfl_dt(p, c, 90.0, 0.2))) for p, c, _ in scenes]
    targets = np.concatenate([t for _, _, t in scenes]).astype(np.float32)
    e = create_mpm_adjoint_engine([(p, c) for p, c, _ in scenes], ADJOINT_GRAVITY)
    try:
        for _ in range(2):
            e.forward(40, dts, targets, 20)
            e.backward()
        print("adjoint: 40 substeps of 64 scenes, forward / backward", e.last_ms(), "ms")
    finally:
        e.dispose()


if __name__ == "__main__":
    {"batched": batched, "dense": lambda: batched(True), "adjoint": adjoint}[sys.argv[1]]()
