"""The differentiable form on the GPU (mpma_* of the C ABI).

* its forward against the default solver stepping the same scenes with the
  same dt: positions within 1e-3 cell sizes after 20 substeps (the sums are
  scattered in another order and the polar rotation has a closed form);
* its adjoint against the FP64 CPU adjoint (oracle/adjoint_fp64.c, itself
  checked against finite differences on the CPU) on a 1,024-particle scene:
  loss within 1e-4, parameter gradients within 2e-2, velocity gradient with
  cosine similarity above 0.999 and relative L2 error below 2e-2;
* its adjoint against central finite differences with a relative step of
  1e-3 of the same algorithm's FP64 forward: within 5e-2;
* the checkpoint interval changes the gradients by rounding only.
"""
import numpy as np
import pytest

from mpm_b200 import create_mpm_batched_gpu_solver
from mpm_b200.adjoint import create_mpm_adjoint_engine, fixed_cfl_dt
from mpm_b200.layout import validate_mpm_mls_gpu_input
from mpm_b200.scenes import ADJOINT_GRAVITY, create_adjoint_scenes
from oracle import adjoint_fp64

pytestmark = pytest.mark.gpu


def _scenes(count=1, seed=9, steps=40):
    # 24 x 32 water + 16 x 16 solid = 1,024 particles on a 64 x 64 grid
    scenes = create_adjoint_scenes(count, seed=seed, water_columns=24, water_rows=32, solid_side=16, cells=64)
    dts = [float(np.float32(fixed_cfl_dt(p, c, 90.0, steps * 1e-3))) for p, c, _ in scenes]
    return scenes, dts


def _fp64(particles, config, targets, dt, steps):
    state = validate_mpm_mls_gpu_input(particles, config)
    pk = state.packed_particles
    liquid = pk[:, 13].view(np.uint32) == 2
    pk64 = pk.astype(np.float64)
    water, solid = pk64[liquid][0], pk64[~liquid][0]
    scene = {"cells_x": config["grid"]["cellsX"], "cells_y": config["grid"]["cellsY"],
             "dx": config["grid"]["cellSize"], "dt": dt, "gx": ADJOINT_GRAVITY["x"], "gy": ADJOINT_GRAVITY["y"],
             "solid_mass": float(np.float32(config["particleMass"])), "wall_friction": config["wallFriction"],
             "rho": float(water[16]), "gamma": float(water[18]), "tait": float(water[14]),
             "lambda_s": float(solid[14]), "mu_s": float(solid[15])}
    return adjoint_fp64(scene, pk64[:, 0:2], pk64[:, 2:4], pk64[:, 4:8], pk64[:, 8:12], pk64[:, 17],
                        liquid.astype(np.int32), np.asarray(targets, np.float32).astype(np.float64), steps)


def _engine(scenes):
    return create_mpm_adjoint_engine([(p, c) for p, c, _ in scenes], ADJOINT_GRAVITY)


def _targets(scenes):
    return np.concatenate([t for _, _, t in scenes])


def test_forward_matches_the_default_solver():
    scenes, dts = _scenes(2, steps=20)
    engine = _engine(scenes)
    batch = create_mpm_batched_gpu_solver([(p, c) for p, c, _ in scenes])
    try:
        engine.forward(20, dts, _targets(scenes), checkpoint_every=20)
        got = engine.read_positions()
        batch.step_batch([20, 20], dts, ADJOINT_GRAVITY)
        assert all(e is None for e in batch.check_numerical_status())
        base = 0
        for k, (p, c, _) in enumerate(scenes):
            want = batch.read_particles_packed(k)[0][:, 0:2]
            n = len(p.px)
            err = np.max(np.abs(got[base:base + n] - want)) / c["grid"]["cellSize"]
            assert err < 1e-3, (k, err)
            base += n
    finally:
        engine.dispose()
        batch.dispose()


@pytest.mark.parametrize("steps, every", [(1, 1), (40, 10)])
def test_adjoint_matches_the_fp64_adjoint(steps, every):
    scenes, dts = _scenes(1, steps=steps)
    (p, c, t), = scenes
    engine = _engine(scenes)
    try:
        loss = engine.forward(steps, dts, t, checkpoint_every=every)
        gv, gp = engine.backward()
    finally:
        engine.dispose()
    ref_loss, ref_gv, ref_gp, _ = _fp64(p, c, t, dts[0], steps)
    assert abs(loss[0] - ref_loss) <= 1e-4 * ref_loss
    for k in range(3):
        assert abs(gp[0, k] - ref_gp[k]) <= 2e-2 * abs(ref_gp[k]) + 1e-6 * np.abs(ref_gp).max(), (k, gp[0], ref_gp)
    a, b = gv.astype(np.float64).ravel(), ref_gv.ravel()
    cosine = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
    assert cosine > 0.999, cosine
    assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b)


def test_adjoint_matches_central_differences():
    # central differences with a relative step of 1e-3 are taken on the FP64
    # forward of the same algorithm: the float32 loss (about 4e5 here) does
    # not resolve the change a 1e-3 step makes (about 1e-7 of it)
    steps = 40
    scenes, dts = _scenes(1, steps=steps)
    (p, c, t), = scenes
    engine = _engine(scenes)
    try:
        engine.forward(steps, dts, t, checkpoint_every=10)
        gv, gp = engine.backward()
    finally:
        engine.dispose()
    state = validate_mpm_mls_gpu_input(p, c)
    pk = state.packed_particles
    liquid = pk[:, 13].view(np.uint32) == 2
    pk64 = pk.astype(np.float64)
    water, solid = pk64[liquid][0], pk64[~liquid][0]
    scene = {"cells_x": 64, "cells_y": 64, "dx": 10.0, "dt": dts[0], "gx": ADJOINT_GRAVITY["x"],
             "gy": ADJOINT_GRAVITY["y"], "solid_mass": float(np.float32(c["particleMass"])), "wall_friction": 0.0,
             "rho": float(water[16]), "gamma": float(water[18]), "tait": float(water[14]),
             "lambda_s": float(solid[14]), "mu_s": float(solid[15])}
    target = np.asarray(t, np.float32).astype(np.float64)

    def loss(sc, v0):
        return adjoint_fp64(sc, pk64[:, 0:2], v0, pk64[:, 4:8], pk64[:, 8:12], pk64[:, 17], liquid.astype(np.int32),
                            target, steps)[0]

    v0 = pk64[:, 2:4]
    for k, name in enumerate(("tait", "lambda_s", "mu_s")):
        eps = 1e-3 * scene[name]
        up, dn = dict(scene), dict(scene)
        up[name] += eps
        dn[name] -= eps
        fd = (loss(up, v0) - loss(dn, v0)) / (2 * eps)
        assert abs(fd - gp[0, k]) <= 5e-2 * abs(fd), (name, fd, gp[0, k])
    d = np.random.default_rng(1).normal(size=v0.shape)
    h = 1e-3 * np.abs(v0).mean()
    fd = (loss(scene, v0 + h * d) - loss(scene, v0 - h * d)) / (2 * h)
    directional = float(np.sum(gv.astype(np.float64) * d))
    assert abs(fd - directional) <= 5e-2 * abs(fd), (fd, directional)


def test_checkpoint_interval_changes_gradients_by_rounding_only():
    steps = 30
    scenes, dts = _scenes(2, steps=steps)
    targets = _targets(scenes)
    engine = _engine(scenes)
    try:
        results = []
        for every in (1, 7, 30):
            engine.forward(steps, dts, targets, checkpoint_every=every)
            results.append(engine.backward())
    finally:
        engine.dispose()
    gv0, gp0 = results[0]
    for gv, gp in results[1:]:
        assert np.allclose(gp, gp0, rtol=1e-3, atol=1e-6 * np.abs(gp0).max())
        assert np.linalg.norm(gv - gv0) <= 1e-3 * np.linalg.norm(gv0)


def test_adjoint_at_the_full_horizon_with_checkpoints():
    # the differentiable workload's horizon: 200 substeps, a checkpoint every
    # 20, on the 1,024-particle subset; against the FP64 adjoint and a
    # directional central difference of the FP64 forward (relative step 1e-3)
    steps = 200
    scenes, dts = _scenes(1, steps=steps)
    (p, c, t), = scenes
    engine = _engine(scenes)
    try:
        loss = engine.forward(steps, dts, t, checkpoint_every=20)
        gv, gp = engine.backward()
    finally:
        engine.dispose()
    ref_loss, ref_gv, ref_gp, _ = _fp64(p, c, t, dts[0], steps)
    assert abs(loss[0] - ref_loss) <= 1e-3 * ref_loss
    for k in range(3):
        assert abs(gp[0, k] - ref_gp[k]) <= 5e-2 * abs(ref_gp[k]) + 1e-6 * np.abs(ref_gp).max(), (k, gp[0], ref_gp)
    a, b = gv.astype(np.float64).ravel(), ref_gv.ravel()
    cosine = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
    assert cosine > 0.995, cosine
    assert np.linalg.norm(a - b) <= 1e-1 * np.linalg.norm(b)
    state = validate_mpm_mls_gpu_input(p, c)
    pk = state.packed_particles
    liquid = pk[:, 13].view(np.uint32) == 2
    pk64 = pk.astype(np.float64)
    water, solid = pk64[liquid][0], pk64[~liquid][0]
    scene = {"cells_x": 64, "cells_y": 64, "dx": 10.0, "dt": dts[0], "gx": ADJOINT_GRAVITY["x"],
             "gy": ADJOINT_GRAVITY["y"], "solid_mass": float(np.float32(c["particleMass"])), "wall_friction": 0.0,
             "rho": float(water[16]), "gamma": float(water[18]), "tait": float(water[14]),
             "lambda_s": float(solid[14]), "mu_s": float(solid[15])}
    target = np.asarray(t, np.float32).astype(np.float64)
    v0 = pk64[:, 2:4]
    d = np.random.default_rng(2).normal(size=v0.shape)
    h = 1e-3 * np.abs(v0).mean()

    def fp64_loss(v):
        return adjoint_fp64(scene, pk64[:, 0:2], v, pk64[:, 4:8], pk64[:, 8:12], pk64[:, 17],
                            liquid.astype(np.int32), target, steps)[0]

    fd = (fp64_loss(v0 + h * d) - fp64_loss(v0 - h * d)) / (2 * h)
    directional = float(np.sum(gv.astype(np.float64) * d))
    assert abs(fd - directional) <= 5e-2 * abs(fd), (fd, directional)
