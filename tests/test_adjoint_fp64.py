"""The FP64 CPU adjoint of the differentiable form (oracle/adjoint_fp64.c)
against central finite differences of its own FP64 forward: the gradient
with respect to the initial velocities (along random directions) and to the
Tait pressure coefficient, solid lambda and solid mu.  CPU only."""
import numpy as np
import pytest

from mpm_b200.adjoint import fixed_cfl_dt
from mpm_b200.layout import validate_mpm_mls_gpu_input
from mpm_b200.scenes import ADJOINT_GRAVITY, create_adjoint_scenes
from oracle import adjoint_fp64


def _small_scene(steps=24, seed=5):
    (particles, config, targets), = create_adjoint_scenes(1, seed=seed, water_columns=12, water_rows=10,
                                                          solid_side=8, cells=40)
    state = validate_mpm_mls_gpu_input(particles, config)
    pk = state.packed_particles.astype(np.float64)
    liquid = (pk[:, 13].view(np.uint32) if pk.dtype == np.float32 else
              state.packed_particles[:, 13].view(np.uint32)) == 2
    water = pk[liquid][0]
    solid = pk[~liquid][0]
    dt = fixed_cfl_dt(particles, config, 90.0, steps * 1e-3)
    scene = {"cells_x": 40, "cells_y": 40, "dx": 10.0, "dt": float(np.float32(dt)), "gx": ADJOINT_GRAVITY["x"],
             "gy": ADJOINT_GRAVITY["y"], "solid_mass": config["particleMass"], "wall_friction": 0.0,
             "rho": float(water[16]), "gamma": float(water[18]), "tait": float(water[14]),
             "lambda_s": float(solid[14]), "mu_s": float(solid[15])}
    arrays = dict(x0=pk[:, 0:2], v0=pk[:, 2:4], C0=pk[:, 4:8], F0=pk[:, 8:12], vol=pk[:, 17],
                  liquid=liquid.astype(np.int32), target=targets)
    return scene, arrays


def _loss(scene, arrays, steps):
    return adjoint_fp64(scene, steps=steps, **arrays)[0]


@pytest.mark.parametrize("steps", [1, 24])
def test_parameter_gradients_match_central_differences(steps):
    scene, arrays = _small_scene()
    loss, gv, gp, _ = adjoint_fp64(scene, steps=steps, **arrays)
    assert np.isfinite(loss) and np.all(np.isfinite(gv)) and np.all(np.isfinite(gp))
    for k, name in enumerate(("tait", "lambda_s", "mu_s")):
        eps = 1e-6 * scene[name]
        up, dn = dict(scene), dict(scene)
        up[name] += eps
        dn[name] -= eps
        fd = (_loss(up, arrays, steps) - _loss(dn, arrays, steps)) / (2 * eps)
        assert abs(fd - gp[k]) <= 1e-5 * abs(fd) + 1e-9 * abs(loss), (name, fd, gp[k])


@pytest.mark.parametrize("steps", [1, 24])
def test_velocity_gradient_matches_central_differences(steps):
    scene, arrays = _small_scene()
    loss, gv, gp, _ = adjoint_fp64(scene, steps=steps, **arrays)
    rng = np.random.default_rng(3)
    for _ in range(3):
        d = rng.normal(size=arrays["v0"].shape)
        eps = 1e-6
        up, dn = dict(arrays), dict(arrays)
        up["v0"] = arrays["v0"] + eps * d
        dn["v0"] = arrays["v0"] - eps * d
        fd = (_loss(scene, up, steps) - _loss(scene, dn, steps)) / (2 * eps)
        directional = float(np.sum(gv * d))
        assert abs(fd - directional) <= 1e-5 * abs(fd) + 1e-9 * abs(loss), (fd, directional)
