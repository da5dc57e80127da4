"""The reference's own known answers, evaluated by the device code (C ABI).

* The float32 deformation update of a near-singular F at the reported
  increment scale, src/lib/mpm/kernels/solver.spec.ts:197-278: increment
  0.35687583684921265, 2 substeps, det > 0 with the fused products (and
  <= 0 without them).  The device's trial F is also checked bit for bit
  against an exact emulation of the fused products (every product and sum
  rounded once to float32, as the kernel's fmaf / __fmul_rn / __fadd_rn do).
* The Tait pressure term of prepareParticle against the reference's EOS,
  src/lib/mpm/reference/tait-eos.spec.ts:80-102 (isotropic P F^T = -J p_gauge):
  relative agreement 2e-5 (float32 pow evaluated as exp2(gamma log2 x)), and
  exactly zero at J = 1.
"""
import ctypes
from fractions import Fraction

import numpy as np
import pytest

from mpm_b200 import _lib, create_experimental_mpm_mls_atomic_gpu_solver
from mpm_b200.tait_eos import (create_mpm_tait_liquid_material, derive_tait_pressure_coefficient_pa,
                               evaluate_tait_fluid_stress_from_volume_ratio)

pytestmark = pytest.mark.gpu

INITIAL = [0.06047571077942848, 0.17931117117404938, 0.17301689088344574, 0.5129971504211426]
GRADIENT = [0.1195390224456787, 0.15536771714687347, 0.040612027049064636, 0.3162637948989868]


def round_f32(value: Fraction) -> np.float32:
    """Correctly rounded (ties to even) float32 of an exact rational."""
    guess = np.float32(float(value))
    best = None
    for cand in (np.nextafter(guess, np.float32(-np.inf)), guess, np.nextafter(guess, np.float32(np.inf))):
        err = abs(Fraction(float(cand)) - value)
        key = (err, int(np.float32(cand).view(np.uint32)) & 1)
        if best is None or key < best[0]:
            best = (key, cand)
    return np.float32(best[1])


def fused_trial(initial, gradient, dt, substeps, fused=True):
    """integrateDeformation (shaders.ts:1459-1483) in exact float32 steps."""
    F = [Fraction(float(np.float32(v))) for v in initial]
    C = [np.float32(v) for v in gradient]
    h = np.float32(dt) if substeps == 1 else round_f32(Fraction(float(np.float32(dt))) / substeps)
    H = Fraction(float(h))
    u = [round_f32(1 + Fraction(float(round_f32(H * Fraction(float(C[0])))))),
         round_f32(H * Fraction(float(C[1]))), round_f32(H * Fraction(float(C[2]))),
         round_f32(1 + Fraction(float(round_f32(H * Fraction(float(C[3]))))))]
    U = [Fraction(float(v)) for v in u]

    def dot(a, b, c, d):
        second = Fraction(float(round_f32(c * d)))
        if fused:
            return Fraction(float(round_f32(a * b + second)))
        return Fraction(float(round_f32(Fraction(float(round_f32(a * b))) + second)))

    r = F
    for _ in range(substeps):
        r = [dot(U[0], r[0], U[1], r[2]), dot(U[0], r[1], U[1], r[3]),
             dot(U[2], r[0], U[3], r[2]), dot(U[2], r[1], U[3], r[3])]
    return np.array([float(v) for v in r], dtype=np.float32)


def probe_deformation(F, C, dt):
    lib = _lib.load_library()
    F = np.ascontiguousarray(F, dtype=np.float32).reshape(-1, 4)
    C = np.ascontiguousarray(C, dtype=np.float32).reshape(-1, 4)
    n = F.shape[0]
    trial = np.zeros((n, 4), np.float32)
    inc = np.zeros(n, np.float32)
    det = np.zeros(n, np.float32)
    sub = np.zeros(n, np.uint32)
    flags = np.zeros(n, np.uint32)
    rc = lib.mpm_probe_deformation(0, _lib.ptr(F), _lib.ptr(C), n, ctypes.c_float(dt), _lib.ptr(trial),
                                   _lib.ptr(inc), _lib.ptr(det), _lib.ptr(sub), _lib.ptr(flags))
    assert rc == _lib.MPM_OK, _lib.last_error()
    return trial, inc, det, sub, flags


def test_near_singular_deformation_keeps_its_orientation_on_the_device():
    trial, inc, det, sub, flags = probe_deformation(INITIAL, GRADIENT, 1.0)
    assert flags[0] == 0
    assert float(inc[0]) == 0.35687583684921265
    assert int(sub[0]) == 2
    t = trial[0].astype(np.float64)
    # the reference's determinant of the fused trial (JavaScript doubles)
    assert t[0] * t[3] - t[1] * t[2] > 0
    assert float(det[0]) > 0
    # bit for bit: the fused products, each rounded once
    expected = fused_trial(INITIAL, GRADIENT, 1.0, 2)
    assert np.array_equal(trial[0].view(np.uint32), expected.view(np.uint32))
    # without the fused term the same increments lose the orientation
    unfused = fused_trial(INITIAL, GRADIENT, 1.0, 2, fused=False).astype(np.float64)
    assert unfused[0] * unfused[3] - unfused[1] * unfused[2] <= 0


def test_deformation_substep_counts_and_limit():
    rng = np.random.default_rng(4)
    F = np.tile(np.array([1.0, 0.0, 0.0, 1.0], np.float32), (6, 1))
    C = np.zeros((6, 4), np.float32)
    C[:, 0] = [0.0, 0.1, 0.24, 0.26, 15.9, 16.1]  # increments at dt = 1: 1, 1, 1, 2, 64, 65 substeps
    trial, inc, det, sub, flags = probe_deformation(F, C, 1.0)
    assert sub[:5].tolist() == [1, 1, 1, 2, 64]
    assert flags[:5].tolist() == [0] * 5 and flags[5] == 32  # ERROR_DEFORMATION_SUBSTEP_LIMIT
    for k in range(5):
        expected = fused_trial(F[k], C[k], 1.0, int(sub[k]))
        assert np.array_equal(trial[k].view(np.uint32), expected.view(np.uint32)), k
    # random well-conditioned cases at small dt match the exact emulation too
    F = (np.eye(2, dtype=np.float32).reshape(1, 4) + rng.uniform(-0.2, 0.2, (16, 4))).astype(np.float32)
    C = rng.uniform(-50, 50, (16, 4)).astype(np.float32)
    trial, inc, det, sub, flags = probe_deformation(F, C, 2e-3)
    for k in range(16):
        if flags[k] == 0 and det[k] > 0:
            expected = fused_trial(F[k], C[k], 2e-3, int(sub[k]))
            assert np.array_equal(trial[k].view(np.uint32), expected.view(np.uint32)), k


def test_tait_stress_of_prepare_particle_matches_the_reference_eos():
    params = {"referenceDensityKgPerM3": 998.2, "exponent": 7.15,
              "pressureCoefficientPa": derive_tait_pressure_coefficient_pa(998.2, 7.15, 20)}
    depth = 0.02
    material = create_mpm_tait_liquid_material(params, depth)
    ratios = [0.99, 0.995, 1.0, 1.005, 1.01]
    area = 0.0025 ** 2 / 4
    particles = []
    for k, j in enumerate(ratios):
        a = float(np.float32(np.sqrt(j)))
        particles.append({"position": {"x": 0.01 + 0.005 * k, "y": 0.02}, "velocity": {"x": 0, "y": 0},
                          "C": {"m00": 0, "m01": 0, "m10": 0, "m11": 0},
                          "F": {"m00": a, "m01": 0, "m10": 0, "m11": a}, "material": material, "volume": area})
    config = {"grid": {"cellsX": 16, "cellsY": 16, "cellSize": 0.0025}, "particleMass": material["density"] * area,
              "particleVolume": area, "material": material}
    dt = 1e-5
    solver = create_experimental_mpm_mls_atomic_gpu_solver(particles, config, fixed_point_shift=24)
    try:
        _, affine = solver.probe_fixed_point(dt)
    finally:
        solver.dispose()
    gs = np.float32(4.0 / (0.0025 * 0.0025))
    scale = float(np.float32(np.float32(-np.float32(dt) * np.float32(area)) * gs))
    for k, j in enumerate(ratios):
        a = np.float32(np.sqrt(j))
        det = float(np.float32(a * a))  # the compensated determinant of a diagonal F: one rounding
        expected = evaluate_tait_fluid_stress_from_volume_ratio(det, params)["stressTimesFtIsotropicPa"] * depth
        got = float(affine[k, 0]) / scale
        assert affine[k, 1] == 0 and affine[k, 2] == 0
        assert affine[k, 0] == affine[k, 3]
        if det == 1.0:
            assert got == 0.0
        else:
            assert abs(got - expected) <= 2e-5 * abs(expected), (j, got, expected)
