"""CFL wave-speed and velocity bounds: src/lib/mpm/kernels/cfl-bounds.ts.

`derive_mpm_mls_gpu_cfl_bounds` (:32-73, per-particle :75-142, vectorised over
particles) and `calculate_mpm_cfl_velocity_bound` (:153-184), with the
8-ulp float32 round-up (:186-208).
"""
from __future__ import annotations

import math
import struct

import numpy as np

from .errors import RangeError
from .layout import as_particle_arrays, fround

F32_ROUNDING_ULPS = 8


def round_up_float32_ulps(value: float) -> float:
    """roundUpFloat32 with 8 extra ulps, cfl-bounds.ts:186-208."""
    if not math.isfinite(value) or value < 0:
        raise RangeError("CFL bounds must be finite and non-negative.")
    if value == 0:
        return 0.0
    bits = struct.unpack("<I", struct.pack("<f", fround(value)))[0]
    as_f = lambda b: struct.unpack("<f", struct.pack("<I", b))[0]  # noqa: E731
    while as_f(bits) < value:
        bits += 1
    bits += F32_ROUNDING_ULPS
    rounded = as_f(bits)
    if not math.isfinite(rounded):
        raise RangeError("CFL bound cannot be represented as a finite float32 value.")
    return rounded


def derive_mpm_mls_gpu_cfl_bounds(particles, config: dict):
    """deriveMpmMlsGpuCflBounds -> {'waveSpeedBound', 'velocityBound'} or None."""
    a = as_particle_arrays(particles)
    n = len(a)
    if n == 0:
        return {"waveSpeedBound": 0.0, "velocityBound": 0.0}
    with np.errstate(over="ignore", invalid="ignore"):
        vx = a.vx.astype(np.float32).astype(np.float64)
        vy = a.vy.astype(np.float32).astype(np.float64)
    if not (np.all(np.isfinite(vx)) and np.all(np.isfinite(vy))):
        bad = int(np.flatnonzero(~(np.isfinite(vx) & np.isfinite(vy)))[0])
        raise RangeError(f"particle {bad} has a non-finite initial velocity.")
    velocity = float(np.max(np.hypot(vx, vy)))
    materials = list(a.materials) + [config["material"]]
    mat_index = np.where(a.material >= 0, a.material, len(a.materials))
    wave = 0.0
    for k, material in enumerate(materials):
        sel = np.flatnonzero(mat_index == k)
        if sel.size == 0:
            continue
        speeds = _material_wave_speeds(a, sel, material, config)
        if speeds is None:
            return None
        wave = max(wave, float(np.max(speeds)))
    return {"waveSpeedBound": round_up_float32_ulps(wave), "velocityBound": round_up_float32_ulps(velocity)}


def _f32(x):
    with np.errstate(over="ignore"):
        return np.asarray(x, dtype=np.float64).astype(np.float32).astype(np.float64)


def _material_wave_speeds(a, sel, material, config):
    """deriveParticleWaveSpeedBound, cfl-bounds.ts:75-142."""
    lam = fround(material["lambda"])
    mu = fround(material.get("mu", 0.0))
    if not math.isfinite(lam) or not math.isfinite(mu):
        raise RangeError("CFL material parameters must be finite float32 values.")
    model = material.get("model")
    if model in ("water", "oil"):
        density = fround(material["density"])
        if not math.isfinite(density) or density <= 0 or lam <= 0:
            raise RangeError("liquid CFL parameters require positive finite lambda and density.")
        eos = material.get("equationOfState")
        if not eos or eos.get("model") != "tait":
            return np.full(sel.size, math.sqrt(lam / density))
        exponent = fround(eos["exponent"])
        F = _f32(a.F[sel])
        det = _f32(F[:, 0] * F[:, 3] - F[:, 1] * F[:, 2])
        if not math.isfinite(exponent) or exponent <= 0 or np.any(~np.isfinite(det)) or np.any(det <= 0):
            raise RangeError("Tait CFL bounds require a positive finite exponent and determinant.")
        c2 = (exponent * lam * np.power(1 / det, exponent - 1)) / density
        if np.any(~np.isfinite(c2)) or np.any(c2 < 0):
            raise RangeError("Tait CFL wave-speed bound is outside the finite range.")
        return np.sqrt(c2)
    if model is not None and model != "neo-hookean":
        return None
    if lam < 0 or mu < 0:
        raise RangeError("Neo-Hookean CFL parameters must be non-negative.")
    volume = _f32(np.where(np.isnan(a.volume[sel]), config["particleVolume"], a.volume[sel]))
    mass = fround(config["particleMass"])
    rho = mass / volume
    F = _f32(a.F[sel])
    det = F[:, 0] * F[:, 3] - F[:, 1] * F[:, 2]
    if (not math.isfinite(mass) or mass <= 0 or np.any(~np.isfinite(volume)) or np.any(volume <= 0)
            or np.any(~np.isfinite(rho)) or np.any(rho <= 0) or np.any(~np.isfinite(det)) or np.any(det <= 0)):
        raise RangeError("Neo-Hookean CFL bounds require positive density and determinant.")
    tr = F[:, 0] ** 2 + F[:, 1] ** 2 + F[:, 2] ** 2 + F[:, 3] ** 2
    disc = np.sqrt(np.maximum(0, tr * tr - 4 * det * det))
    maxs2 = 0.5 * (tr + disc)
    vt = np.abs(lam + mu - lam * np.log(det))
    c2 = (mu * maxs2 + vt) / rho
    if np.any(~np.isfinite(c2)) or np.any(c2 < 0):
        raise RangeError("Neo-Hookean CFL wave-speed bound is outside the finite range.")
    return np.sqrt(c2)


def calculate_mpm_cfl_velocity_bound(currentVelocityBound, durationSeconds, gravityMagnitude, oscillationAmplitude,
                                     dragRadius, dragStiffness, dragDamping) -> float:
    """calculateMpmCflVelocityBound, cfl-bounds.ts:153-184."""
    inputs = (("currentVelocityBound", currentVelocityBound), ("durationSeconds", durationSeconds),
              ("gravityMagnitude", gravityMagnitude), ("oscillationAmplitude", oscillationAmplitude),
              ("dragRadius", dragRadius), ("dragStiffness", dragStiffness), ("dragDamping", dragDamping))
    for name, value in inputs:
        if not isinstance(value, (int, float)) or not math.isfinite(value) or value < 0:
            raise RangeError(f"{name} must be finite and non-negative.")
    acceleration = math.hypot(gravityMagnitude, oscillationAmplitude) + dragRadius * dragStiffness
    bound = currentVelocityBound + acceleration * durationSeconds
    if not math.isfinite(bound):
        raise RangeError("external-input velocity bound exceeds the finite numeric range.")
    return round_up_float32_ulps(bound)
