"""The Tait equation of state of the reference's SI water scenes
(src/lib/mpm/reference/tait-eos.ts): the pressure coefficient derived from a
sound speed, the pressure, bulk modulus and sound speed at a density, and the
isotropic P F^T term of a liquid particle at a volume ratio J = det F.

The device kernels evaluate the same stress per particle in float32 (the
Tait branch of prepareParticle): -J * lambda * (J^-gamma - 1), with lambda the
areal pressure coefficient (pressure coefficient x extrusion depth).  The
functions here are the host-side reference values that pin it.
"""
from __future__ import annotations

import math

from .errors import RangeError

ATMOSPHERIC_PRESSURE_PA = 101_325.0  # src/lib/mpm/reference/gas-state.ts:3


def _finite(value, name: str) -> float:
    if isinstance(value, bool) or not isinstance(value, (int, float)) or not math.isfinite(value):
        raise RangeError(f"{name} must be a finite number.")
    return float(value)


def _positive(value, name: str) -> float:
    v = _finite(value, name)
    if v <= 0:
        raise RangeError(f"{name} must be a finite positive number.")
    return v


def _validate_parameters(parameters) -> None:
    """validateParameters, tait-eos.ts:64-71."""
    if not isinstance(parameters, dict):
        raise TypeError("parameters must be an object.")
    _positive(parameters.get("referenceDensityKgPerM3"), "referenceDensityKgPerM3")
    _positive(parameters.get("exponent"), "exponent")
    _positive(parameters.get("pressureCoefficientPa"), "pressureCoefficientPa")
    if parameters.get("ambientPressurePa") is not None:
        _positive(parameters["ambientPressurePa"], "ambientPressurePa")


def derive_tait_pressure_coefficient_pa(reference_density, exponent, sound_speed) -> float:
    """deriveTaitPressureCoefficientPa, tait-eos.ts:73-86: B = rho c^2 / gamma."""
    rho = _positive(reference_density, "referenceDensityKgPerM3")
    gamma = _positive(exponent, "exponent")
    c = _positive(sound_speed, "soundSpeedMPerS")
    return _positive((rho * c * c) / gamma, "calculated pressureCoefficientPa")


def evaluate_tait_eos(density, parameters) -> dict:
    """evaluateTaitEos, tait-eos.ts:88-141: gauge p = B ((rho / rho0)^gamma - 1),
    absolute = ambient + gauge (must stay positive: no cavitation model), bulk
    modulus gamma B (rho / rho0)^gamma, sound speed sqrt(K / rho)."""
    rho = _positive(density, "densityKgPerM3")
    _validate_parameters(parameters)
    ambient = parameters.get("ambientPressurePa")
    ambient = ATMOSPHERIC_PRESSURE_PA if ambient is None else float(ambient)
    rho0, gamma, b = (float(parameters["referenceDensityKgPerM3"]), float(parameters["exponent"]),
                      float(parameters["pressureCoefficientPa"]))
    ratio = _positive(rho / rho0, "calculated densityRatio")
    try:
        power = ratio ** gamma
    except OverflowError:
        power = math.inf
    power = _positive(power, "calculated density ratio power")
    k0 = _positive(gamma * b, "calculated referenceBulkModulusPa")
    c0 = _positive(math.sqrt(k0 / rho0), "calculated referenceSoundSpeedMPerS")
    gauge = _finite(b * (power - 1), "calculated gaugePressurePa")
    absolute = _finite(ambient + gauge, "calculated absolutePressurePa")
    if absolute <= 0:
        raise RangeError("calculated absolutePressurePa must be positive; low-pressure or cavitation handling is "
                         "required.")
    k = _positive(k0 * power, "calculated bulkModulusPa")
    c = _positive(math.sqrt(k / rho), "calculated soundSpeedMPerS")
    return {"densityKgPerM3": rho, "gaugePressurePa": gauge, "absolutePressurePa": absolute, "bulkModulusPa": k,
            "soundSpeedMPerS": c, "referenceSoundSpeedMPerS": c0}


def evaluate_tait_fluid_stress_from_volume_ratio(volume_ratio, parameters) -> dict:
    """evaluateTaitFluidStressFromVolumeRatio, tait-eos.ts:143-166: the
    isotropic P F^T = -J p_gauge at density rho0 / J (no -0)."""
    j = _positive(volume_ratio, "volumeRatio")
    _validate_parameters(parameters)
    rho = _positive(float(parameters["referenceDensityKgPerM3"]) / j, "calculated densityKgPerM3")
    pressure = evaluate_tait_eos(rho, parameters)
    raw = _finite(-j * pressure["gaugePressurePa"], "calculated stressTimesFtIsotropicPa")
    return {"volumeRatio": j, "pressure": pressure, "stressTimesFtIsotropicPa": 0.0 if raw == 0 else raw}


def create_mpm_tait_liquid_material(parameters, extrusion_depth_m, model: str = "water") -> dict:
    """createMpmTaitLiquidMaterial, tait-eos.ts:26-44: areal density and
    pressure coefficient (x extrusion depth) of a Tait liquid."""
    _validate_parameters(parameters)
    depth = _positive(extrusion_depth_m, "extrusionDepthM")
    density = _positive(parameters["referenceDensityKgPerM3"] * depth, "calculated areal reference density")
    lam = _positive(parameters["pressureCoefficientPa"] * depth, "calculated areal pressure coefficient")
    return {"model": model, "lambda": lam, "mu": 0.0, "density": density,
            "equationOfState": {"model": "tait", "exponent": parameters["exponent"]}}
