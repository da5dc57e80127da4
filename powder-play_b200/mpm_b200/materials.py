"""Constitutive model codes and material constants.

Restates src/lib/mpm/materials.ts (7korobi/powder-play) and the SI domain of
src/lib/mpm/si-domain.ts.
"""
from __future__ import annotations

from .errors import RangeError

MODEL_CODES = {"neo-hookean": 0, "snow": 1, "water": 2, "oil": 3, "powder": 4, "fixed-corotated": 5}
"""materials.ts:8-16.  'fixed-corotated' (code 5) has no reference counterpart:
the snow stress with plastic volume 1 and no plastic projection."""

MODEL_NAMES = {code: name for name, code in MODEL_CODES.items()}

MPM_LIQUID_CONTACT_SEPARATION_FRACTION = 0.25
MPM_LIQUID_CONTACT_APPROACH_SPEED_MULTIPLIER = 1.0
MPM_LIQUID_CONTACT_RELAXATION_SECONDS = 0.05
MPM_LIQUID_STABLE_ORDER_EPSILON = 1e-3
MPM_TRIANGLE_FLUID_TANGENTIAL_DRAG_RATE = 4.0

SNOW_PLASTICITY = {
    "compressionYield": 0.025,
    "stretchYield": 0.0075,
    "hardening": 10.0,
    "minPlasticVolume": 0.6,
    "maxPlasticVolume": 20.0,
    "maxHardeningExponent": 20.0,
}

MPM_SI_BOX_DOMAIN = {
    "innerWidthM": 0.2,
    "innerHeightM": 0.2,
    "extrusionDepthM": 0.02,
    "exteriorWallThicknessM": 0.05,
}


def normalize_mpm_constitutive_model(value, name: str) -> str:
    """normalizeMpmConstitutiveModel, materials.ts:56-69."""
    if value is None or value == "neo-hookean":
        return "neo-hookean"
    if value in ("snow", "water", "oil", "powder", "fixed-corotated"):
        return value
    raise RangeError(f"{name} must be 'neo-hookean', 'snow', 'water', 'oil', or 'powder'")


def normalize_mpm_tait_equation_of_state(value, name: str):
    """normalizeMpmTaitEquationOfState, materials.ts:18-38."""
    if value is None:
        return None
    if not isinstance(value, dict):
        raise TypeError(f"{name} must be an object.")
    if value.get("model") != "tait":
        raise RangeError(f"{name}.model must be 'tait'.")
    exponent = value.get("exponent")
    if not isinstance(exponent, (int, float)) or isinstance(exponent, bool) or not (exponent > 0) or exponent != exponent or exponent == float("inf"):
        raise RangeError(f"{name}.exponent must be positive and finite.")
    return {"model": "tait", "exponent": float(exponent)}


def encode_mpm_constitutive_model(model: str) -> int:
    return MODEL_CODES[model]


def decode_mpm_constitutive_model(code: int) -> str:
    """decodeMpmConstitutiveModel, materials.ts:75-90."""
    if code not in MODEL_NAMES:
        raise RangeError(f"GPU returned an unsupported MPM material model {code}.")
    return MODEL_NAMES[code]
