"""Known answers from the reference's own specs, restated on the host side.

* Tait equation of state: src/lib/mpm/reference/tait-eos.spec.ts:17-193.
* Packing of the 20-word particle record (the wire format of the C ABI):
  src/lib/mpm/kernels/layout.spec.ts:67-93 and :272-380.
* The float32 deformation-increment arithmetic of
  src/lib/mpm/kernels/solver.spec.ts:197-278 (the device's own evaluation of
  the same case is in tests/test_gpu_known_answers.py).
"""
import math

import numpy as np
import pytest

from mpm_b200.errors import RangeError
from mpm_b200.layout import PARTICLE_STRIDE_BYTES, fround, validate_mpm_mls_gpu_input
from mpm_b200.solver import native_config
from mpm_b200.tait_eos import (ATMOSPHERIC_PRESSURE_PA, create_mpm_tait_liquid_material,
                               derive_tait_pressure_coefficient_pa, evaluate_tait_eos,
                               evaluate_tait_fluid_stress_from_volume_ratio)

WATER_REFERENCE = {"referenceDensityKgPerM3": 998.2, "exponent": 7.15}


def close_to(actual, expected, digits):
    """vitest toBeCloseTo(expected, digits): |actual - expected| < 10^-digits / 2."""
    return abs(actual - expected) < 10 ** (-digits) / 2


# ------------------------------------------------------------ tait-eos.spec --

def test_tait_pressure_coefficient_from_the_reference_sound_speed():
    b = derive_tait_pressure_coefficient_pa(998.2, 7.15, 1_482)
    assert close_to(b, 306_625_260, -4)
    ev = evaluate_tait_eos(998.2, dict(WATER_REFERENCE, pressureCoefficientPa=b))
    assert ev["gaugePressurePa"] == 0
    assert ev["absolutePressurePa"] == ATMOSPHERIC_PRESSURE_PA
    assert close_to(ev["referenceSoundSpeedMPerS"], 1_482, 10)
    assert close_to(ev["soundSpeedMPerS"], 1_482, 10)
    assert close_to(ev["bulkModulusPa"], 7.15 * b, 8)


def test_tait_compression_and_expansion_without_clamping_tension():
    b = derive_tait_pressure_coefficient_pa(998.2, 7.15, 20)
    params = dict(WATER_REFERENCE, pressureCoefficientPa=b)
    compression = evaluate_tait_eos(998.2 * 1.01, params)
    expansion = evaluate_tait_eos(998.2 * 0.99, params)
    assert compression["gaugePressurePa"] > 0
    assert compression["absolutePressurePa"] > ATMOSPHERIC_PRESSURE_PA
    assert compression["soundSpeedMPerS"] > 20
    assert expansion["gaugePressurePa"] < 0
    assert expansion["absolutePressurePa"] > 0
    assert expansion["soundSpeedMPerS"] < 20


def test_tait_rejects_a_non_positive_absolute_pressure():
    b = derive_tait_pressure_coefficient_pa(998.2, 7.15, 1_482)
    with pytest.raises(RangeError, match="low-pressure or cavitation handling is required"):
        evaluate_tait_eos(998.2 * 0.9, dict(WATER_REFERENCE, pressureCoefficientPa=b))


def test_tait_pressure_maps_to_the_isotropic_p_ft_term():
    b = derive_tait_pressure_coefficient_pa(998.2, 7.15, 20)
    params = dict(WATER_REFERENCE, pressureCoefficientPa=b)
    equilibrium = evaluate_tait_fluid_stress_from_volume_ratio(1, params)
    compressed = evaluate_tait_fluid_stress_from_volume_ratio(0.99, params)
    expanded = evaluate_tait_fluid_stress_from_volume_ratio(1.01, params)
    assert equilibrium["pressure"]["gaugePressurePa"] == 0
    assert equilibrium["stressTimesFtIsotropicPa"] == 0
    assert math.copysign(1.0, equilibrium["stressTimesFtIsotropicPa"]) == 1.0  # no -0
    assert compressed["pressure"]["gaugePressurePa"] > 0
    assert close_to(compressed["stressTimesFtIsotropicPa"], -0.99 * compressed["pressure"]["gaugePressurePa"], 10)
    assert compressed["stressTimesFtIsotropicPa"] < 0
    assert expanded["pressure"]["gaugePressurePa"] < 0
    assert expanded["stressTimesFtIsotropicPa"] > 0


def test_tait_si_parameters_become_areal_material_values():
    b = derive_tait_pressure_coefficient_pa(998.2, 7.15, 20)
    material = create_mpm_tait_liquid_material(dict(WATER_REFERENCE, pressureCoefficientPa=b), 0.02)
    assert material == {"model": "water", "lambda": b * 0.02, "mu": 0.0, "density": 998.2 * 0.02,
                        "equationOfState": {"model": "tait", "exponent": 7.15}}


def test_tait_explicit_ambient_pressure():
    b = derive_tait_pressure_coefficient_pa(1_000, 7, 20)
    ev = evaluate_tait_eos(1_010, {"referenceDensityKgPerM3": 1_000, "exponent": 7, "pressureCoefficientPa": b,
                                   "ambientPressurePa": 90_000})
    assert close_to(ev["absolutePressurePa"], 90_000 + b * (1.01 ** 7 - 1), 8)


def test_tait_rejects_invalid_inputs():
    valid = dict(WATER_REFERENCE, pressureCoefficientPa=55_000)
    for invalid in (0, -1, math.nan, math.inf):
        with pytest.raises(RangeError):
            evaluate_tait_eos(invalid, valid)
        with pytest.raises(RangeError):
            derive_tait_pressure_coefficient_pa(invalid, 7.15, 20)
        with pytest.raises(RangeError):
            derive_tait_pressure_coefficient_pa(1_000, invalid, 20)
        with pytest.raises(RangeError):
            derive_tait_pressure_coefficient_pa(1_000, 7, invalid)
    with pytest.raises(TypeError, match="parameters must be an object"):
        evaluate_tait_eos(1_000, None)
    with pytest.raises(RangeError, match="referenceBulkModulusPa"):
        evaluate_tait_eos(1_000, dict(valid, pressureCoefficientPa=1.7976931348623157e308))


# ----------------------------------------------------------- layout.spec --

def _layout_config(**overrides):
    """makeConfig of layout.spec.ts:23-31."""
    cfg = {"grid": {"cellsX": 16, "cellsY": 8, "cellSize": 1}, "particleMass": 0.1, "particleVolume": 0.01,
           "material": {"lambda": 20, "mu": 10}}
    cfg.update(overrides)
    return cfg


def _layout_particle(**overrides):
    """makeParticle of layout.spec.ts:33-41."""
    p = {"position": {"x": 8, "y": 4}, "velocity": {"x": 0, "y": 0},
         "C": {"m00": 0, "m01": 0, "m10": 0, "m11": 0}, "F": {"m00": 1, "m01": 0, "m10": 0, "m11": 1}}
    p.update(overrides)
    return p


def test_packs_the_complete_particle_state_at_both_domain_edges():
    state = validate_mpm_mls_gpu_input([_layout_particle(position={"x": 0, "y": 0}),
                                        _layout_particle(position={"x": 16, "y": 8})], _layout_config())
    packed = state.packed_particles
    words = packed.view(np.uint32)
    assert packed[0, 0:12].tolist() == [0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 1]
    assert packed[0, 12] == 1
    assert words[0, 13] == 0
    assert packed[0, 14:16].tolist() == [20, 10]
    assert packed[1, 0:2].tolist() == [16, 8]
    assert state.particle_count == 2 and state.particle_capacity == 2
    assert state.packed_object_ids.tolist() == [0, 0]
    assert state.domain_width == 16 and state.domain_height == 8
    assert state.domain_width_f32 == 16 and state.domain_height_f32 == 8
    assert PARTICLE_STRIDE_BYTES == 80 and packed.dtype == np.float32 and packed.shape[1] * 4 == 80


def test_packs_material_and_snow_plastic_history():
    particles = [_layout_particle(objectId=3, plasticVolume=0.82, material={"lambda": 36, "mu": 18, "model": "snow"}),
                 _layout_particle(position={"x": 9, "y": 4}, objectId=3,
                                  material={"lambda": 24, "mu": 12, "model": "neo-hookean"})]
    state = validate_mpm_mls_gpu_input(particles, _layout_config())
    flat = state.packed_particles.reshape(-1)
    words = flat.view(np.uint32)
    assert flat[12] == np.float32(fround(0.82))
    assert words[13] == 1
    assert flat[14:16].tolist() == [36, 18]
    assert flat[32] == 1
    assert words[33] == 0
    assert flat[34:36].tolist() == [24, 12]
    assert flat[16:20].tolist() == [0, np.float32(0.01), 0, 0]


def test_packs_liquid_density_volume_and_powder_friction():
    particles = [_layout_particle(material={"lambda": 8, "mu": 0, "model": "water", "density": 1}, volume=0.02),
                 _layout_particle(position={"x": 9, "y": 4},
                                  material={"lambda": 6, "mu": 0, "model": "oil", "density": 0.8}),
                 _layout_particle(position={"x": 10, "y": 4},
                                  material={"lambda": 20, "mu": 10, "model": "powder", "frictionCoefficient": 0.55})]
    state = validate_mpm_mls_gpu_input(particles, _layout_config())
    flat = state.packed_particles.reshape(-1)
    words = flat.view(np.uint32)
    assert words[13] == 2
    assert flat[14:19].tolist() == [8, 0, 1, np.float32(0.02), 0]
    assert words[33] == 3
    assert flat[36] == np.float32(0.8)
    assert flat[37] == np.float32(0.01)
    assert words[53] == 4
    assert flat[58] == np.float32(0.55)


def test_packs_the_tait_exponent_and_wall_friction_without_changing_the_stride():
    material = {"lambda": 1_116, "mu": 0, "model": "water", "density": 19.964,
                "equationOfState": {"model": "tait", "exponent": 7.15}}
    state = validate_mpm_mls_gpu_input([_layout_particle(material=material)],
                                       _layout_config(material=material, wallFriction=1))
    assert state.packed_particles[0, 18] == np.float32(fround(7.15))
    assert state.packed_particles.shape == (1, 20)
    # the per-solver wall-friction parameter (the reference's step-parameter word at byte 128)
    assert native_config(state, False, 24, 0).wall_friction == 1.0


# ------------------------------------------------- solver.spec.ts:197-278 --

def test_near_singular_deformation_increment_arithmetic():
    f32 = np.float32
    initial = np.array([0.06047571077942848, 0.17931117117404938, 0.17301689088344574, 0.5129971504211426], f32)
    gradient = np.array([0.1195390224456787, 0.15536771714687347, 0.040612027049064636, 0.3162637948989868], f32)
    row = max(f32(abs(gradient[0])) + f32(abs(gradient[1])), f32(abs(gradient[2])) + f32(abs(gradient[3])))
    assert float(row) == 0.35687583684921265
    assert max(1, math.ceil(float(row) / 0.25)) == 2
    det = float(initial[0]) * float(initial[3]) - float(initial[1]) * float(initial[2])
    assert 0 < det < 1e-8
