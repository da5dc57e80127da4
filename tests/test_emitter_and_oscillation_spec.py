"""The emitter and the oscillating gravity input, restating
src/lib/mpm/scenes/emitter.spec.ts and src/lib/mpm/kernels/oscillation.spec.ts
on the host mirror (create_mpm_emitter_particles, mean_sinusoidal_acceleration).
"""
import math

import pytest

from mpm_b200 import RangeError
from mpm_b200.scenes import (GATE4_LIQUID_BULK_MODULUS_SCALE, GATE4_LIQUID_PARTICLE_AREA,
                              create_mpm_emitter_particles)
from mpm_b200.step_scheduler import (DEFAULT_HORIZONTAL_OSCILLATION_AMPLITUDE, HORIZONTAL_OSCILLATION_FREQUENCY_HZ,
                                     INITIAL_HORIZONTAL_OSCILLATION_AMPLITUDE, mean_sinusoidal_acceleration)

BASE_CONFIG = {
    "count": 24,
    "seed": 0x51EED,
    "center": {"x": 24, "y": 24},
    "shape": "circle",
    "spacing": 1,
    "velocity": {"x": 2, "y": -3},
    "material": "water",
    "grid": {"cellsX": 64, "cellsY": 64, "cellSize": 1},
}


def test_the_emitter_is_repeatable_and_phase_specific():
    first = create_mpm_emitter_particles(BASE_CONFIG)
    second = create_mpm_emitter_particles(BASE_CONFIG)
    assert first == second
    assert len(first) == BASE_CONFIG["count"]
    assert all(p["material"]["model"] == "water" for p in first)
    assert all(p["material"]["lambda"] == 40_000 * GATE4_LIQUID_BULK_MODULUS_SCALE for p in first)
    assert all(p["volume"] == 25 for p in first)
    assert all(p["velocity"] == {"x": 2, "y": -3} for p in first)
    assert all(p["position"]["x"] >= 0 and p["position"]["y"] >= 0 for p in first)


def test_the_emitter_supports_oil_solid_and_rectangle_sources():
    water = create_mpm_emitter_particles(dict(BASE_CONFIG, particleVolume=GATE4_LIQUID_PARTICLE_AREA))
    oil = create_mpm_emitter_particles(dict(BASE_CONFIG, material="oil", particleVolume=GATE4_LIQUID_PARTICLE_AREA))
    solid = create_mpm_emitter_particles(dict(BASE_CONFIG, material="neo-hookean", shape="rectangle",
                                              particleVolume=100))
    assert all(p["volume"] == GATE4_LIQUID_PARTICLE_AREA for p in water)
    assert all(p["material"]["model"] == "oil" for p in oil)
    assert all(p["material"]["lambda"] == 30_000 * GATE4_LIQUID_BULK_MODULUS_SCALE for p in oil)
    assert all(p["material"]["model"] == "neo-hookean" for p in solid)
    assert all(p["volume"] == 100 for p in solid)
    assert all(p["volume"] == GATE4_LIQUID_PARTICLE_AREA for p in oil)
    assert len({(p["position"]["x"], p["position"]["y"]) for p in solid}) == BASE_CONFIG["count"]


@pytest.mark.parametrize("change,message", [
    ({"count": 0}, "count"),
    ({"seed": -1}, "seed"),
    ({"particleVolume": 0}, "particleVolume"),
    ({"center": {"x": 0, "y": 0}, "count": 16}, "outside the simulation domain"),
], ids=["count", "seed", "particleVolume", "domain"])
def test_the_emitter_rejects_unsafe_inputs_rather_than_emitting_partial_batches(change, message):
    with pytest.raises(RangeError, match=message):
        create_mpm_emitter_particles(dict(BASE_CONFIG, **change))


PERIOD = 1 / HORIZONTAL_OSCILLATION_FREQUENCY_HZ
AMPLITUDE = 240


def test_a_full_oscillation_averages_to_zero():
    assert mean_sinusoidal_acceleration(0, PERIOD, AMPLITUDE) == pytest.approx(0, abs=5e-13)


def test_the_batch_interval_average_is_the_time_average():
    assert mean_sinusoidal_acceleration(0, PERIOD / 2, AMPLITUDE) == pytest.approx(2 * AMPLITUDE / math.pi,
                                                                                 abs=5e-13)


def test_a_disabled_oscillation_is_zero():
    assert mean_sinusoidal_acceleration(2, 1, 0) == 0


def test_the_default_horizontal_oscillation_is_enabled():
    assert DEFAULT_HORIZONTAL_OSCILLATION_AMPLITUDE == 240
    assert INITIAL_HORIZONTAL_OSCILLATION_AMPLITUDE == DEFAULT_HORIZONTAL_OSCILLATION_AMPLITUDE


def test_invalid_intervals_and_frequencies_are_rejected():
    with pytest.raises(RangeError):
        mean_sinusoidal_acceleration(0, -1, 1)
    with pytest.raises(RangeError):
        mean_sinusoidal_acceleration(0, 1, 1, -0.1)
