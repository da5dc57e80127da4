"""Macrostep / CFL microstep scheduling: src/lib/mpm/kernels/step-scheduler.ts
(`calculateMpmStepBatch` :50-158, `calculateMpmCflStepBatch` :160-200) and
the oscillating gravity input of src/lib/mpm/kernels/oscillation.ts."""
from __future__ import annotations

import math
import re

from .cfl import calculate_mpm_cfl_microsteps, calculate_mpm_cfl_safe_dt
from .cfl_bounds import calculate_mpm_cfl_velocity_bound
from .errors import RangeError
from .layout import _is_safe_integer, fround

DEFAULT_HORIZONTAL_OSCILLATION_AMPLITUDE = 240
INITIAL_HORIZONTAL_OSCILLATION_AMPLITUDE = DEFAULT_HORIZONTAL_OSCILLATION_AMPLITUDE
MAX_HORIZONTAL_OSCILLATION_AMPLITUDE = 360
HORIZONTAL_OSCILLATION_FREQUENCY_HZ = 0.16


def _is_capacity_error(error: Exception) -> bool:
    return isinstance(error, RangeError) and re.search(
        r"exceeds maxMicrosteps|microDt is too small to represent", str(error)) is not None


def calculate_mpm_step_batch(accumulatorSeconds, elapsedSeconds, simulationSpeed, fixedStepSeconds, cellSize,
                             waveSpeedBound, velocityBound, maxMicrosteps, courantLimit=None,
                             allowPartialBatch=False) -> dict:
    """calculateMpmStepBatch, step-scheduler.ts:50-158."""
    for name, value, strict in (("accumulatorSeconds", accumulatorSeconds, False),
                                ("elapsedSeconds", elapsedSeconds, False),
                                ("simulationSpeed", simulationSpeed, False)):
        if not math.isfinite(value) or value < 0:
            raise RangeError(f"{name} must be finite and non-negative.")
    if not math.isfinite(fixedStepSeconds) or fixedStepSeconds <= 0:
        raise RangeError("fixedStepSeconds must be positive and finite.")
    accumulated = accumulatorSeconds + elapsedSeconds * simulationSpeed
    if not math.isfinite(accumulated):
        raise RangeError("accumulated simulation time is outside the supported range.")
    macro_dt = fixedStepSeconds
    try:
        plan = calculate_mpm_cfl_microsteps(macro_dt, cellSize, waveSpeedBound, velocityBound, maxMicrosteps,
                                            courantLimit=courantLimit)
    except RangeError as error:
        if not allowPartialBatch or not _is_capacity_error(error):
            raise
        safe = calculate_mpm_cfl_safe_dt(cellSize, waveSpeedBound, velocityBound, courantLimit)
        reserved = max(1, maxMicrosteps - (1 if maxMicrosteps > 1 else 0))
        macro_dt = min(fixedStepSeconds, safe * reserved * (1 - 1e-6))
        if not math.isfinite(macro_dt) or macro_dt <= 0:
            raise RangeError(f"No positive CFL-safe macrostep duration fits the {maxMicrosteps}-microstep batch cap.")
        plan = calculate_mpm_cfl_microsteps(macro_dt, cellSize, waveSpeedBound, velocityBound, maxMicrosteps,
                                            courantLimit=courantLimit)
    requested = math.floor(accumulated / fixedStepSeconds)
    if not _is_safe_integer(requested):
        raise RangeError("requested macrostep count is outside the supported range.")
    if macro_dt < fixedStepSeconds:
        macro_count = 1 if requested > 0 else 0
    elif allowPartialBatch:
        macro_count = min(requested, maxMicrosteps // plan["stepCount"])
    else:
        macro_count = requested
    micro_count = macro_count * plan["stepCount"]
    if not _is_safe_integer(micro_count) or micro_count > maxMicrosteps:
        raise RangeError(f"requested microstep count ({micro_count}) exceeds maxMicrosteps ({maxMicrosteps}).")
    simulated = macro_count * macro_dt
    if not math.isfinite(simulated):
        raise RangeError("requested simulation duration is outside the supported range.")
    return {"macroStepCount": macro_count, "macroDt": macro_dt, "microStepCount": micro_count,
            "simulatedSeconds": simulated, "remainderSeconds": max(0.0, accumulated - simulated),
            "microstepPlan": plan}


def calculate_mpm_cfl_step_batch(currentVelocityBound, gravityMagnitude, oscillationAmplitude, dragRadius,
                                 dragStiffness, dragDamping, **batch_input) -> dict:
    """calculateMpmCflStepBatch, step-scheduler.ts:160-200."""
    base = dict(batch_input, velocityBound=currentVelocityBound)
    preview = calculate_mpm_step_batch(**base)
    velocity = calculate_mpm_cfl_velocity_bound(currentVelocityBound, preview["simulatedSeconds"], gravityMagnitude,
                                                oscillationAmplitude, dragRadius, dragStiffness, dragDamping)
    batch = calculate_mpm_step_batch(**dict(base, velocityBound=velocity))
    gpu_micro = fround(batch["microstepPlan"]["microDt"])
    gpu_damping = fround(dragDamping)
    if batch["macroStepCount"] > 0 and dragRadius > 0 and (
            not math.isfinite(gpu_micro) or gpu_micro <= 0 or not math.isfinite(gpu_damping)
            or gpu_micro * gpu_damping > 1):
        raise RangeError("CFL microDt is too large for the explicit drag damping update to remain dissipative.")
    return {"batch": batch, "velocityBound": velocity}


def mean_sinusoidal_acceleration(startSeconds, durationSeconds, amplitude,
                                 frequencyHz=HORIZONTAL_OSCILLATION_FREQUENCY_HZ) -> float:
    """meanSinusoidalAcceleration, src/lib/mpm/kernels/oscillation.ts:7-34."""
    if (not math.isfinite(startSeconds) or not math.isfinite(durationSeconds) or durationSeconds < 0
            or not math.isfinite(amplitude) or not math.isfinite(frequencyHz) or frequencyHz < 0):
        raise RangeError("Oscillation inputs must be finite, with non-negative duration and frequency.")
    if amplitude == 0 or frequencyHz == 0:
        return 0.0
    w = 2 * math.pi * frequencyHz
    half = (w * durationSeconds) / 2
    sinc = 1.0 if half == 0 else math.sin(half) / half
    return amplitude * math.sin(w * (startSeconds + durationSeconds / 2)) * sinc
