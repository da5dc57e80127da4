"""CFL microstep policy: src/lib/mpm/kernels/cfl.ts of 7korobi/powder-play.

`calculate_mpm_cfl_safe_dt` (cfl.ts:121-147), the overflow-safe safe-dt
(:64-114), `calculate_mpm_cfl_microsteps` with its float32 microDt guard
(:151-232) and `calculate_mpm_cfl_velocity_limit` (:234-273) with the float32
round-down/round-up helpers (:275-315).  Arithmetic is IEEE double as in
JavaScript; Math.fround is numpy float32 rounding.
"""
from __future__ import annotations

import math
import struct

from .errors import RangeError
from .layout import fround, _is_safe_integer

DEFAULT_MPM_COURANT_LIMIT = 0.3
MAX_FLOAT32 = 3.4028234663852886e38


def _pow2(e: int) -> float:
    return math.ldexp(1.0, e)


def _decompose_positive(value: float):
    """decomposePositive, cfl.ts:34-50."""
    exponent = math.floor(math.log2(value)) + 1
    exponent = min(1024, max(-1073, exponent))
    mantissa = (value / _pow2(exponent - 1)) / 2
    while mantissa >= 1:
        mantissa *= 0.5
        exponent += 1
    while mantissa < 0.5:
        mantissa *= 2
        exponent -= 1
    return mantissa, exponent


def _scale_by_power_of_two(mantissa: float, exponent: int) -> float:
    """scaleByPowerOfTwo, cfl.ts:52-63."""
    if exponent > 1024:
        return math.inf
    if exponent < -1074:
        return 0.0
    if exponent == 1024:
        return (mantissa * _pow2(1023)) * 2
    return mantissa * _pow2(exponent)


def _calculate_safe_dt(courant: float, cell: float, wave: float, velocity: float) -> float:
    """calculateSafeDt, cfl.ts:64-114."""
    speed = wave + velocity
    if speed == 0:
        return math.inf
    distance = courant * cell
    if math.isfinite(speed) and math.isfinite(distance) and distance > 0:
        safe = distance / speed
        if safe > 0:
            return safe
    speed_scale = max(wave, velocity)
    scaled_speed = wave / speed_scale + velocity / speed_scale
    lm, le = _decompose_positive(courant)
    cm, ce = _decompose_positive(cell)
    sm, se = _decompose_positive(speed_scale)
    qm, qe = _decompose_positive(scaled_speed)
    mantissa = (lm * cm) / (sm * qm)
    exponent = le + ce - se - qe
    while mantissa >= 1:
        mantissa *= 0.5
        exponent += 1
    while mantissa < 0.5:
        mantissa *= 2
        exponent -= 1
    return _scale_by_power_of_two(mantissa, exponent)


def _num(value) -> float:
    if isinstance(value, bool) or not isinstance(value, (int, float)):
        return math.nan
    return float(value)


def calculate_mpm_cfl_safe_dt(cellSize, waveSpeedBound, velocityBound, courantLimit=DEFAULT_MPM_COURANT_LIMIT):
    """calculateMpmCflSafeDt, cfl.ts:121-147."""
    cell, wave, vel, courant = map(_num, (cellSize, waveSpeedBound, velocityBound, courantLimit))
    if not math.isfinite(cell) or cell <= 0:
        raise RangeError("cellSize must be positive and finite.")
    if not math.isfinite(wave) or wave < 0:
        raise RangeError("waveSpeedBound must be finite and non-negative.")
    if not math.isfinite(vel) or vel < 0:
        raise RangeError("velocityBound must be finite and non-negative.")
    if not math.isfinite(courant) or courant <= 0:
        raise RangeError("courantLimit must be positive and finite.")
    safe = _calculate_safe_dt(courant, cell, wave, vel)
    if math.isnan(safe) or safe <= 0:
        raise RangeError("safeDt is outside the positive representable numeric range.")
    return safe


_PLAN_CACHE: dict = {}
_PLAN_CACHE_LIMIT = 4096


def calculate_mpm_cfl_microsteps(macroDt, cellSize, waveSpeedBound, velocityBound, maxMicrosteps,
                                 minimumStepCount=1, courantLimit=DEFAULT_MPM_COURANT_LIMIT) -> dict:
    """calculateMpmCflMicrosteps, cfl.ts:151-232 -> {stepCount, microDt, safeDt}.

    A pure function of its arguments; the adaptive stepping loop asks for the
    same plan several times per macrostep (the caller's plan, then the
    solver's certification of it), so successful plans are remembered by the
    arguments' types and values (errors are raised afresh every time)."""
    args = (macroDt, cellSize, waveSpeedBound, velocityBound, maxMicrosteps, minimumStepCount, courantLimit)
    try:
        key = tuple((type(a), a) for a in args)
        plan = _PLAN_CACHE.get(key)
    except TypeError:  # an unhashable argument: no caching
        key, plan = None, None
    if plan is None:
        plan = _calculate_mpm_cfl_microsteps(*args)
        if key is not None:
            if len(_PLAN_CACHE) >= _PLAN_CACHE_LIMIT:
                _PLAN_CACHE.clear()
            _PLAN_CACHE[key] = plan
    return dict(plan)


def _calculate_mpm_cfl_microsteps(macroDt, cellSize, waveSpeedBound, velocityBound, maxMicrosteps,
                                  minimumStepCount=1, courantLimit=DEFAULT_MPM_COURANT_LIMIT) -> dict:
    if courantLimit is None:
        courantLimit = DEFAULT_MPM_COURANT_LIMIT
    if minimumStepCount is None:
        minimumStepCount = 1
    macro = _num(macroDt)
    if not math.isfinite(macro) or macro <= 0:
        raise RangeError("macroDt must be positive and finite.")
    if not _is_safe_integer(maxMicrosteps) or maxMicrosteps < 1:
        raise RangeError("maxMicrosteps must be a positive safe integer.")
    if not _is_safe_integer(minimumStepCount) or minimumStepCount < 1:
        raise RangeError("minimumStepCount must be a positive safe integer.")
    max_steps = int(maxMicrosteps)
    safe = calculate_mpm_cfl_safe_dt(cellSize, waveSpeedBound, velocityBound, courantLimit)
    step_count = max(int(minimumStepCount), math.ceil(macro / safe) if math.isfinite(macro / safe) else 0)
    if macro / safe == math.inf:
        step_count = math.inf
    if step_count > max_steps:
        raise RangeError(f"required microstep count ({_fmt(step_count)}) exceeds maxMicrosteps ({max_steps}).")
    micro = macro / step_count
    gpu_micro = fround(micro)
    if not math.isfinite(gpu_micro):
        minimum_f32 = math.ceil(macro / MAX_FLOAT32)
        if not _is_safe_integer(minimum_f32) or minimum_f32 > max_steps:
            raise RangeError(
                f"required float32 microstep count ({_fmt(minimum_f32)}) exceeds maxMicrosteps ({max_steps}).")
        step_count = max(step_count, minimum_f32)
        micro = macro / step_count
        gpu_micro = fround(micro)
    while micro > safe or gpu_micro > safe:
        if gpu_micro == 0:
            raise RangeError("microDt is too small to represent as a positive float32 value.")
        step_count += 1
        if step_count > max_steps:
            raise RangeError(f"required microstep count ({step_count}) exceeds maxMicrosteps ({max_steps}).")
        micro = macro / step_count
        gpu_micro = fround(micro)
    if gpu_micro <= 0:
        raise RangeError("microDt is too small to represent as a positive float32 value.")
    if not math.isfinite(gpu_micro):
        raise RangeError("microDt cannot be represented as a finite float32 value.")
    return {"stepCount": int(step_count), "microDt": micro, "safeDt": safe}


def _fmt(value) -> str:
    if value == math.inf:
        return "Infinity"
    return str(int(value))


def _f32_bits(value: float) -> int:
    return struct.unpack("<I", struct.pack("<f", value))[0]


def _bits_f32(bits: int) -> float:
    return struct.unpack("<f", struct.pack("<I", bits & 0xFFFFFFFF))[0]


def round_down_float32(value: float) -> float:
    """roundDownFloat32, cfl.ts:275-295."""
    if not math.isfinite(value) or value < 0:
        raise RangeError("CFL velocity limits must be finite and non-negative.")
    if value == 0:
        return 0.0
    rounded = fround(value)
    if not math.isfinite(rounded):
        raise RangeError("CFL velocity limit cannot be represented as a finite float32 value.")
    if rounded > value:
        rounded = _bits_f32(_f32_bits(rounded) - 1)
    return rounded


def round_up_float32(value: float) -> float:
    """roundUpFloat32, cfl.ts:297-315."""
    if not math.isfinite(value) or value < 0:
        raise RangeError("CFL wave-speed bounds must be finite and non-negative.")
    if value == 0:
        return 0.0
    rounded = fround(value)
    if not math.isfinite(rounded):
        raise RangeError("CFL wave-speed bound cannot be represented as a finite float32 value.")
    if rounded < value:
        rounded = _bits_f32(_f32_bits(rounded) + 1)
    return rounded


_LIMIT_CACHE: dict = {}


def calculate_mpm_cfl_velocity_limit(cellSize, waveSpeedBound, microDt, courantLimit=DEFAULT_MPM_COURANT_LIMIT):
    """calculateMpmCflVelocityLimit, cfl.ts:234-273.  A pure function of its
    arguments, remembered like the microstep plans (the solver certifies
    every submitted plan with it)."""
    args = (cellSize, waveSpeedBound, microDt, courantLimit)
    try:
        key = tuple((type(a), a) for a in args)
        limit = _LIMIT_CACHE.get(key)
    except TypeError:  # an unhashable argument: no caching
        key, limit = None, None
    if limit is None:
        limit = _calculate_mpm_cfl_velocity_limit(*args)
        if key is not None:
            if len(_LIMIT_CACHE) >= _PLAN_CACHE_LIMIT:
                _LIMIT_CACHE.clear()
            _LIMIT_CACHE[key] = limit
    return limit


def _calculate_mpm_cfl_velocity_limit(cellSize, waveSpeedBound, microDt, courantLimit=DEFAULT_MPM_COURANT_LIMIT):
    if courantLimit is None:
        courantLimit = DEFAULT_MPM_COURANT_LIMIT
    cell, wave, micro, courant = map(_num, (cellSize, waveSpeedBound, microDt, courantLimit))
    if not math.isfinite(cell) or cell <= 0:
        raise RangeError("cellSize must be positive and finite.")
    if not math.isfinite(wave) or wave < 0:
        raise RangeError("waveSpeedBound must be finite and non-negative.")
    if not math.isfinite(micro) or micro <= 0:
        raise RangeError("microDt must be positive and finite.")
    if not math.isfinite(courant) or courant <= 0:
        raise RangeError("courantLimit must be positive and finite.")
    gpu_cell = round_down_float32(cell)
    gpu_wave = round_up_float32(wave)
    gpu_micro = fround(micro)
    if gpu_cell <= 0 or not math.isfinite(gpu_micro) or gpu_micro <= 0:
        raise RangeError("CFL inputs must be representable as positive float32 values.")
    distance = courant * gpu_cell
    max_speed = distance / gpu_micro
    limit = max_speed - gpu_wave
    if not math.isfinite(distance) or distance <= 0 or not math.isfinite(max_speed) or not math.isfinite(limit) or limit < 0:
        raise RangeError("microDt leaves no finite non-negative CFL velocity allowance.")
    return round_down_float32(limit)
