"""Error types of the host API, mirroring the reference's JavaScript errors.

`RangeError` stands for the reference's RangeError (Python's TypeError is used
where the reference throws TypeError).  `MpmMlsGpuNumericalError` restates the
status decoding of src/lib/mpm/kernels/solver.ts:146-206 so that messages and
recoverability (isRecoverableCflError, :296-312) match.
"""
from __future__ import annotations

import math
import struct

ERROR_DEFORMATION = 2
ERROR_DEFORMATION_SUBSTEP_LIMIT = 32
ERROR_CFL_BOUND = 16384
ERROR_FIXED_POINT_RANGE = 65536
MAX_U32 = 0xFFFFFFFF

_FLAG_DETAILS = (
    (1, "invalid particle stencil or linked-list state"),
    (2, "non-positive trial deformation determinant"),
    (4, "P2G validation failed"),
    (8, "non-finite grid state"),
    (16, "non-finite G2P particle state"),
    (32, "deformation update exceeded the adaptive substep limit"),
    (64, "non-positive projected deformation determinant"),
    (128, "invalid P2G material parameters"),
    (256, "non-finite particle stress or momentum"),
    (1024, "non-finite P2G node accumulation"),
    (2048, "non-finite P2G node output"),
    (4096, "invalid triangle contact field or reaction"),
    (8192, "invalid bonded triangle state"),
    (16384, "particle exceeded the enforced CFL wave-speed or velocity bound"),
    (32768, "invalid persistent solid-fracture bond state"),
    (65536, "experimental fixed-point P2G contribution or accumulator overflow"),
    (1 << 20, "a grid barrier wait of the substep kernel ran out (launch abandoned; particle state undefined)"),
)


class RangeError(ValueError):
    """The reference's RangeError."""


class MpmNativeError(RuntimeError):
    """A CUDA or state failure reported by the native library."""


def _js_number(value: float) -> str:
    if value != value:
        return "NaN"
    if value == math.inf:
        return "Infinity"
    if value == -math.inf:
        return "-Infinity"
    if value == int(value) and abs(value) < 1e21:
        return str(int(value))
    return repr(value)


def _f32(word: int) -> float:
    return struct.unpack("<f", struct.pack("<I", word & 0xFFFFFFFF))[0]


class MpmMlsGpuNumericalError(Exception):
    """MpmMlsGpuNumericalError, src/lib/mpm/kernels/solver.ts:146-206."""

    def __init__(self, flags, particle_index=None, diagnostics=None, particle_state=None,
                 projected_deformation=None, cfl_details=None, completed_microsteps=None,
                 measured_maximum_speed=None):
        self.flags = flags
        self.particle_index = particle_index
        self.diagnostics = diagnostics
        self.particle_state = particle_state
        self.projected_deformation = projected_deformation
        self.cfl_details = cfl_details
        self.completed_microsteps = completed_microsteps
        self.measured_maximum_speed = measured_maximum_speed
        message = "; ".join(text for flag, text in _FLAG_DETAILS if flags & flag)
        particle_context = "" if particle_index is None else f" at particle {particle_index}"
        diagnostic_context = "" if diagnostics is None else (
            f" (det={_js_number(diagnostics['determinant'])}, deformation increment="
            f"{_js_number(diagnostics['deformationIncrement'])}, preceding det="
            f"{_js_number(diagnostics['precedingDeterminant'])})")
        projection_context = "" if projected_deformation is None else (
            " (projected F=({},{},{},{}))".format(*(_js_number(projected_deformation[k])
                                                    for k in ("m00", "m01", "m10", "m11"))))
        cfl_context = "" if cfl_details is None else (
            f" (particle speed={_js_number(cfl_details['particleSpeed'])}, wave speed="
            f"{_js_number(cfl_details['waveSpeed'])}, limits=({_js_number(cfl_details['velocityLimit'])}, "
            f"{_js_number(cfl_details['waveSpeedLimit'])}))")
        body = message or f"status 0x{flags:x}"
        super().__init__(
            f"GPU MLS-MPM rejected a step ({body}{particle_context}{diagnostic_context}"
            f"{projection_context}{cfl_context}); all particles were rolled back to the last valid state.")


def decode_numerical_error(status, completed_microsteps=None, measured_maximum_speed=None):
    """decodeNumericalError, src/lib/mpm/kernels/solver.ts:232-284."""
    if status[0] == 0:
        return None
    particle_index = None if status[1] == MAX_U32 else int(status[1])
    values = [_f32(status[k]) for k in (2, 3, 4, 5)]
    diagnostics = None if status[6] != 1 else {
        "determinant": values[0], "deformationIncrement": values[1], "precedingDeterminant": values[2]}
    projected = None if status[6] != 2 else {
        "m00": values[0], "m01": values[1], "m10": values[2], "m11": values[3]}
    cfl = None if status[6] != 3 else {
        "particleSpeed": values[0], "waveSpeed": values[1], "velocityLimit": values[2], "waveSpeedLimit": values[3]}
    return MpmMlsGpuNumericalError(int(status[0]), particle_index, diagnostics, None, projected, cfl,
                                   completed_microsteps, measured_maximum_speed)


def is_recoverable_cfl_error(error: MpmMlsGpuNumericalError) -> bool:
    """isRecoverableCflError, src/lib/mpm/kernels/solver.ts:296-312."""
    if error.flags == ERROR_CFL_BOUND:
        d = error.cfl_details
        return d is not None and all(math.isfinite(d[k]) for k in (
            "particleSpeed", "waveSpeed", "velocityLimit", "waveSpeedLimit"))
    return (error.flags in (ERROR_DEFORMATION, ERROR_DEFORMATION_SUBSTEP_LIMIT)
            and error.measured_maximum_speed is not None and math.isfinite(error.measured_maximum_speed))


_SURFACE_FLAG_DETAILS = (
    (1, "invalid free-surface bucket state"),
    (2, "invalid particle area or deformation determinant"),
    (4, "non-finite free-surface occupancy accumulation"),
)


class MpmMlsGpuSurfaceError(Exception):
    """MpmMlsGpuSurfaceError, src/lib/mpm/kernels/solver.ts:208-224."""

    def __init__(self, flags):
        self.flags = flags
        message = "; ".join(text for flag, text in _SURFACE_FLAG_DETAILS if flags & flag)
        body = message or f"status 0x{flags:x}"
        super().__init__(f"GPU free-surface occupancy generation failed ({body}); particle state was not modified.")


def decode_surface_error(status):
    """decodeSurfaceError, src/lib/mpm/kernels/solver.ts:286-294: status word 7."""
    flags = int(status[7])
    return None if flags == 0 else MpmMlsGpuSurfaceError(flags)
