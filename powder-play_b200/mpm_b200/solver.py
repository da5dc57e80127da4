"""The GPU solver host API: a drop-in for `MpmMlsGpuSolver`.

Restates the host control flow of src/lib/mpm/kernels/solver.ts
(7korobi/powder-play): the factories `createMpmMlsGpuSolver` /
`createExperimentalMpmMlsAtomicGpuSolver` (:390-469), CFL-bound certification
`validateCflBounds` (:471-528), `stepBatch` (:1407-1599), `stepCflBatch`
(:1601-1722), the adaptive retry/rollback loop `stepCflBatchAdaptive`
(:1724-2021), `measureMaximumParticleSpeed` (:2388-2512),
`checkNumericalStatus` (:2514-2570) and `readParticles` (:2594-).  The device
work runs in libmpm_b200.so through the C ABI of include/mpm_b200.h; the
reference's Promises become blocking calls.
"""
from __future__ import annotations

import ctypes
import math
import time

import numpy as np

from . import _lib
from .cfl import calculate_mpm_cfl_microsteps, calculate_mpm_cfl_safe_dt, calculate_mpm_cfl_velocity_limit
from .cfl_bounds import derive_mpm_mls_gpu_cfl_bounds
from .errors import (MpmMlsGpuNumericalError, MpmNativeError, RangeError, decode_numerical_error,
                     decode_surface_error, is_recoverable_cfl_error)
from .layout import (PARTICLE_FLOATS, ValidatedInput, fround, pack_step_parameters, particles_from_dicts,
                     unpack_particles, validate_mpm_mls_gpu_input, _is_safe_integer)

CFL_RECOVERY_BOUND_SAFETY_FACTOR = 1.25
MPM_MLS_GPU_DRAG_STIFFNESS = 20.0
MPM_MLS_GPU_DRAG_DAMPING = 8.0
EPSILON = 2.220446049250313e-16
MIN_VALUE = 5e-324
DEFAULT_FIXED_POINT_SHIFT = 24


def _interaction_float32(value, name: str) -> float:
    """finiteInteractionFloat32, solver.ts:3268-3277."""
    if isinstance(value, bool) or not isinstance(value, (int, float)) or not math.isfinite(value):
        raise TypeError(f"{name} must be a finite number.")
    result = fround(value)
    if not math.isfinite(result):
        raise RangeError(f"{name} is outside the supported float32 range.")
    return result


def _is_capacity_error(error) -> bool:
    import re
    return isinstance(error, RangeError) and re.search(
        r"exceeds maxMicrosteps|microDt is too small to represent", str(error)) is not None


def _check(rc: int, what: str):
    if rc == _lib.MPM_OK:
        return
    message = _lib.last_error()
    if rc == _lib.MPM_ERR_INVALID_ARGUMENT:
        raise RangeError(message or f"{what}: invalid argument")
    raise MpmNativeError(f"{what}: {message}")


def validate_cfl_bounds(bounds, state: ValidatedInput, derived):
    """validateCflBounds, solver.ts:471-528."""
    if bounds is None:
        return derived
    if not isinstance(bounds, dict):
        raise RangeError("cflBounds must be an object of valid speed bounds.")
    if derived is None:
        raise RangeError("this solver configuration has no derived CFL bounds for its constitutive material.")
    wave, vel = bounds.get("waveSpeedBound"), bounds.get("velocityBound")
    if not isinstance(wave, (int, float)) or not math.isfinite(wave) or wave < 0:
        raise RangeError("cflBounds.waveSpeedBound must be finite and non-negative.")
    if not isinstance(vel, (int, float)) or not math.isfinite(vel) or vel < 0:
        raise RangeError("cflBounds.velocityBound must be finite and non-negative.")
    courant = bounds.get("courantLimit")
    if courant is not None and (not math.isfinite(courant) or courant <= 0):
        raise RangeError("cflBounds.courantLimit must be positive and finite.")
    if wave < derived["waveSpeedBound"]:
        raise RangeError("cflBounds.waveSpeedBound must not be lower than the material-derived initial bound.")
    if vel < derived["velocityBound"]:
        raise RangeError("cflBounds.velocityBound must not be lower than the configured initial-state bound.")
    speeds = np.hypot(state.packed_particles[:, 2].astype(np.float64), state.packed_particles[:, 3].astype(np.float64))
    over = np.flatnonzero(speeds > vel)
    if over.size:
        raise RangeError(f"initial velocity at particle {int(over[0])} exceeds cflBounds.velocityBound.")
    out = {"waveSpeedBound": float(wave), "velocityBound": float(vel)}
    if courant is not None:
        out["courantLimit"] = float(courant)
    return out


def native_config(state: ValidatedInput, atomic_p2g: bool, fixed_point_shift: int, device: int):
    """The mpm_config of a validated input (the float32 values that
    validateMpmMlsGpuInput, layout.ts:122-607, derives)."""
    cfg = state.config
    c = _lib.MpmConfig()
    c.cells_x, c.cells_y = cfg["grid"]["cellsX"], cfg["grid"]["cellsY"]
    c.cell_size = state.cell_size_f32
    c.particle_mass = state.particle_mass_f32
    c.particle_volume = state.particle_volume_f32
    c.bond_rest_length = state.bond_rest_length_f32
    c.bond_stiffness = state.bond_stiffness_f32
    c.bond_reference_dt = state.bond_reference_dt_f32 or 0.0
    c.wall_friction = state.wall_friction_f32
    c.lambda_ = state.lambda_f32
    c.mu = state.mu_f32
    c.capacity = state.particle_capacity
    c.p2g_mode = _lib.MPM_P2G_FIXED_POINT if atomic_p2g else _lib.MPM_P2G_GATHER
    c.fixed_point_shift = fixed_point_shift
    c.device = device
    return c


class MpmMlsGpuSolver:
    """MpmMlsGpuSolver, solver.ts:106-144, backed by libmpm_b200.so."""

    def __init__(self, state: ValidatedInput, cfl_bounds, atomic_p2g: bool, device: int = 0,
                 fixed_point_shift: int = DEFAULT_FIXED_POINT_SHIFT):
        self._lib = _lib.load_library()
        self._state = state
        c = native_config(state, atomic_p2g, fixed_point_shift, device)
        handle = ctypes.c_void_p()
        packed = np.ascontiguousarray(state.packed_particles, dtype=np.float32)
        ids = np.ascontiguousarray(state.packed_object_ids, dtype=np.uint32)
        starts = np.ascontiguousarray(state.bonded_body_starts, dtype=np.uint32)
        bonds = np.ascontiguousarray(state.packed_fracture_bonds, dtype=np.uint32)
        topo = np.ascontiguousarray(state.packed_fracture_bond_topology, dtype=np.uint32)
        rc = self._lib.mpm_create(ctypes.byref(c), _lib.ptr(packed), _lib.ptr(ids), state.particle_count,
                                  _lib.ptr(starts), len(starts), _lib.ptr(bonds), state.fracture_bond_count,
                                  _lib.ptr(topo), len(topo), ctypes.byref(handle))
        if rc != _lib.MPM_OK:
            message = _lib.last_error()
            raise RuntimeError(f"Failed to initialize the GPU MLS-MPM solver: {message}")
        self._handle = handle
        self.cfl_bounds = cfl_bounds
        self.atomic_p2g = atomic_p2g
        self.fixed_point_shift = fixed_point_shift
        self._disposed = False
        # the factor a failed batch's observed speed and wave speed are raised by
        # before the retry (solver.ts:73 fixes it at 1.25); callers may study others
        self.recovery_bound_factor = CFL_RECOVERY_BOUND_SAFETY_FACTOR
        self._slot_count = state.particle_count      # particleSlotCount (allocated original indices)
        self._active_count = state.particle_count    # activeParticleCount
        self._has_removed = False
        self._object_ranges = {r["objectId"]: (r["start"], r["count"]) for r in state.object_ranges}
        self._next_object_id = max([r["objectId"] + 1 for r in state.object_ranges] + [0])
        self._cfl_speed_measurement_submitted = False
        self._cfl_state_usable = cfl_bounds is not None
        self._last_scheduled_velocity_bound = None if cfl_bounds is None else cfl_bounds["velocityBound"]
        self._latest_cfl_batch_sequence = 0
        self._latest_cfl_batch_microstep_count = 0
        self._latest_completed_cfl_measurement_sequence = 0
        self._active_drag = None
        self.device_ms_total = 0.0
        self.committed_microsteps_total = 0

    # ---------------------------------------------------------------- props --
    @property
    def particle_count(self) -> int:
        return self._active_count

    @property
    def allocated_particle_count(self) -> int:
        return self._slot_count

    @property
    def particle_capacity(self) -> int:
        return self._state.particle_capacity

    @property
    def node_count(self) -> int:
        return int(self._lib.mpm_node_count(self._handle))

    def _assert_active(self):
        if self._disposed:
            raise RuntimeError("GPU MLS-MPM solver has been disposed.")

    # ----------------------------------------------------------------- steps --
    def step(self, dt: float, gravity: dict) -> None:
        self.step_batch(1, dt, gravity)

    def step_batch(self, step_count: int, dt: float, gravity: dict, cfl_velocity_bound=None,
                   bond_reference_dt=None) -> None:
        """stepBatch, solver.ts:1407-1599."""
        self._assert_active()
        if not _is_safe_integer(step_count) or step_count < 1:
            raise RangeError("stepCount must be a positive safe integer.")
        guard = None
        if cfl_velocity_bound is not None:
            if self.cfl_bounds is None:
                raise RangeError("this solver configuration has no safely derived CFL bounds.")
            if not math.isfinite(cfl_velocity_bound) or cfl_velocity_bound < 0:
                raise RangeError("velocityBound must be finite and non-negative.")
            guard = {"waveSpeedBound": self.cfl_bounds["waveSpeedBound"], "velocityBound": cfl_velocity_bound}
        dt32, gx, gy, wave, vel, bref = pack_step_parameters(self._state, dt, gravity, guard, bond_reference_dt)
        native_guard = None
        if guard is not None:
            native_guard = _lib.MpmCflGuard(wave, vel)
        try:
            rc = self._lib.mpm_step_batch(self._handle, int(step_count), dt32, gx, gy,
                                          ctypes.byref(native_guard) if native_guard is not None else None, bref)
            _check(rc, f"Failed to encode or submit an MLS-MPM batch of {step_count} step(s).")
        except Exception:
            self._cfl_state_usable = False
            self._cfl_speed_measurement_submitted = False
            raise
        self._cfl_speed_measurement_submitted = guard is not None
        if guard is None:
            self._cfl_state_usable = False

    def step_cfl_batch(self, macro_step_count, macro_dt, microstep_plan, velocity_bound, max_microsteps, gravity,
                       bond_reference_dt=None) -> None:
        """stepCflBatch, solver.ts:1601-1722."""
        self._assert_active()
        if self.cfl_bounds is None:
            raise RangeError("CFL stepping requires a material-derived wave-speed bound; this solver configuration "
                             "has no safely derived CFL bounds.")
        if not self._cfl_state_usable:
            raise RuntimeError("a direct non-CFL GPU step or a failed CFL measurement invalidated the tracked "
                               "velocity bound; recreate the solver before CFL stepping.")
        if self._cfl_speed_measurement_submitted:
            raise RuntimeError("queue measureMaximumParticleSpeed() after the previous CFL batch before submitting "
                               "another one.")
        if self._last_scheduled_velocity_bound is not None and velocity_bound < self._last_scheduled_velocity_bound:
            raise RangeError("velocityBound must cover the last submitted GPU maximum-particle envelope.")
        if not _is_safe_integer(macro_step_count) or macro_step_count < 1:
            raise RangeError("macroStepCount must be a positive safe integer.")
        if not _is_safe_integer(max_microsteps) or max_microsteps < 1:
            raise RangeError("maxMicrosteps must be a positive safe integer.")
        cell = self._state.config["grid"]["cellSize"]
        b = self.cfl_bounds
        expected = calculate_mpm_cfl_microsteps(macro_dt, cell, b["waveSpeedBound"], velocity_bound, max_microsteps,
                                                courantLimit=b.get("courantLimit"))
        certified = None
        if isinstance(microstep_plan, dict) and microstep_plan.get("stepCount") == expected["stepCount"] \
                and _is_safe_integer(microstep_plan["stepCount"]):
            # the plan at the required count: the refinement with that minimum
            # is the required plan itself
            certified = expected
        elif (isinstance(microstep_plan, dict) and _is_safe_integer(microstep_plan.get("stepCount"))
                and microstep_plan["stepCount"] >= expected["stepCount"]):
            certified = calculate_mpm_cfl_microsteps(macro_dt, cell, b["waveSpeedBound"], velocity_bound,
                                                     max_microsteps, minimumStepCount=microstep_plan["stepCount"],
                                                     courantLimit=b.get("courantLimit"))
        if (certified is None or microstep_plan["stepCount"] != certified["stepCount"]
                or microstep_plan["microDt"] != certified["microDt"] or microstep_plan["safeDt"] != certified["safeDt"]):
            raise RangeError("microstepPlan does not match this solver configuration or is not a certified CFL "
                             "refinement.")
        micro_count = macro_step_count * certified["stepCount"]
        if not _is_safe_integer(micro_count) or micro_count > max_microsteps:
            raise RangeError(f"requested microstep count ({micro_count}) exceeds maxMicrosteps ({max_microsteps}).")
        represented = certified["microDt"] * certified["stepCount"]
        tolerance = max(macro_dt, MIN_VALUE) * EPSILON * 4
        if abs(represented - macro_dt) > tolerance:
            raise RangeError("microstepPlan does not preserve the requested macro dt.")
        gpu_micro = fround(certified["microDt"])
        if self._active_drag is not None and (not math.isfinite(gpu_micro) or gpu_micro <= 0
                                              or gpu_micro * MPM_MLS_GPU_DRAG_DAMPING > 1):
            raise RangeError("CFL microDt is too large for the explicit drag damping update to remain dissipative.")
        limit = calculate_mpm_cfl_velocity_limit(cell, b["waveSpeedBound"], certified["microDt"], b.get("courantLimit"))
        if limit < velocity_bound:
            raise RangeError("float32 microDt does not preserve the planned CFL velocity bound; increase the "
                             "microstep count.")
        sb = self._state.bond_reference_dt_f32
        self.step_batch(micro_count, certified["microDt"], gravity, limit,
                        bond_reference_dt if bond_reference_dt is not None else (sb if sb is not None else macro_dt))
        self._latest_cfl_batch_sequence += 1
        self._latest_cfl_batch_microstep_count = micro_count
        self._last_scheduled_velocity_bound = velocity_bound

    def step_cfl_batch_adaptive(self, macro_step_count, macro_dt, microstep_plan, velocity_bound, max_microsteps,
                                gravity, gravity_for_duration=None) -> dict:
        """stepCflBatchAdaptive, solver.ts:1724-2021 (the retry/rollback loop)."""
        if self.cfl_bounds is None:
            raise RangeError("CFL stepping requires a material-derived wave-speed bound; this solver configuration "
                             "has no safely derived CFL bounds.")
        if not _is_safe_integer(macro_step_count) or macro_step_count < 1:
            raise RangeError("macroStepCount must be a positive safe integer.")
        if not math.isfinite(macro_dt) or macro_dt <= 0:
            raise RangeError("macroDt must be positive and finite.")
        total = macro_step_count * macro_dt
        if not math.isfinite(total):
            raise RangeError("CFL batch duration is outside the supported range.")
        bref = self._state.bond_reference_dt_f32 if self._state.bond_reference_dt_f32 is not None else macro_dt
        remaining = total
        attempt_macro_count, attempt_macro_dt = macro_step_count, macro_dt
        attempt_plan, attempt_velocity = microstep_plan, velocity_bound
        consumed = retry_count = submissions = 0
        retry_ms = readback_ms = 0.0
        tolerance = max(total, MIN_VALUE) * EPSILON * 4
        cell = self._state.config["grid"]["cellSize"]

        def result(measurement, recommended=None):
            return dict(measurement,
                        recommendedVelocityBound=measurement["maximumSpeed"] if recommended is None else recommended,
                        attemptedMicroStepCount=consumed, retryCount=retry_count,
                        retrySubmissionMilliseconds=retry_ms, readbackMilliseconds=readback_ms,
                        simulatedDuration=max(0.0, total - remaining), remainingDuration=remaining)

        while True:
            attempt_micro = attempt_macro_count * attempt_plan["stepCount"]
            attempt_duration = attempt_macro_count * attempt_macro_dt
            budget = max_microsteps - consumed
            if (not _is_safe_integer(attempt_micro) or attempt_micro < 1 or not math.isfinite(attempt_duration)
                    or attempt_duration <= 0 or attempt_micro > budget):
                raise RangeError(f"adaptive CFL retry requires {attempt_micro} microsteps with {budget} remaining.")
            started = time.perf_counter()
            attempt_gravity = gravity if gravity_for_duration is None else gravity_for_duration(
                total - remaining, attempt_duration)
            self.step_cfl_batch(attempt_macro_count, attempt_macro_dt, attempt_plan, attempt_velocity, budget,
                                attempt_gravity, bref)
            if submissions > 0:
                retry_ms += (time.perf_counter() - started) * 1e3
            submissions += 1
            read_started = time.perf_counter()
            try:
                measurement = self.measure_maximum_particle_speed()
            except MpmMlsGpuNumericalError as error:
                readback_ms += (time.perf_counter() - read_started) * 1e3
                if not is_recoverable_cfl_error(error):
                    raise
                completed = error.completed_microsteps
                if completed is None or completed < 0 or completed >= attempt_micro:
                    raise RuntimeError(f"Adaptive CFL recovery could not determine completed microsteps: {error}") from error
                completed_duration = completed * attempt_plan["microDt"]
                if not math.isfinite(completed_duration) or completed_duration >= remaining:
                    raise RuntimeError(f"Adaptive CFL recovery received invalid simulation progress: {error}") from error
                remaining -= completed_duration
                consumed += attempt_micro
                self.committed_microsteps_total += completed
                observed = max(error.measured_maximum_speed or 0.0,
                               (error.cfl_details or {}).get("particleSpeed", 0.0))
                retry_velocity = max(attempt_velocity, self._last_scheduled_velocity_bound or 0.0,
                                     observed * self.recovery_bound_factor)
                if not math.isfinite(retry_velocity):
                    raise RuntimeError(f"Adaptive CFL recovery stopped after {retry_count} retry attempt(s) "
                                       f"(non-finite velocity bound); last GPU error: {error}") from error
                self._last_scheduled_velocity_bound = retry_velocity
                if error.cfl_details is not None:
                    retry_wave = error.cfl_details["waveSpeed"] * self.recovery_bound_factor
                    if not math.isfinite(retry_wave):
                        raise RuntimeError(f"Adaptive CFL recovery stopped after {retry_count} retry attempt(s) "
                                           f"(non-finite wave-speed bound); last GPU error: {error}") from error
                    self.cfl_bounds = dict(self.cfl_bounds,
                                           waveSpeedBound=max(self.cfl_bounds["waveSpeedBound"], retry_wave))
                retry_budget = max_microsteps - consumed
                if retry_budget < 2:
                    self._clear_status()
                    self._cfl_state_usable = True
                    return result({"maximumSpeed": observed, "sequence": self._latest_cfl_batch_sequence},
                                  retry_velocity)
                failed_interval = min(remaining, attempt_plan["microDt"])
                try:
                    attempt_plan = calculate_mpm_cfl_microsteps(
                        failed_interval, cell, self.cfl_bounds["waveSpeedBound"], retry_velocity, retry_budget,
                        minimumStepCount=2, courantLimit=self.cfl_bounds.get("courantLimit"))
                except RangeError as cause:
                    if not _is_capacity_error(cause):
                        raise RuntimeError(f"Adaptive CFL recovery could not schedule a finer step ({cause}; "
                                           f"retry={retry_count + 1}): {error}") from cause
                    self._clear_status()
                    self._cfl_state_usable = True
                    return result({"maximumSpeed": observed, "sequence": self._latest_cfl_batch_sequence},
                                  retry_velocity)
                self._clear_status()
                self._cfl_state_usable = True
                attempt_macro_count, attempt_macro_dt = 1, failed_interval
                attempt_velocity = retry_velocity
                retry_count += 1
                continue
            readback_ms += (time.perf_counter() - read_started) * 1e3
            consumed += attempt_micro
            self.committed_microsteps_total += attempt_micro
            remaining = max(0.0, remaining - attempt_duration)
            if remaining <= tolerance:
                remaining = 0.0
                return result(measurement, max(attempt_velocity, measurement["maximumSpeed"]) if retry_count > 0
                              else measurement["maximumSpeed"])
            continuation_budget = max_microsteps - consumed
            if continuation_budget < 2:
                return result(measurement, max(attempt_velocity, measurement["maximumSpeed"]))
            attempt_velocity = max(attempt_velocity, measurement["maximumSpeed"])
            safe = calculate_mpm_cfl_safe_dt(cell, self.cfl_bounds["waveSpeedBound"], attempt_velocity,
                                             self.cfl_bounds.get("courantLimit", 0.3))
            max_step = min(attempt_plan["microDt"], safe)
            if not math.isfinite(max_step) or max_step <= 0:
                raise RangeError(f"Adaptive CFL recovery produced an invalid continuation timestep ({max_step}).")
            required = math.ceil(remaining / max_step)
            continuation = remaining
            minimum = max(1, required)
            if required >= continuation_budget:
                continuation = min(remaining, max_step * (continuation_budget - 1) * (1 - EPSILON * 8))
                minimum = max(1, math.ceil(continuation / max_step))
            if not math.isfinite(continuation) or continuation <= 0:
                return result(measurement, max(attempt_velocity, measurement["maximumSpeed"]))
            attempt_plan = calculate_mpm_cfl_microsteps(continuation, cell, self.cfl_bounds["waveSpeedBound"],
                                                        attempt_velocity, continuation_budget,
                                                        minimumStepCount=minimum,
                                                        courantLimit=self.cfl_bounds.get("courantLimit"))
            attempt_macro_count, attempt_macro_dt = 1, continuation

    # -------------------------------------------------------------- readback --
    def _read_compact(self):
        speed = ctypes.c_float()
        done = ctypes.c_uint32()
        status = np.zeros(8, dtype=np.uint32)
        _check(self._lib.mpm_read_compact(self._handle, ctypes.byref(speed), ctypes.byref(done), _lib.ptr(status)),
               "Failed to read the compact GPU CFL speed measurement.")
        return float(speed.value), int(done.value), status

    def _clear_status(self):
        _check(self._lib.mpm_clear_status(self._handle), "Failed to clear the GPU numerical status.")

    def measure_maximum_particle_speed(self) -> dict:
        """measureMaximumParticleSpeed, solver.ts:2388-2512."""
        self._assert_active()
        if not self._cfl_speed_measurement_submitted:
            raise RuntimeError("No completed CFL batch has a maximum-speed measurement to read.")
        self._cfl_speed_measurement_submitted = False
        sequence = self._latest_cfl_batch_sequence
        try:
            speed, completed, status = self._read_compact()
            self.device_ms_total += self.last_batch_device_ms()
            if completed > self._latest_cfl_batch_microstep_count:
                raise RangeError(f"GPU reported {completed} completed microsteps for a batch of "
                                 f"{self._latest_cfl_batch_microstep_count}.")
            error = decode_numerical_error(status, completed, speed)
            if error is not None:
                raise error
            surface_error = decode_surface_error(status)
            if surface_error is not None:
                raise surface_error
            if not math.isfinite(speed) or speed < 0:
                raise RangeError("GPU returned an invalid maximum-particle-speed scalar.")
            if sequence >= self._latest_completed_cfl_measurement_sequence:
                self._latest_completed_cfl_measurement_sequence = sequence
                if sequence == self._latest_cfl_batch_sequence:
                    self._last_scheduled_velocity_bound = speed
            return {"maximumSpeed": speed, "sequence": sequence}
        except Exception:
            self._cfl_state_usable = False
            raise

    def last_batch_device_ms(self) -> float:
        """Device time of the last submitted batch (CUDA events on the solver's stream)."""
        out = ctypes.c_double()
        _check(self._lib.mpm_last_batch_device_ms(self._handle, ctypes.byref(out)), "batch timing failed")
        return float(out.value)

    def profile_substeps(self, step_count: int, dt: float, gravity: dict, velocity_limit=None) -> dict:
        """Runs real substeps kernel by kernel with CUDA events between them:
        {kernel name: (milliseconds, launches)}."""
        slots = int(self._lib.mpm_profile_kernel_slots())
        ms = np.zeros(slots, dtype=np.float64)
        launches = np.zeros(slots, dtype=np.uint32)
        guard = None
        if velocity_limit is not None:
            guard = _lib.MpmCflGuard(fround(self.cfl_bounds["waveSpeedBound"]), fround(velocity_limit))
        _check(self._lib.mpm_profile_substeps(self._handle, step_count, fround(dt), fround(gravity["x"]),
                                              fround(gravity["y"]), ctypes.byref(guard) if guard else None,
                                              _lib.ptr(ms), _lib.ptr(launches)), "profiled substeps failed")
        out = {}
        for k in range(slots):
            if launches[k]:
                out[self._lib.mpm_profile_kernel_name(k).decode()] = (float(ms[k]), int(launches[k]))
        return out

    def count_active_nodes(self):
        counts = np.zeros(3, dtype=np.uint32)
        _check(self._lib.mpm_count_active_nodes(self._handle, _lib.ptr(counts)), "active node count failed")
        return tuple(int(c) for c in counts)

    def check_numerical_status(self) -> None:
        """checkNumericalStatus, solver.ts:2514-2570."""
        self._assert_active()
        _, _, status = self._read_compact()
        error = decode_numerical_error(status)
        if error is not None:
            raise error
        surface_error = decode_surface_error(status)
        if surface_error is not None:
            raise surface_error

    def read_status_words(self) -> np.ndarray:
        self._assert_active()
        return self._read_compact()[2]

    def read_particles_packed(self, particle_indices=None):
        """The packed 20-word records and object ids (readParticles without decoding)."""
        self._assert_active()
        if particle_indices is None:
            count = self._slot_count
            idx = None
        else:
            if not isinstance(particle_indices, (list, tuple, np.ndarray)):
                raise TypeError("particleIndices must be an array of active particle indices.")
            idx = np.ascontiguousarray(particle_indices, dtype=np.int64)
            if idx.size and (idx.min() < 0 or idx.max() >= self._slot_count):
                raise RangeError("particleIndices must identify active GPU particles.")
            idx = idx.astype(np.uint32)
            count = idx.size
        packed = np.zeros((count, PARTICLE_FLOATS), dtype=np.float32)
        ids = np.zeros(count, dtype=np.uint32)
        _check(self._lib.mpm_read_particles(self._handle, _lib.ptr(idx), count, _lib.ptr(packed), _lib.ptr(ids)),
               "Failed to read GPU MLS-MPM particles.")
        status = self._read_compact()[2]
        error = decode_numerical_error(status)
        if error is not None:
            raise error
        return packed, ids

    def read_particles(self, particle_indices=None) -> list:
        """readParticles, solver.ts:2594- (decoded like unpackParticles :3148-3226)."""
        packed, ids = self.read_particles_packed(particle_indices)
        return unpack_particles(packed, ids)

    def write_particles_packed(self, packed: np.ndarray) -> None:
        self._assert_active()
        packed = np.ascontiguousarray(packed, dtype=np.float32)
        _check(self._lib.mpm_write_particles(self._handle, _lib.ptr(packed), packed.shape[0]),
               "Failed to upload GPU MLS-MPM particles.")

    def measure_queue_completion_ms(self) -> float:
        self._assert_active()
        out = ctypes.c_double()
        _check(self._lib.mpm_queue_completion_ms(self._handle, ctypes.byref(out)), "Failed to measure the queue.")
        return float(out.value)

    # ----------------------------------------------------------- interaction --
    def _world_point(self, point, name: str) -> tuple:
        """validateMpmWorldPoint, solver.ts:3228-3242."""
        if not isinstance(point, dict):
            raise TypeError(f"{name} must be a vector.")
        x, y = _interaction_float32(point.get("x"), f"{name}.x"), _interaction_float32(point.get("y"), f"{name}.y")
        if x < 0 or x > self._state.domain_width_f32 or y < 0 or y > self._state.domain_height_f32:
            raise RangeError(f"{name} must be inside the MLS-MPM domain.")
        return x, y

    def _pick_radius(self, radius) -> float:
        """validateMpmPickRadius, solver.ts:3244-3250."""
        value = _interaction_float32(radius, "pick radius")
        if value < 0 or value > max(self._state.domain_width_f32, self._state.domain_height_f32):
            raise RangeError("pick radius must be non-negative and within the MLS-MPM domain extent.")
        return value

    def _resolve_selection(self, selection) -> tuple:
        """resolveSelection, solver.ts:1363-1387 -> (start, count)."""
        if not isinstance(selection, dict):
            raise TypeError("selection must identify an MPM particle.")
        index, oid = selection.get("particleIndex"), selection.get("objectId")
        if (not _is_safe_integer(index) or index < 0 or index >= self._slot_count or not _is_safe_integer(oid)
                or oid < 0 or oid > 0xFFFFFFFF):
            raise RangeError("selection must identify an active MPM particle.")
        self._world_point(selection.get("anchor"), "selection anchor")
        rng = self._object_ranges.get(oid)
        if rng is None or not rng[0] <= index < rng[0] + rng[1]:
            raise RangeError("selection objectId does not match the selected particle.")
        return rng

    def pick(self, point, radius):
        """pick, solver.ts:2733-2815: the nearest active particle within
        `radius` as {particleIndex, objectId, anchor}, or None."""
        self._assert_active()
        x, y = self._world_point(point, "pick point")
        r = self._pick_radius(radius)
        if self._active_count == 0:
            return None
        index, oid = ctypes.c_uint32(), ctypes.c_uint32()
        anchor = np.zeros(2, dtype=np.float32)
        _check(self._lib.mpm_pick(self._handle, x, y, r, ctypes.byref(index), _lib.ptr(anchor), ctypes.byref(oid)),
               "Failed to pick an MLS-MPM particle from GPU state.")
        if index.value == 0xFFFFFFFF:
            return None
        rng = self._object_ranges.get(oid.value)
        if rng is None or not rng[0] <= index.value < rng[0] + rng[1]:
            raise RuntimeError("GPU returned an object id inconsistent with the selected particle.")
        return {"particleIndex": int(index.value), "objectId": int(oid.value),
                "anchor": {"x": float(anchor[0]), "y": float(anchor[1])}}

    def begin_drag(self, selection, target, radius) -> None:
        """beginDrag (solver.ts:2817-2829): a grid-node spring toward `target`
        within `radius` (finishGridVelocity, shaders.ts:1757-1775)."""
        self._assert_active()
        self._resolve_selection(selection)
        x, y = self._world_point(target, "drag target")
        r = self._pick_radius(radius)
        if r <= 0:
            raise RangeError("drag radius must be greater than zero.")
        self._write_drag(x, y, r)
        self._active_drag = {"radius": r}

    def update_drag(self, target) -> None:
        """updateDrag (solver.ts:2831-2836)."""
        self._assert_active()
        if self._active_drag is None:
            return
        x, y = self._world_point(target, "drag target")
        self._write_drag(x, y, self._active_drag["radius"])

    def end_drag(self) -> None:
        """endDrag (solver.ts:2838-2843)."""
        if self._active_drag is None:
            return
        self._active_drag = None
        if not self._disposed:
            _check(self._lib.mpm_set_drag(self._handle, None), "Failed to end the drag.")

    def _write_drag(self, x: float, y: float, radius: float) -> None:
        drag = _lib.MpmDrag(x, y, radius, MPM_MLS_GPU_DRAG_STIFFNESS, MPM_MLS_GPU_DRAG_DAMPING)
        _check(self._lib.mpm_set_drag(self._handle, ctypes.byref(drag)), "Failed to set the drag target.")

    def append_particles(self, particles) -> dict:
        """appendParticles, solver.ts:2108-2278: an emitter batch as a new
        object; returns the reference's MpmMlsGpuAppendResult."""
        self._assert_active()
        if not isinstance(particles, (list, tuple)) and not hasattr(particles, "px"):
            raise TypeError("particles must be an array of emitter particles.")
        requested = len(particles)

        def result(accepted, refused, dropped, velocity_bound=0.0, reason=None):
            out = {"requested": requested, "accepted": accepted, "refused": refused, "dropped": dropped,
                   "activeParticleCount": self._active_count, "allocatedParticleCount": self._slot_count,
                   "capacity": self.particle_capacity, "velocityBound": velocity_bound}
            if reason is not None:
                out["reason"] = reason
            return out

        if requested == 0:
            return result(0, 0, 0)
        if self._cfl_speed_measurement_submitted:
            return result(0, requested, 0, 0.0,
                          "wait for the submitted CFL speed readback before emitting particles")
        available = self.particle_capacity - self._slot_count
        if available <= 0:
            return result(0, 0, requested, 0.0, f"particle slot capacity {self.particle_capacity} is full")
        if self._next_object_id > 0xFFFFFFFF:
            return result(0, requested, 0, 0.0, "no object ids remain for a new emitter group")
        object_id = self._next_object_id
        arrays = particles if hasattr(particles, "px") else particles_from_dicts(particles)
        if np.any(arrays.bonded_vertex >= 0):
            return result(0, requested, 0, 0.0,
                          "triangle-bonded particles cannot be appended without a complete object topology")
        arrays = arrays.copy()
        arrays.object_id[:] = object_id
        cfg = dict(self._state.config, capacity=requested, fractureBonds=[])
        try:
            candidate = validate_mpm_mls_gpu_input(arrays, cfg)
        except Exception as error:  # noqa: BLE001 - the reference reports any validation failure as a refusal
            reason = str(error).strip() or "emitter particles failed GPU input validation"
            return result(0, requested, 0, 0.0, reason)
        if len(candidate.bonded_body_starts) > 0:
            return result(0, requested, 0, 0.0,
                          "triangle-bonded particles cannot be appended without a complete object topology")
        accepted = min(requested, available)
        additions = derive_mpm_mls_gpu_cfl_bounds(arrays.take(np.arange(accepted)), candidate.config)
        if self.cfl_bounds is not None and additions is None:
            return result(0, requested, 0, 0.0, "appended material has no safely derived CFL wave-speed bound")
        packed = np.ascontiguousarray(candidate.packed_particles[:accepted], dtype=np.float32)
        ids = np.full(accepted, object_id, dtype=np.uint32)
        first = ctypes.c_uint32()
        try:
            _check(self._lib.mpm_append_particles(self._handle, _lib.ptr(packed), _lib.ptr(ids), accepted,
                                                  ctypes.byref(first)),
                   "Failed to append a validated GPU MLS-MPM emitter batch.")
        except Exception:
            self._cfl_state_usable = False
            raise
        self._object_ranges[object_id] = (int(first.value), accepted)
        self._slot_count += accepted
        self._active_count += accepted
        self._next_object_id += 1
        if additions is not None and self.cfl_bounds is not None:
            self.cfl_bounds = dict(self.cfl_bounds,
                                   waveSpeedBound=max(self.cfl_bounds["waveSpeedBound"], additions["waveSpeedBound"]),
                                   velocityBound=max(self.cfl_bounds["velocityBound"], additions["velocityBound"]))
            self._last_scheduled_velocity_bound = max(self._last_scheduled_velocity_bound or 0.0,
                                                      additions["velocityBound"])
        velocity_bound = additions["velocityBound"] if additions is not None else 0.0
        return result(accepted, 0, requested - accepted, velocity_bound,
                      None if requested == accepted else
                      f"accepted only {accepted} of {requested}; GPU slot capacity is exhausted")

    def remove_particles_in_outlet(self, bounds) -> int:
        """removeParticlesInOutlet, solver.ts:2280-2386: removes the water and
        oil particles inside the bounds; returns how many."""
        self._assert_active()
        if not isinstance(bounds, dict):
            raise TypeError("outlet bounds must be an object.")
        x0, y0 = self._world_point({"x": bounds.get("minX"), "y": bounds.get("minY")}, "outlet minimum")
        x1, y1 = self._world_point({"x": bounds.get("maxX"), "y": bounds.get("maxY")}, "outlet maximum")
        if x0 > x1 or y0 > y1:
            raise RangeError("outlet minimum coordinates must not exceed the maximum.")
        if self._slot_count == 0 or self._active_count == 0:
            return 0
        removed = ctypes.c_uint32()
        try:
            _check(self._lib.mpm_remove_particles_in_outlet(self._handle, x0, y0, x1, y1, ctypes.byref(removed)),
                   "Failed to remove liquid particles from the GPU outlet region.")
        except Exception:
            self._cfl_state_usable = False
            raise
        if removed.value > self._active_count:
            raise RuntimeError("GPU reported an outlet removal count above the active particle count.")
        self._active_count -= removed.value
        self._has_removed = self._has_removed or removed.value > 0
        return int(removed.value)

    def gather_surface_occupancy(self) -> np.ndarray:
        """The water/oil free-surface field that render('surface') draws
        (solver.ts:2043-2066; gatherSurfaceOccupancy, shaders.ts:700-806),
        gathered on the GPU from the current state without the renderer:
        (node_h, node_w, 2) float32, halo node (x, y) at [y + 1, x + 1], the
        water and oil display area 2 V det(F) w / cellSize^2.  The device copy
        stays in the solver (surface_field_device).  Raises
        MpmMlsGpuSurfaceError when the gather set a surface flag."""
        self._assert_active()
        nodes = int(self._lib.mpm_node_count(self._handle))
        field = np.zeros((nodes, 2), dtype=np.float32)
        flags = ctypes.c_uint32()
        _check(self._lib.mpm_gather_surface_occupancy(self._handle, _lib.ptr(field), ctypes.byref(flags)),
               "GPU free-surface occupancy gather failed")
        error = decode_surface_error([0] * 7 + [flags.value])
        if error is not None:
            raise error
        grid = self._state.config["grid"]
        return field.reshape(grid["cellsY"] + 3, grid["cellsX"] + 3, 2)

    def surface_field_device(self):
        """(device pointer, node_w, node_h) of the last gathered surface field
        (two float32 per halo node, owned by the solver)."""
        self._assert_active()
        ptr, w, h = ctypes.c_void_p(), ctypes.c_uint32(), ctypes.c_uint32()
        _check(self._lib.mpm_surface_field_device(self._handle, ctypes.byref(ptr), ctypes.byref(w), ctypes.byref(h)),
               "no surface field")
        return int(ptr.value), int(w.value), int(h.value)

    def clone(self, selection, offset) -> bool:
        """clone, solver.ts:2852-2940: a copy of the selected object moved by
        `offset`; False when it cannot be placed."""
        self._assert_active()
        start, count = self._resolve_selection(selection)
        if not isinstance(offset, dict):
            raise TypeError("clone offset must be a vector.")
        ox = _interaction_float32(offset.get("x"), "clone offset.x")
        oy = _interaction_float32(offset.get("y"), "clone offset.y")
        if self._has_removed or self._state.fracture_bond_count > 0 or len(self._state.bonded_body_starts) > 0:
            return False
        if count > self.particle_capacity - self._slot_count:
            return False
        if self._next_object_id > 0xFFFFFFFF:
            raise RangeError("No unsigned 32-bit object ids remain for MLS-MPM cloning.")
        object_id = self._next_object_id
        self.end_drag()
        first = ctypes.c_uint32()
        _check(self._lib.mpm_clone_range(self._handle, start, count, ox, oy, object_id, ctypes.byref(first)),
               "Failed to clone the selected MLS-MPM object on the GPU.")
        self._object_ranges[object_id] = (int(first.value), count)
        self._slot_count += count
        self._active_count += count
        self._next_object_id += 1
        return True

    # ---------------------------------------------------------------- probes --
    def probe_sort(self, dt: float):
        n, nodes = self._slot_count, self.node_count
        keys = np.zeros(n, dtype=np.uint32)
        perm = np.zeros(n, dtype=np.uint32)
        starts = np.zeros(nodes + 1, dtype=np.uint32)
        _check(self._lib.mpm_probe_sort(self._handle, fround(dt), _lib.ptr(keys), _lib.ptr(perm), _lib.ptr(starts)),
               "sort probe failed")
        return keys, perm, starts

    def probe_fixed_point(self, dt: float):
        n, nodes = self._slot_count, self.node_count
        words = np.zeros((nodes, 11), dtype=np.int32)
        affine = np.zeros((n, 4), dtype=np.float32)
        _check(self._lib.mpm_probe_fixed_point(self._handle, fround(dt), _lib.ptr(words), _lib.ptr(affine)),
               "fixed-point probe failed")
        return words, affine

    def probe_triangle_field(self, dt: float) -> dict:
        """The bonded-triangle field of the current particles (measurement /
        parity probe): sd, body (first-vertex index, -1: none), normal, bary
        (three weights), as (cellsY+3, cellsX+3) arrays."""
        nodes = self.node_count
        raw = np.zeros((nodes, 8), dtype=np.float32)
        _check(self._lib.mpm_probe_triangle_field(self._handle, fround(dt), _lib.ptr(raw)),
               "triangle field probe failed")
        grid = self._state.config["grid"]
        h, w = int(grid["cellsY"]) + 3, int(grid["cellsX"]) + 3
        words = raw.view(np.uint32)
        b1, b2 = raw[:, 4].astype(np.float64), raw[:, 5].astype(np.float64)
        return {"sd": raw[:, 0].reshape(h, w), "body": (words[:, 1].astype(np.int64) - 1).reshape(h, w),
                "normal": raw[:, 2:4].reshape(h, w, 2),
                "bary": np.stack([1.0 - b1 - b2, b1, b2], axis=1).reshape(h, w, 3)}

    def launch_shape(self) -> dict:
        """The persistent grids of the default path's P2G and G2P kernels."""
        p, g, sms = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        _check(self._lib.mpm_get_launch_shape(self._handle, ctypes.byref(p), ctypes.byref(g), ctypes.byref(sms)),
               "launch shape read failed")
        return {"p2gCtas": int(p.value), "g2pCtas": int(g.value), "smCount": int(sms.value)}

    def set_launch_shape(self, p2g_ctas: int = 0, g2p_ctas: int = 0) -> None:
        """Sets the persistent grids of the default path's P2G and G2P
        kernels (0 keeps a value); results do not depend on them."""
        self._assert_active()
        _check(self._lib.mpm_set_launch_shape(self._handle, int(p2g_ctas), int(g2p_ctas)), "launch shape failed")

    def autotune(self, substeps: int = 8) -> dict:
        """Picks the fastest persistent grids for P2G and G2P on this
        workload (mpm_autotune: real substeps timed per candidate, the state
        restored); call after a first batch."""
        self._assert_active()
        p, g, ms = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_double()
        _check(self._lib.mpm_autotune(self._handle, int(substeps), ctypes.byref(p), ctypes.byref(g), ctypes.byref(ms)),
               "autotune failed")
        return dict(self.substep_variant(), p2gCtas=int(p.value), g2pCtas=int(g.value),
                    transferMsPerSubstep=float(ms.value))

    def substep_variant(self) -> dict:
        """How the default path runs a substep: `fused` (one cooperative launch
        of persistent CTAs, else four launches), the P2G stage capacity, the
        one-launch form's persistent grid and its co-resident limit, whether
        G2P runs its water-and-oil instantiation and whether G2P writes the
        next P2G's records."""
        f, cap, n, most, liq, rec = (ctypes.c_uint32() for _ in range(6))
        _check(self._lib.mpm_get_substep_variant(self._handle, ctypes.byref(f), ctypes.byref(cap), ctypes.byref(n),
                                                 ctypes.byref(most), ctypes.byref(liq), ctypes.byref(rec)),
               "substep variant read failed")
        return {"fused": bool(f.value), "stageCapacity": int(cap.value), "substepCtas": int(n.value),
                "maxSubstepCtas": int(most.value), "liquidKernels": bool(liq.value), "p2gRecords": bool(rec.value)}

    def set_substep_variant(self, fused: bool = True, stage_capacity: int = 0, substep_ctas: int = 0,
                            liquid_kernels: bool = True, p2g_records=None) -> None:
        """Chooses the substep variant (mpm_set_substep_variant; 0 keeps the
        stage capacity or the grid; `p2g_records` None picks by the
        materials).  Results do not depend on `fused`, the grid,
        `liquid_kernels` or `p2g_records`."""
        self._assert_active()
        records = 2 if p2g_records is None else (1 if p2g_records else 0)
        _check(self._lib.mpm_set_substep_variant(self._handle, 1 if fused else 0, int(stage_capacity),
                                                 int(substep_ctas), 1 if liquid_kernels else 0, records),
               "substep variant change failed")

    def set_barrier_limit(self, limit_ns: int, skip_cta: int = 0xFFFFFFFF) -> None:
        """The one-launch substep's barrier wait limit in nanoseconds; `skip_cta`
        makes one CTA leave without arriving (a test of the limit)."""
        self._assert_active()
        _check(self._lib.mpm_set_barrier_limit(self._handle, int(limit_ns), int(skip_cta)),
               "barrier limit change failed")

    def dispose(self) -> None:
        if self._disposed:
            return
        self._disposed = True
        self._lib.mpm_destroy(self._handle)
        self._handle = None

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass


def _create(particles, config, cfl_bounds, atomic, device, fixed_point_shift):
    state = validate_mpm_mls_gpu_input(particles, config)
    derived = derive_mpm_mls_gpu_cfl_bounds(particles, state.config)
    certified = validate_cfl_bounds(cfl_bounds, state, derived)
    return MpmMlsGpuSolver(state, certified, atomic, device, fixed_point_shift)


def create_mpm_mls_gpu_solver(particles, config, cfl_bounds=None, device: int = 0) -> MpmMlsGpuSolver:
    """createMpmMlsGpuSolver, solver.ts:390-397 (headless: a device ordinal
    replaces the canvas)."""
    return _create(particles, config, cfl_bounds, False, device, DEFAULT_FIXED_POINT_SHIFT)


def create_experimental_mpm_mls_atomic_gpu_solver(particles, config, cfl_bounds=None, device: int = 0,
                                                  fixed_point_shift: int = DEFAULT_FIXED_POINT_SHIFT):
    """createExperimentalMpmMlsAtomicGpuSolver, solver.ts:399-406.  The
    fixed-point scale 2^fixed_point_shift defaults to the reference's 2^24."""
    return _create(particles, config, cfl_bounds, True, device, fixed_point_shift)
