"""Many independent scenes stepped together by one GPU solver.

No counterpart in the reference, which creates one solver per scene
(createMpmMlsGpuSolver, src/lib/mpm/kernels/solver.ts:390-406) and steps it
with stepBatch / stepCflBatch (:1407-1722).  Here one handle holds every
scene (mpmb_create) and one submit runs each scene's own microstep count and
microstep dt (mpmb_step_batch): one launch per kernel and substep for all
scenes, every scene's tiles in one tile list.  Each scene keeps the
single-scene semantics: its own CFL plan (calculateMpmCflMicrosteps,
src/lib/mpm/kernels/cfl.ts), its own status words and rollback, and the
retry and continuation rules of stepCflBatchAdaptive (solver.ts:1724-2021)
applied scene by scene.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from .cfl import calculate_mpm_cfl_microsteps, calculate_mpm_cfl_safe_dt, calculate_mpm_cfl_velocity_limit
from .cfl_bounds import derive_mpm_mls_gpu_cfl_bounds
from .errors import RangeError, decode_numerical_error, is_recoverable_cfl_error
from .layout import PARTICLE_FLOATS, fround, pack_step_parameters, unpack_particles, validate_mpm_mls_gpu_input
from .solver import (CFL_RECOVERY_BOUND_SAFETY_FACTOR, EPSILON, MIN_VALUE, _check, _is_capacity_error,
                     native_config, validate_cfl_bounds)


class MpmBatchedGpuSolver:
    """A batch of independent scenes (particles and config each) on one GPU."""

    def __init__(self, states, cfl_bounds, device: int = 0):
        if not states:
            raise RangeError("a batch needs at least one scene")
        for k, state in enumerate(states):
            if len(state.bonded_body_starts) or state.fracture_bond_count:
                raise RangeError(f"scene {k}: bonded triangle bodies and fracture bonds take a single-scene solver")
        self._lib = _lib.load_library()
        self._states = states
        self.cfl_bounds = cfl_bounds
        configs = (_lib.MpmConfig * len(states))()
        for k, state in enumerate(states):
            configs[k] = native_config(state, False, 0, device)
        counts = np.array([s.particle_count for s in states], dtype=np.uint32)
        packed = np.ascontiguousarray(np.concatenate([s.packed_particles for s in states]), dtype=np.float32)
        ids = np.ascontiguousarray(np.concatenate([s.packed_object_ids for s in states]), dtype=np.uint32)
        handle = ctypes.c_void_p()
        rc = self._lib.mpmb_create(ctypes.cast(configs, ctypes.c_void_p), len(states), _lib.ptr(counts),
                                   _lib.ptr(packed), _lib.ptr(ids), ctypes.byref(handle))
        if rc != _lib.MPM_OK:
            raise RuntimeError(f"Failed to initialize the batched GPU MLS-MPM solver: {_lib.last_error()}")
        self._handle = handle
        self._counts = counts
        self._bases = np.concatenate([[0], np.cumsum(counts, dtype=np.int64)])
        self._disposed = False
        # the factor a failed batch's observed speed and wave speed are raised by
        # before the retry (solver.ts:73 fixes it at 1.25); callers may study others
        self.recovery_bound_factor = CFL_RECOVERY_BOUND_SAFETY_FACTOR
        self.device_ms_total = 0.0
        self.committed_particle_substeps = 0

    # ---------------------------------------------------------------- props --
    @property
    def scene_count(self) -> int:
        return len(self._states)

    @property
    def particle_counts(self) -> np.ndarray:
        return self._counts.copy()

    def _assert_active(self):
        if self._disposed:
            raise RuntimeError("MLS-MPM GPU solver has been disposed.")

    # ------------------------------------------------------------- stepping --
    def step_batch(self, step_counts, dts, gravity, velocity_limits=None) -> None:
        """One submit: scene k runs step_counts[k] substeps of dts[k] (0:
        the scene sits the submit out), under `gravity` (one {x, y} for all
        scenes or one per scene) and, when `velocity_limits` is given, the
        CFL guard (the scene's wave-speed bound, velocity_limits[k])."""
        self._assert_active()
        s = self.scene_count
        if len(step_counts) != s or len(dts) != s:
            raise RangeError("step_counts and dts need one entry per scene")
        gravities = gravity if isinstance(gravity, (list, tuple)) else [gravity] * s
        steps = np.zeros(s, dtype=np.uint32)
        dt32 = np.zeros(s, dtype=np.float32)
        g = np.zeros(2 * s, dtype=np.float32)
        guards = None
        if velocity_limits is not None:
            if self.cfl_bounds is None:
                raise RangeError("this solver configuration has no safely derived CFL bounds.")
            guards = (_lib.MpmCflGuard * s)()
        for k in range(s):
            count = int(step_counts[k])
            if count < 0:
                raise RangeError("stepCount must be a non-negative safe integer.")
            steps[k] = count
            if count == 0:
                g[2 * k], g[2 * k + 1] = fround(gravities[k]["x"]), fround(gravities[k]["y"])
                continue
            guard = None
            if guards is not None:
                guard = {"waveSpeedBound": self.cfl_bounds[k]["waveSpeedBound"],
                         "velocityBound": float(velocity_limits[k])}
            d, gx, gy, wave, vel, _ = pack_step_parameters(self._states[k], dts[k], gravities[k], guard)
            dt32[k], g[2 * k], g[2 * k + 1] = d, gx, gy
            if guards is not None:
                guards[k] = _lib.MpmCflGuard(wave, vel)
        if int(steps.max()) < 1:
            raise RangeError("stepCount must be a positive safe integer.")
        native_guards = None if guards is None else ctypes.cast(guards, ctypes.c_void_p)
        _check(self._lib.mpmb_step_batch(self._handle, _lib.ptr(steps), _lib.ptr(dt32), _lib.ptr(g), native_guards),
               "Failed to encode or submit a batch of MLS-MPM scenes.")

    def last_batch_device_ms(self) -> float:
        """Device time of the last submit (CUDA events on the solver's stream)."""
        out = ctypes.c_double()
        _check(self._lib.mpm_last_batch_device_ms(self._handle, ctypes.byref(out)), "batch timing failed")
        return float(out.value)

    def read_compact(self):
        """Per scene: maximum speed, committed microsteps, 8 status words."""
        self._assert_active()
        s = self.scene_count
        speeds = np.zeros(s, dtype=np.float32)
        done = np.zeros(s, dtype=np.uint32)
        status = np.zeros((s, 8), dtype=np.uint32)
        _check(self._lib.mpmb_read_compact(self._handle, _lib.ptr(speeds), _lib.ptr(done), _lib.ptr(status)),
               "Failed to read the compact GPU measurements of the scenes.")
        return speeds, done, status

    def clear_status(self) -> None:
        _check(self._lib.mpm_clear_status(self._handle), "Failed to clear the GPU numerical status.")

    def check_numerical_status(self) -> list:
        """checkNumericalStatus (solver.ts:2514-2570) per scene: None or the
        scene's MpmMlsGpuNumericalError."""
        _, _, status = self.read_compact()
        return [decode_numerical_error(status[k]) for k in range(self.scene_count)]

    def step_cfl_batch_adaptive(self, macro_dt: float, velocity_bounds, max_microsteps: int, gravity) -> list:
        """One macrostep of `macro_dt` for every scene under the rules of
        stepCflBatchAdaptive (solver.ts:1724-2021), scene by scene: a CFL plan
        from the scene's wave-speed bound and velocity_bounds[k]; a scene that
        fails its guard is rolled back to the failed microstep and retries the
        failed interval at a finer plan, then continues with the remaining
        duration, while the scenes that are done sit out.  Returns per scene
        the measured maximum speed, the recommended velocity bound for the
        next macrostep, the committed and attempted microsteps and the
        retries."""
        self._assert_active()
        if self.cfl_bounds is None:
            raise RangeError("CFL stepping requires a material-derived wave-speed bound; this solver configuration "
                             "has no safely derived CFL bounds.")
        if not math.isfinite(macro_dt) or macro_dt <= 0:
            raise RangeError("macroDt must be positive and finite.")
        s = self.scene_count
        scenes = []
        for k in range(s):
            cell = self._states[k].config["grid"]["cellSize"]
            b = self.cfl_bounds[k]
            vb = float(velocity_bounds[k])
            plan = calculate_mpm_cfl_microsteps(macro_dt, cell, b["waveSpeedBound"], vb, max_microsteps,
                                                courantLimit=b.get("courantLimit"))
            scenes.append({"cell": cell, "velocity": vb, "plan": plan, "duration": macro_dt, "remaining": macro_dt,
                           "consumed": 0, "committed": 0, "retries": 0, "speed": 0.0, "done": False,
                           "recommended": None})
        tolerance = max(macro_dt, MIN_VALUE) * EPSILON * 4
        while True:
            live = [k for k in range(s) if not scenes[k]["done"]]
            if not live:
                break
            steps, dts, limits = [0] * s, [0.0] * s, [0.0] * s
            for k in live:
                sc = scenes[k]
                plan = sc["plan"]
                budget = max_microsteps - sc["consumed"]
                if plan["stepCount"] < 1 or plan["stepCount"] > budget:
                    raise RangeError(f"scene {k}: adaptive CFL retry requires {plan['stepCount']} microsteps with "
                                     f"{budget} remaining.")
                b = self.cfl_bounds[k]
                limit = calculate_mpm_cfl_velocity_limit(sc["cell"], b["waveSpeedBound"], plan["microDt"],
                                                         b.get("courantLimit"))
                if limit < sc["velocity"]:
                    raise RangeError(f"scene {k}: float32 microDt does not preserve the planned CFL velocity bound; "
                                     "increase the microstep count.")
                steps[k], dts[k], limits[k] = plan["stepCount"], plan["microDt"], limit
            self.step_batch(steps, dts, gravity, limits)
            self.device_ms_total += self.last_batch_device_ms()
            speeds, done, status = self.read_compact()
            cleared = False
            for k in live:
                sc = scenes[k]
                plan = sc["plan"]
                attempt = plan["stepCount"]
                error = decode_numerical_error(status[k], int(done[k]), float(speeds[k]))
                b = self.cfl_bounds[k]
                if error is not None:
                    if not is_recoverable_cfl_error(error):
                        raise error
                    completed = int(done[k])
                    if completed >= attempt:
                        raise RuntimeError(f"scene {k}: adaptive CFL recovery could not determine completed "
                                           f"microsteps: {error}") from error
                    sc["remaining"] -= completed * plan["microDt"]
                    sc["consumed"] += attempt
                    sc["committed"] += completed
                    self.committed_particle_substeps += completed * int(self._counts[k])
                    observed = max(error.measured_maximum_speed or 0.0,
                                   (error.cfl_details or {}).get("particleSpeed", 0.0))
                    retry_velocity = max(sc["velocity"], observed * self.recovery_bound_factor)
                    if error.cfl_details is not None:
                        wave = error.cfl_details["waveSpeed"] * self.recovery_bound_factor
                        self.cfl_bounds[k] = b = dict(b, waveSpeedBound=max(b["waveSpeedBound"], wave))
                    sc["velocity"], sc["speed"] = retry_velocity, observed
                    cleared = True
                    retry_budget = max_microsteps - sc["consumed"]
                    failed_interval = min(sc["remaining"], plan["microDt"])
                    if retry_budget < 2:
                        sc["done"], sc["recommended"] = True, retry_velocity
                        continue
                    try:
                        sc["plan"] = calculate_mpm_cfl_microsteps(
                            failed_interval, sc["cell"], b["waveSpeedBound"], retry_velocity, retry_budget,
                            minimumStepCount=2, courantLimit=b.get("courantLimit"))
                    except RangeError as cause:
                        if not _is_capacity_error(cause):
                            raise
                        sc["done"], sc["recommended"] = True, retry_velocity
                        continue
                    sc["duration"] = failed_interval
                    sc["retries"] += 1
                    continue
                sc["consumed"] += attempt
                sc["committed"] += attempt
                self.committed_particle_substeps += attempt * int(self._counts[k])
                sc["speed"] = float(speeds[k])
                sc["remaining"] = max(0.0, sc["remaining"] - sc["duration"])
                if sc["remaining"] <= tolerance:
                    sc["remaining"] = 0.0
                    sc["done"] = True
                    sc["recommended"] = max(sc["velocity"], sc["speed"]) if sc["retries"] > 0 else sc["speed"]
                    continue
                budget = max_microsteps - sc["consumed"]
                sc["velocity"] = max(sc["velocity"], sc["speed"])
                if budget < 2:
                    sc["done"], sc["recommended"] = True, sc["velocity"]
                    continue
                safe = calculate_mpm_cfl_safe_dt(sc["cell"], b["waveSpeedBound"], sc["velocity"],
                                                 b.get("courantLimit", 0.3))
                max_step = min(plan["microDt"], safe)
                required = math.ceil(sc["remaining"] / max_step)
                continuation, minimum = sc["remaining"], max(1, required)
                if required >= budget:
                    continuation = min(sc["remaining"], max_step * (budget - 1) * (1 - EPSILON * 8))
                    minimum = max(1, math.ceil(continuation / max_step))
                sc["plan"] = calculate_mpm_cfl_microsteps(continuation, sc["cell"], b["waveSpeedBound"],
                                                          sc["velocity"], budget, minimumStepCount=minimum,
                                                          courantLimit=b.get("courantLimit"))
                sc["duration"] = continuation
            if cleared:
                self.clear_status()
        return [{"maximumSpeed": sc["speed"], "recommendedVelocityBound": sc["recommended"],
                 "committedMicroStepCount": sc["committed"], "attemptedMicroStepCount": sc["consumed"],
                 "retryCount": sc["retries"], "remainingDuration": sc["remaining"]} for sc in scenes]

    def profile_substeps(self, step_count: int, dt: float, gravity: dict) -> dict:
        """Runs `step_count` real substeps of `dt` in every scene, kernel by
        kernel with CUDA events between them: {kernel name: (milliseconds,
        launches)}."""
        self._assert_active()
        slots = int(self._lib.mpm_profile_kernel_slots())
        ms = np.zeros(slots, dtype=np.float64)
        launches = np.zeros(slots, dtype=np.uint32)
        _check(self._lib.mpm_profile_substeps(self._handle, step_count, fround(dt), fround(gravity["x"]),
                                              fround(gravity["y"]), None, _lib.ptr(ms), _lib.ptr(launches)),
               "profiled substeps failed")
        return {self._lib.mpm_profile_kernel_name(k).decode(): (float(ms[k]), int(launches[k]))
                for k in range(slots) if launches[k]}

    def count_active_nodes(self):
        """Active solid / water / oil nodes per substep of the last batch,
        summed over the scenes."""
        counts = np.zeros(3, dtype=np.uint32)
        _check(self._lib.mpm_count_active_nodes(self._handle, _lib.ptr(counts)), "active node count failed")
        return tuple(int(c) for c in counts)

    # -------------------------------------------------------------- readback --
    def read_particles_packed(self, scene: int):
        """The packed 20-word records and object ids of one scene, in its own
        particle order."""
        self._assert_active()
        if not 0 <= scene < self.scene_count:
            raise RangeError("scene must identify a scene of the batch.")
        base, count = int(self._bases[scene]), int(self._counts[scene])
        idx = np.arange(base, base + count, dtype=np.uint32)
        packed = np.zeros((count, PARTICLE_FLOATS), dtype=np.float32)
        ids = np.zeros(count, dtype=np.uint32)
        _check(self._lib.mpm_read_particles(self._handle, _lib.ptr(idx), count, _lib.ptr(packed), _lib.ptr(ids)),
               "Failed to read GPU MLS-MPM particles.")
        return packed, ids

    def read_particles(self, scene: int) -> list:
        packed, ids = self.read_particles_packed(scene)
        return unpack_particles(packed, ids)

    def launch_shape(self) -> dict:
        """The persistent grids of the default path's P2G and G2P kernels."""
        p, g, sms = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        _check(self._lib.mpm_get_launch_shape(self._handle, ctypes.byref(p), ctypes.byref(g), ctypes.byref(sms)),
               "launch shape read failed")
        return {"p2gCtas": int(p.value), "g2pCtas": int(g.value), "smCount": int(sms.value)}

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


def create_mpm_batched_gpu_solver(scenes, cfl_bounds=None, device: int = 0) -> MpmBatchedGpuSolver:
    """A batched solver over `scenes`, a list of (particles, config) pairs,
    each validated like createMpmMlsGpuSolver's input (layout.ts:122-607) with
    its CFL bounds derived per scene (cfl-bounds.ts); `cfl_bounds`, when
    given, holds one certified bound dict per scene."""
    states, bounds = [], []
    for k, (particles, config) in enumerate(scenes):
        state = validate_mpm_mls_gpu_input(particles, config)
        derived = derive_mpm_mls_gpu_cfl_bounds(particles, state.config)
        bounds.append(validate_cfl_bounds(None if cfl_bounds is None else cfl_bounds[k], state, derived))
        states.append(state)
    certified = None if any(b is None for b in bounds) else bounds
    return MpmBatchedGpuSolver(states, certified, device)
