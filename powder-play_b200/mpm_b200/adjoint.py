"""The differentiable form: gradients of a trajectory loss through the substep.

No counterpart in the reference, which computes no gradients.  An engine over
a batch of scenes of Tait water and fixed-corotated solid particles steps
them with the default path's arithmetic for those two models (prepareParticle,
p2g, updateGrid, g2p of src/lib/mpm/kernels/shaders.ts) at a fixed dt per
scene, evaluates the loss sum |x(T) - target|^2 per scene, and returns the
gradients of the total loss with respect to the initial velocities and the
per-scene material parameters (the water's Tait pressure coefficient, the
solid's lambda and mu) by checkpoint and recompute over the C ABI
(include/mpm_b200.h, mpma_*).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .cfl import calculate_mpm_cfl_safe_dt
from .errors import RangeError
from .layout import fround, validate_mpm_mls_gpu_input
from .solver import _check, native_config

PARAMETER_NAMES = ("tait", "lambda", "mu")


class MpmAdjointEngine:
    """Forward substeps with checkpoints and their adjoint, for many scenes."""

    def __init__(self, states, gravity, device: int = 0):
        if not states:
            raise RangeError("a batch needs at least one scene")
        self._lib = _lib.load_library()
        self._states = states
        configs = (_lib.MpmConfig * len(states))()
        for k, state in enumerate(states):
            configs[k] = native_config(state, False, 0, device)
        counts = np.array([s.particle_count for s in states], dtype=np.uint32)
        packed = np.ascontiguousarray(np.concatenate([s.packed_particles for s in states]), dtype=np.float32)
        gravities = gravity if isinstance(gravity, (list, tuple)) else [gravity] * len(states)
        g = np.array([[fround(gv["x"]), fround(gv["y"])] for gv in gravities], dtype=np.float32)
        handle = ctypes.c_void_p()
        _check(self._lib.mpma_create(ctypes.cast(configs, ctypes.c_void_p), len(states), _lib.ptr(counts),
                                     _lib.ptr(packed), _lib.ptr(g), ctypes.byref(handle)),
               "Failed to initialize the differentiable MLS-MPM engine")
        self._handle = handle
        self._counts = counts
        self._n = int(counts.sum())
        self._disposed = False
        self._forward_done = False

    @property
    def scene_count(self) -> int:
        return len(self._states)

    @property
    def particle_counts(self) -> np.ndarray:
        return self._counts.copy()

    def _assert_active(self):
        if self._disposed:
            raise RuntimeError("the differentiable engine has been disposed.")

    @property
    def parameters(self) -> np.ndarray:
        """(scenes, 3): Tait pressure coefficient, solid lambda, solid mu."""
        self._assert_active()
        out = np.zeros((self.scene_count, 3), dtype=np.float32)
        _check(self._lib.mpma_get_parameters(self._handle, _lib.ptr(out)), "parameter read failed")
        return out

    @parameters.setter
    def parameters(self, values) -> None:
        self._assert_active()
        values = np.ascontiguousarray(values, dtype=np.float32).reshape(self.scene_count, 3)
        _check(self._lib.mpma_set_parameters(self._handle, _lib.ptr(values)), "parameter update failed")
        self._forward_done = False

    def set_velocities(self, velocities) -> None:
        """Replaces the initial velocities, (particles, 2) in scene order."""
        self._assert_active()
        velocities = np.ascontiguousarray(velocities, dtype=np.float32).reshape(self._n, 2)
        _check(self._lib.mpma_set_velocities(self._handle, _lib.ptr(velocities)), "velocity update failed")
        self._forward_done = False

    def forward(self, substeps: int, dts, targets, checkpoint_every: int = 20) -> np.ndarray:
        """Steps every scene `substeps` times with its own dt from the initial
        state; returns the loss per scene against `targets` ((particles, 2))."""
        self._assert_active()
        dts = np.ascontiguousarray(dts, dtype=np.float32).reshape(self.scene_count)
        targets = np.ascontiguousarray(targets, dtype=np.float32).reshape(self._n, 2)
        loss = np.zeros(self.scene_count, dtype=np.float64)
        _check(self._lib.mpma_forward(self._handle, int(substeps), _lib.ptr(dts), int(checkpoint_every),
                                      _lib.ptr(targets), _lib.ptr(loss)), "forward pass failed")
        self._forward_done = True
        return loss

    def backward(self):
        """Gradients of the last forward pass's total loss: (initial velocities
        (particles, 2), parameters (scenes, 3))."""
        self._assert_active()
        if not self._forward_done:
            raise RuntimeError("backward() needs a completed forward() of the current inputs.")
        gv = np.zeros((self._n, 2), dtype=np.float32)
        gp = np.zeros((self.scene_count, 3), dtype=np.float64)
        _check(self._lib.mpma_backward(self._handle, _lib.ptr(gv), _lib.ptr(gp)), "adjoint pass failed")
        return gv, gp

    def read_positions(self) -> np.ndarray:
        self._assert_active()
        out = np.zeros((self._n, 2), dtype=np.float32)
        _check(self._lib.mpma_read_positions(self._handle, _lib.ptr(out)), "position read failed")
        return out

    def last_ms(self):
        """Device milliseconds of the last forward and backward passes."""
        f, b = ctypes.c_double(), ctypes.c_double()
        _check(self._lib.mpma_last_ms(self._handle, ctypes.byref(f), ctypes.byref(b)), "timing read failed")
        return float(f.value), float(b.value)

    def dispose(self) -> None:
        if self._disposed:
            return
        self._disposed = True
        self._lib.mpma_destroy(self._handle)
        self._handle = None

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass


def create_mpm_adjoint_engine(scenes, gravity, device: int = 0) -> MpmAdjointEngine:
    """An engine over `scenes`, a list of (particles, config) pairs validated
    like createMpmMlsGpuSolver's input (layout.ts:122-607)."""
    states = [validate_mpm_mls_gpu_input(particles, config) for particles, config in scenes]
    return MpmAdjointEngine(states, gravity, device)


def wave_speed_bound(particles, config) -> float:
    """The rest wave speed of the differentiable form's materials: Tait water
    sqrt(gamma B / rho), fixed-corotated solid sqrt((lambda + 2 mu) / rho)
    with rho the configured particle mass over its volume."""
    materials = list(particles.materials) + [config["material"]]
    used = set(int(m) if m >= 0 else len(particles.materials) for m in np.unique(particles.material))
    wave = 0.0
    for k in used:
        m = materials[k]
        if m["model"] == "water":
            gamma = (m.get("equationOfState") or {}).get("exponent", 0.0)
            wave = max(wave, float(np.sqrt(max(gamma, 1.0) * m["lambda"] / m["density"])))
        elif m["model"] == "fixed-corotated":
            rho = config["particleMass"] / config["particleVolume"]
            wave = max(wave, float(np.sqrt((m["lambda"] + 2.0 * m["mu"]) / rho)))
        else:
            raise RangeError("the differentiable form takes Tait water and fixed-corotated solids only")
    return wave


def fixed_cfl_dt(particles, config, gravity_magnitude: float, duration: float, courant: float = 0.3) -> float:
    """The fixed dt of a scene's schedule: the CFL step (calculateMpmCflSafeDt,
    cfl.ts:121-147) for the materials' rest wave speed and a velocity bound of
    the largest initial speed plus what gravity adds over `duration`."""
    speed = float(np.max(np.hypot(particles.vx, particles.vy))) if len(particles.vx) else 0.0
    velocity = speed + gravity_magnitude * duration
    return calculate_mpm_cfl_safe_dt(config["grid"]["cellSize"], wave_speed_bound(particles, config), velocity,
                                     courant)
