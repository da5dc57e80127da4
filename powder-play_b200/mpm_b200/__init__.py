"""B200-native MLS-MPM substep: the Python host mirror of the reference's
GPU solver API (7korobi/powder-play src/lib/mpm/kernels/*) over the C ABI of
libmpm_b200.so (include/mpm_b200.h)."""
from .cfl import (DEFAULT_MPM_COURANT_LIMIT, calculate_mpm_cfl_microsteps, calculate_mpm_cfl_safe_dt,
                  calculate_mpm_cfl_velocity_limit)
from .cfl_bounds import calculate_mpm_cfl_velocity_bound, derive_mpm_mls_gpu_cfl_bounds
from .errors import MpmMlsGpuNumericalError, MpmMlsGpuSurfaceError, MpmNativeError, RangeError
from .layout import ParticleArrays, particles_from_dicts, particles_to_dicts, validate_mpm_mls_gpu_input
from .solver import (MpmMlsGpuSolver, create_experimental_mpm_mls_atomic_gpu_solver, create_mpm_mls_gpu_solver)
from .batched import MpmBatchedGpuSolver, create_mpm_batched_gpu_solver
from .step_scheduler import calculate_mpm_cfl_step_batch, calculate_mpm_step_batch, mean_sinusoidal_acceleration

__all__ = [
    "DEFAULT_MPM_COURANT_LIMIT", "calculate_mpm_cfl_microsteps", "calculate_mpm_cfl_safe_dt",
    "calculate_mpm_cfl_velocity_limit", "calculate_mpm_cfl_velocity_bound", "derive_mpm_mls_gpu_cfl_bounds",
    "MpmMlsGpuNumericalError", "MpmMlsGpuSurfaceError", "MpmNativeError", "RangeError", "ParticleArrays", "particles_from_dicts",
    "particles_to_dicts", "validate_mpm_mls_gpu_input", "MpmMlsGpuSolver",
    "create_experimental_mpm_mls_atomic_gpu_solver", "create_mpm_mls_gpu_solver", "calculate_mpm_cfl_step_batch",
    "calculate_mpm_step_batch", "mean_sinusoidal_acceleration", "MpmBatchedGpuSolver",
    "create_mpm_batched_gpu_solver",
]
