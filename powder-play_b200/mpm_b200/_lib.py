"""ctypes binding of libmpm_b200.so (include/mpm_b200.h).

The library is built in-tree by powder-play_b200/build.py.  Loading fails
loudly when it is missing: there is no CPU fallback on the product path.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(os.path.dirname(HERE), "libmpm_b200.so")

MPM_OK = 0
MPM_ERR_INVALID_ARGUMENT = -1
MPM_ERR_CUDA = -2
MPM_ERR_STATE = -3
MPM_P2G_GATHER = 0
MPM_P2G_FIXED_POINT = 1

EXPORTED_SYMBOLS = (
    "mpm_create", "mpm_step_batch", "mpm_read_compact", "mpm_read_status", "mpm_clear_status",
    "mpm_read_particles", "mpm_write_particles", "mpm_set_drag", "mpm_queue_completion_ms",
    "mpm_particle_count", "mpm_particle_capacity", "mpm_destroy", "mpm_last_error", "mpm_probe_sort",
    "mpm_probe_fixed_point", "mpm_probe_triangle_field", "mpm_probe_deformation", "mpm_node_count", "mpm_last_batch_device_ms", "mpm_profile_substeps",
    "mpm_profile_kernel_name", "mpm_profile_kernel_slots", "mpm_count_active_nodes", "mpm_stream",
    "mpmb_create", "mpmb_step_batch", "mpmb_read_compact", "mpmb_scene_count",
    "mpm_allocated_particle_count", "mpm_append_particles", "mpm_remove_particles_in_outlet", "mpm_pick",
    "mpm_clone_range", "mpm_set_launch_shape", "mpm_get_launch_shape", "mpm_autotune",
    "mpm_set_substep_variant", "mpm_get_substep_variant", "mpm_set_barrier_limit",
    "mpm_gather_surface_occupancy", "mpm_surface_field_device",
    "mpma_create", "mpma_set_parameters", "mpma_get_parameters", "mpma_set_velocities", "mpma_forward",
    "mpma_backward", "mpma_read_positions", "mpma_last_ms", "mpma_destroy",
)


class MpmConfig(ctypes.Structure):
    _fields_ = [
        ("cells_x", ctypes.c_uint32), ("cells_y", ctypes.c_uint32), ("cell_size", ctypes.c_float),
        ("particle_mass", ctypes.c_float), ("particle_volume", ctypes.c_float),
        ("bond_rest_length", ctypes.c_float), ("bond_stiffness", ctypes.c_float),
        ("bond_reference_dt", ctypes.c_float), ("wall_friction", ctypes.c_float), ("lambda_", ctypes.c_float),
        ("mu", ctypes.c_float), ("capacity", ctypes.c_uint32), ("p2g_mode", ctypes.c_uint32),
        ("fixed_point_shift", ctypes.c_uint32), ("device", ctypes.c_int32),
    ]


class MpmCflGuard(ctypes.Structure):
    _fields_ = [("wave_speed_bound", ctypes.c_float), ("velocity_limit", ctypes.c_float)]


class MpmDrag(ctypes.Structure):
    _fields_ = [("target_x", ctypes.c_float), ("target_y", ctypes.c_float), ("radius", ctypes.c_float),
                ("stiffness", ctypes.c_float), ("damping", ctypes.c_float)]


_lib = None


def load_library(path: str = LIBRARY_PATH) -> ctypes.CDLL:
    """Loads libmpm_b200.so and declares every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libmpm_b200.so is not built at {path}; run powder-play_b200/build.py")
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    u32, i32, f32 = ctypes.c_uint32, ctypes.c_int32, ctypes.c_float
    lib.mpm_create.argtypes = [P(MpmConfig), vp, vp, u32, vp, u32, vp, u32, vp, u32, P(vp)]
    lib.mpm_create.restype = i32
    lib.mpm_step_batch.argtypes = [vp, u32, f32, f32, f32, P(MpmCflGuard), f32]
    lib.mpm_step_batch.restype = i32
    lib.mpm_read_compact.argtypes = [vp, P(f32), P(u32), vp]
    lib.mpm_read_compact.restype = i32
    lib.mpm_read_status.argtypes = [vp, vp]
    lib.mpm_read_status.restype = i32
    lib.mpm_clear_status.argtypes = [vp]
    lib.mpm_clear_status.restype = i32
    lib.mpm_read_particles.argtypes = [vp, vp, u32, vp, vp]
    lib.mpm_read_particles.restype = i32
    lib.mpm_write_particles.argtypes = [vp, vp, u32]
    lib.mpm_write_particles.restype = i32
    lib.mpm_set_drag.argtypes = [vp, P(MpmDrag)]
    lib.mpm_set_drag.restype = i32
    lib.mpm_queue_completion_ms.argtypes = [vp, P(ctypes.c_double)]
    lib.mpm_queue_completion_ms.restype = i32
    lib.mpm_particle_count.argtypes = [vp]
    lib.mpm_particle_count.restype = u32
    lib.mpm_particle_capacity.argtypes = [vp]
    lib.mpm_particle_capacity.restype = u32
    lib.mpm_node_count.argtypes = [vp]
    lib.mpm_node_count.restype = u32
    lib.mpm_destroy.argtypes = [vp]
    lib.mpm_destroy.restype = None
    lib.mpm_last_error.argtypes = []
    lib.mpm_last_error.restype = ctypes.c_char_p
    lib.mpm_probe_sort.argtypes = [vp, f32, vp, vp, vp]
    lib.mpm_probe_sort.restype = i32
    lib.mpm_probe_triangle_field.argtypes = [vp, f32, vp]
    lib.mpm_probe_triangle_field.restype = i32
    lib.mpm_probe_fixed_point.argtypes = [vp, f32, vp, vp]
    lib.mpm_probe_fixed_point.restype = i32
    lib.mpm_probe_deformation.argtypes = [i32, vp, vp, u32, f32, vp, vp, vp, vp, vp]
    lib.mpm_probe_deformation.restype = i32
    lib.mpm_last_batch_device_ms.argtypes = [vp, P(ctypes.c_double)]
    lib.mpm_last_batch_device_ms.restype = i32
    lib.mpm_profile_substeps.argtypes = [vp, u32, f32, f32, f32, P(MpmCflGuard), vp, vp]
    lib.mpm_profile_substeps.restype = i32
    lib.mpm_profile_kernel_name.argtypes = [u32]
    lib.mpm_profile_kernel_name.restype = ctypes.c_char_p
    lib.mpm_profile_kernel_slots.argtypes = []
    lib.mpm_profile_kernel_slots.restype = u32
    lib.mpm_count_active_nodes.argtypes = [vp, vp]
    lib.mpm_count_active_nodes.restype = i32
    lib.mpm_stream.argtypes = [vp]
    lib.mpm_stream.restype = vp
    lib.mpmb_create.argtypes = [vp, u32, vp, vp, vp, P(vp)]
    lib.mpmb_create.restype = i32
    lib.mpmb_step_batch.argtypes = [vp, vp, vp, vp, vp]
    lib.mpmb_step_batch.restype = i32
    lib.mpmb_read_compact.argtypes = [vp, vp, vp, vp]
    lib.mpmb_read_compact.restype = i32
    lib.mpmb_scene_count.argtypes = [vp]
    lib.mpmb_scene_count.restype = u32
    lib.mpm_allocated_particle_count.argtypes = [vp]
    lib.mpm_allocated_particle_count.restype = u32
    lib.mpm_append_particles.argtypes = [vp, vp, vp, u32, P(u32)]
    lib.mpm_append_particles.restype = i32
    lib.mpm_remove_particles_in_outlet.argtypes = [vp, f32, f32, f32, f32, P(u32)]
    lib.mpm_remove_particles_in_outlet.restype = i32
    lib.mpm_pick.argtypes = [vp, f32, f32, f32, P(u32), vp, P(u32)]
    lib.mpm_pick.restype = i32
    lib.mpm_clone_range.argtypes = [vp, u32, u32, f32, f32, u32, P(u32)]
    lib.mpm_clone_range.restype = i32
    lib.mpm_gather_surface_occupancy.argtypes = [vp, vp, P(u32)]
    lib.mpm_gather_surface_occupancy.restype = i32
    lib.mpm_surface_field_device.argtypes = [vp, P(vp), P(u32), P(u32)]
    lib.mpm_surface_field_device.restype = i32
    lib.mpm_set_launch_shape.argtypes = [vp, u32, u32]
    lib.mpm_set_launch_shape.restype = i32
    lib.mpm_get_launch_shape.argtypes = [vp, P(u32), P(u32), P(u32)]
    lib.mpm_get_launch_shape.restype = i32
    lib.mpm_autotune.argtypes = [vp, u32, P(u32), P(u32), P(ctypes.c_double)]
    lib.mpm_autotune.restype = i32
    lib.mpm_set_substep_variant.argtypes = [vp, u32, u32, u32, u32, u32]
    lib.mpm_set_substep_variant.restype = i32
    lib.mpm_get_substep_variant.argtypes = [vp, P(u32), P(u32), P(u32), P(u32), P(u32), P(u32)]
    lib.mpm_get_substep_variant.restype = i32
    lib.mpm_set_barrier_limit.argtypes = [vp, ctypes.c_uint64, u32]
    lib.mpm_set_barrier_limit.restype = i32
    lib.mpma_create.argtypes = [vp, u32, vp, vp, vp, P(vp)]
    lib.mpma_create.restype = i32
    for name in ("mpma_set_parameters", "mpma_get_parameters", "mpma_set_velocities", "mpma_read_positions"):
        getattr(lib, name).argtypes = [vp, vp]
        getattr(lib, name).restype = i32
    lib.mpma_forward.argtypes = [vp, u32, vp, u32, vp, vp]
    lib.mpma_forward.restype = i32
    lib.mpma_backward.argtypes = [vp, vp, vp]
    lib.mpma_backward.restype = i32
    lib.mpma_last_ms.argtypes = [vp, P(ctypes.c_double), P(ctypes.c_double)]
    lib.mpma_last_ms.restype = i32
    lib.mpma_destroy.argtypes = [vp]
    lib.mpma_destroy.restype = None
    _lib = lib
    return lib


def last_error() -> str:
    return load_library().mpm_last_error().decode("utf-8", "replace")


def ptr(array) -> ctypes.c_void_p:
    """Data pointer of a C-contiguous numpy array (None -> NULL)."""
    if array is None:
        return None
    return ctypes.c_void_p(array.ctypes.data)
