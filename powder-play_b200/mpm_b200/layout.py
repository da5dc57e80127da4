"""Input validation and packing into the reference's 20-word particle record.

Restates src/lib/mpm/kernels/layout.ts (7korobi/powder-play): validation and
packing `validateMpmMlsGpuInput` (:122-607), the step-parameter checks of
`packMpmMlsGpuStepParameters` (:896-997), and the float32 helpers (:1126-1160).

Particles are accepted either as reference-shaped dicts
(`{'position': {'x', 'y'}, 'velocity', 'C', 'F', 'objectId', 'material', ...}`)
or, for large scenes, as a columnar `ParticleArrays`.  Checks are vectorised;
when a check fails, the failing particle with the smallest index is re-checked
in the reference's order so the message names the same particle and field.
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass, field

import numpy as np

from .errors import RangeError
from .materials import (MODEL_CODES, SNOW_PLASTICITY, normalize_mpm_constitutive_model,
                        normalize_mpm_tait_equation_of_state)

PARTICLE_FLOATS = 20
PARTICLE_STRIDE_BYTES = PARTICLE_FLOATS * 4
NUMERICAL_STATUS_WORDS = 8
DEFAULT_BONDED_TRIANGLE_STIFFNESS = 0.35
UINT32_MAX = 0xFFFFFFFF
INT32_MAX = 0x7FFFFFFF
MAX_FLOAT32 = 3.4028234663852886e38
MAX_SAFE_INTEGER = 2 ** 53 - 1


_F32 = struct.Struct("<f")


def fround(value: float) -> float:
    """Math.fround: round to the nearest float32 (ties to even); beyond the
    float32 range, to an infinity."""
    try:
        return _F32.unpack(_F32.pack(value))[0]
    except (OverflowError, TypeError, struct.error):
        with np.errstate(over="ignore"):
            return float(np.float32(value))


def finite_float32(value: float, name: str, positive: bool = False) -> float:
    """finiteFloat32, layout.ts:1126-1138."""
    result = fround(value)
    if not math.isfinite(result) or abs(value) > MAX_FLOAT32:
        raise RangeError(f"{name} is outside the supported float32 range")
    if value != 0 and result == 0:
        raise RangeError(f"{name} underflows the supported float32 range")
    if positive and result <= 0:
        raise RangeError(f"{name} must remain positive in the supported float32 range")
    return result


def _finite_number(value, name: str) -> float:
    if isinstance(value, bool) or not isinstance(value, (int, float, np.floating, np.integer)) or not math.isfinite(value):
        raise TypeError(f"{name} must be a finite number")
    return float(value)


def _is_safe_integer(value) -> bool:
    """Number.isSafeInteger."""
    if isinstance(value, bool):
        return False
    if isinstance(value, (int, np.integer)):
        return abs(int(value)) <= MAX_SAFE_INTEGER
    if isinstance(value, (float, np.floating)):
        return float(value).is_integer() and abs(value) <= MAX_SAFE_INTEGER
    return False


def validate_material(value, name: str) -> dict:
    """validateMaterial, layout.ts:1019-1089."""
    if not isinstance(value, dict):
        raise TypeError(f"{name} must be an object")
    lam = _finite_number(value.get("lambda"), f"{name}.lambda")
    mu = _finite_number(value.get("mu"), f"{name}.mu")
    model = normalize_mpm_constitutive_model(value.get("model"), f"{name}.model")
    if not math.isfinite(lam + 2 * mu):
        raise RangeError(f"{name} parameters are outside the supported numeric range")
    if model in ("water", "oil"):
        density = _finite_number(value.get("density"), f"{name}.density")
        eos = normalize_mpm_tait_equation_of_state(value.get("equationOfState"), f"{name}.equationOfState")
        if lam <= 0:
            raise RangeError(f"{name}.lambda must be greater than zero")
        if mu != 0:
            raise RangeError(f"{name}.mu must be zero for a liquid material")
        if value.get("frictionCoefficient") is not None:
            raise RangeError(f"{name}.frictionCoefficient is only valid for powder")
        if density <= 0:
            raise RangeError(f"{name}.density must be greater than zero")
        finite_float32(lam, f"{name}.lambda", True)
        finite_float32(mu, f"{name}.mu")
        finite_float32(density, f"{name}.density", True)
        if eos is not None:
            finite_float32(eos["exponent"], f"{name}.equationOfState.exponent", True)
        out = {"lambda": lam, "mu": 0.0, "model": model, "density": density}
        if eos is not None:
            out["equationOfState"] = eos
        return out
    if model == "powder":
        friction = _finite_number(value.get("frictionCoefficient"), f"{name}.frictionCoefficient")
        if lam < 0:
            raise RangeError(f"{name}.lambda must be non-negative")
        if mu <= 0:
            raise RangeError(f"{name}.mu must be greater than zero")
        if friction < 0:
            raise RangeError(f"{name}.frictionCoefficient must be non-negative")
        if value.get("density") is not None or value.get("equationOfState") is not None:
            raise RangeError(f"{name}.density and {name}.equationOfState are only valid for liquids")
        finite_float32(lam, f"{name}.lambda")
        finite_float32(mu, f"{name}.mu", True)
        finite_float32(friction, f"{name}.frictionCoefficient")
        return {"lambda": lam, "mu": mu, "model": model, "frictionCoefficient": friction}
    if (value.get("density") is not None or value.get("frictionCoefficient") is not None
            or value.get("equationOfState") is not None):
        raise RangeError(f"{name} has parameters that do not match its constitutive model")
    if lam < 0:
        raise RangeError(f"{name}.lambda must be non-negative")
    if mu <= 0:
        raise RangeError(f"{name}.mu must be greater than zero")
    finite_float32(lam, f"{name}.lambda")
    finite_float32(mu, f"{name}.mu", True)
    return {"lambda": lam, "mu": mu, "model": model}


@dataclass
class ParticleArrays:
    """Columnar particles.  NaN marks an absent optional value; -1 marks no
    bonded vertex and the config material."""

    px: np.ndarray
    py: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    C: np.ndarray  # (n, 4): m00, m01, m10, m11
    F: np.ndarray  # (n, 4)
    object_id: np.ndarray
    bonded_vertex: np.ndarray
    damage: np.ndarray
    plastic_volume: np.ndarray
    volume: np.ndarray
    material: np.ndarray
    materials: list = field(default_factory=list)

    def __len__(self) -> int:
        return int(self.px.shape[0])

    @staticmethod
    def empty(n: int) -> "ParticleArrays":
        return ParticleArrays(
            px=np.zeros(n), py=np.zeros(n), vx=np.zeros(n), vy=np.zeros(n),
            C=np.zeros((n, 4)), F=np.tile(np.array([1.0, 0.0, 0.0, 1.0]), (n, 1)),
            object_id=np.zeros(n, dtype=np.int64), bonded_vertex=np.full(n, -1, dtype=np.int8),
            damage=np.full(n, np.nan), plastic_volume=np.full(n, np.nan), volume=np.full(n, np.nan),
            material=np.full(n, -1, dtype=np.int32), materials=[])

    def take(self, indices) -> "ParticleArrays":
        idx = np.asarray(indices, dtype=np.int64)
        return ParticleArrays(self.px[idx], self.py[idx], self.vx[idx], self.vy[idx], self.C[idx], self.F[idx],
                              self.object_id[idx], self.bonded_vertex[idx], self.damage[idx],
                              self.plastic_volume[idx], self.volume[idx], self.material[idx], list(self.materials))

    def copy(self) -> "ParticleArrays":
        return self.take(np.arange(len(self)))


def _material_key(m: dict):
    eos = m.get("equationOfState")
    return (m.get("model"), m.get("lambda"), m.get("mu"), m.get("density"), m.get("frictionCoefficient"),
            None if eos is None else (eos.get("model"), eos.get("exponent")))


def particles_from_dicts(particles) -> ParticleArrays:
    """Columns from reference-shaped particle dicts (MpmParticle, solver.ts:29-40)."""
    if not isinstance(particles, (list, tuple)):
        raise TypeError("particles must be an array")
    n = len(particles)
    out = ParticleArrays.empty(n)
    keys = {}
    for i, p in enumerate(particles):
        if not isinstance(p, dict):
            raise TypeError(f"particles[{i}] must be an object")
        for vec, (ax, ay) in (("position", ("px", "py")), ("velocity", ("vx", "vy"))):
            v = p.get(vec)
            if not isinstance(v, dict):
                raise TypeError(f"particles[{i}].{vec} must be a vector")
            getattr(out, ax)[i] = _finite_number(v.get("x"), f"particles[{i}].{vec}.x")
            getattr(out, ay)[i] = _finite_number(v.get("y"), f"particles[{i}].{vec}.y")
        for mat_name in ("C", "F"):
            m = p.get(mat_name)
            if not isinstance(m, dict):
                raise TypeError(f"particles[{i}].{mat_name} must be a matrix")
            getattr(out, mat_name)[i] = [_finite_number(m.get(k), f"particles[{i}].{mat_name}.{k}")
                                         for k in ("m00", "m01", "m10", "m11")]
        oid = p.get("objectId")
        if oid is not None:
            if not _is_safe_integer(oid) or oid < 0 or oid > UINT32_MAX:
                raise RangeError(f"particles[{i}].objectId must be an unsigned 32-bit integer")
            out.object_id[i] = int(oid)
        bv = p.get("bondedTriangleVertex")
        if bv is not None:
            if not _is_safe_integer(bv) or bv < 0 or bv > 2:
                raise RangeError(f"particles[{i}].bondedTriangleVertex must be 0, 1, or 2")
            out.bonded_vertex[i] = int(bv)
        for key, arr in (("damage", out.damage), ("plasticVolume", out.plastic_volume), ("volume", out.volume)):
            val = p.get(key)
            if val is not None:
                arr[i] = _finite_number(val, f"particles[{i}].{key}")
        mat = p.get("material")
        if mat is not None:
            k = _material_key(mat) if isinstance(mat, dict) else id(mat)
            if k not in keys:
                keys[k] = len(out.materials)
                out.materials.append(mat)
            out.material[i] = keys[k]
    return out


def particles_to_dicts(arrays: ParticleArrays, config_material=None) -> list:
    out = []
    for i in range(len(arrays)):
        p = {
            "position": {"x": float(arrays.px[i]), "y": float(arrays.py[i])},
            "velocity": {"x": float(arrays.vx[i]), "y": float(arrays.vy[i])},
            "C": dict(zip(("m00", "m01", "m10", "m11"), map(float, arrays.C[i]))),
            "F": dict(zip(("m00", "m01", "m10", "m11"), map(float, arrays.F[i]))),
            "objectId": int(arrays.object_id[i]),
        }
        if arrays.bonded_vertex[i] >= 0:
            p["bondedTriangleVertex"] = int(arrays.bonded_vertex[i])
        if not np.isnan(arrays.damage[i]):
            p["damage"] = float(arrays.damage[i])
        if not np.isnan(arrays.plastic_volume[i]):
            p["plasticVolume"] = float(arrays.plastic_volume[i])
        if not np.isnan(arrays.volume[i]):
            p["volume"] = float(arrays.volume[i])
        if arrays.material[i] >= 0:
            p["material"] = arrays.materials[arrays.material[i]]
        elif config_material is not None:
            p["material"] = config_material
        out.append(p)
    return out


def as_particle_arrays(particles) -> ParticleArrays:
    return particles if isinstance(particles, ParticleArrays) else particles_from_dicts(particles)


@dataclass
class ValidatedInput:
    """ValidatedMpmMlsGpuInput, layout.ts:66-95."""

    config: dict
    particle_count: int
    particle_capacity: int
    packed_particles: np.ndarray  # float32 (n, 20); words 13 and 19 hold u32 bits
    packed_object_ids: np.ndarray  # uint32 (n,)
    bonded_body_starts: np.ndarray  # uint32
    packed_fracture_bonds: np.ndarray  # uint32 (nb, 6)
    packed_fracture_bond_topology: np.ndarray  # uint32
    fracture_bond_count: int
    fracture_bond_incidence_count: int
    object_ranges: list
    domain_width: float
    domain_height: float
    domain_width_f32: float
    domain_height_f32: float
    cell_size_f32: float
    particle_mass_f32: float
    particle_volume_f32: float
    bond_rest_length_f32: float
    bond_stiffness_f32: float
    bond_reference_dt_f32: float | None
    lambda_f32: float
    mu_f32: float
    wall_friction_f32: float
    gradient_scale: float
    gradient_scale_f32: float


def _first_bad(mask: np.ndarray):
    idx = np.flatnonzero(mask)
    return int(idx[0]) if idx.size else None


def validate_mpm_mls_gpu_input(particles, config: dict) -> ValidatedInput:
    """validateMpmMlsGpuInput, layout.ts:122-607."""
    if not isinstance(config, dict):
        raise TypeError("config must be an object")
    grid = config.get("grid")
    if not isinstance(grid, dict):
        raise TypeError("grid must be an object")
    material = validate_material(config.get("material"), "material")
    cells_x = _finite_number(grid.get("cellsX"), "grid.cellsX")
    cells_y = _finite_number(grid.get("cellsY"), "grid.cellsY")
    cell_size = _finite_number(grid.get("cellSize"), "grid.cellSize")
    particle_mass = _finite_number(config.get("particleMass"), "particleMass")
    particle_volume = _finite_number(config.get("particleVolume"), "particleVolume")
    bond_rest_length = None if config.get("bondRestLength") is None else _finite_number(
        config.get("bondRestLength"), "bondRestLength")
    bond_stiffness = DEFAULT_BONDED_TRIANGLE_STIFFNESS if config.get("bondStiffness") is None else _finite_number(
        config.get("bondStiffness"), "bondStiffness")
    bond_reference_dt = None if config.get("bondReferenceDt") is None else _finite_number(
        config.get("bondReferenceDt"), "bondReferenceDt")
    wall_friction = 0.0 if config.get("wallFriction") is None else _finite_number(
        config.get("wallFriction"), "wallFriction")
    lam, mu = material["lambda"], material["mu"]
    if not float(cells_x).is_integer() or cells_x < 1 or cells_x + 3 > UINT32_MAX:
        raise RangeError("grid.cellsX must be a positive safe integer that fits the GPU layout")
    if not float(cells_y).is_integer() or cells_y < 1 or cells_y + 3 > UINT32_MAX:
        raise RangeError("grid.cellsY must be a positive safe integer that fits the GPU layout")
    cells_x, cells_y = int(cells_x), int(cells_y)
    if cell_size <= 0:
        raise RangeError("grid.cellSize must be greater than zero")
    if particle_mass <= 0:
        raise RangeError("particleMass must be greater than zero")
    if particle_volume <= 0:
        raise RangeError("particleVolume must be greater than zero")
    if bond_rest_length is not None and bond_rest_length <= 0:
        raise RangeError("bondRestLength must be greater than zero")
    if bond_stiffness <= 0 or bond_stiffness > 1:
        raise RangeError("bondStiffness must be greater than zero and at most one")
    if bond_reference_dt is not None and bond_reference_dt <= 0:
        raise RangeError("bondReferenceDt must be greater than zero")
    if wall_friction < 0 or wall_friction > 1:
        raise RangeError("wallFriction must be between zero and one")
    if lam < 0:
        raise RangeError("material.lambda must be non-negative")
    if mu <= 0 and material["model"] not in ("water", "oil"):
        raise RangeError("material.mu must be greater than zero")
    domain_width = cells_x * cell_size
    domain_height = cells_y * cell_size
    cs2 = cell_size * cell_size
    gradient_scale = 4 / cs2 if cs2 > 0 else math.inf
    if not math.isfinite(domain_width) or not math.isfinite(domain_height):
        raise RangeError("grid dimensions produce a non-finite domain")
    if not math.isfinite(cs2) or cs2 <= 0 or not math.isfinite(gradient_scale):
        raise RangeError("grid.cellSize is outside the supported numeric range")
    if not math.isfinite(particle_mass / particle_volume) or particle_mass / particle_volume <= 0 or not math.isfinite(lam + 2 * mu):
        raise RangeError("mass and material parameters are outside the supported numeric range")
    cell_size_f32 = finite_float32(cell_size, "grid.cellSize", True)
    particle_mass_f32 = finite_float32(particle_mass, "particleMass", True)
    particle_volume_f32 = finite_float32(particle_volume, "particleVolume", True)
    bond_rest_length_f32 = 0.0 if bond_rest_length is None else finite_float32(bond_rest_length, "bondRestLength", True)
    bond_stiffness_f32 = finite_float32(bond_stiffness, "bondStiffness", True)
    bond_reference_dt_f32 = None if bond_reference_dt is None else finite_float32(bond_reference_dt, "bondReferenceDt", True)
    lambda_f32 = finite_float32(lam, "material.lambda")
    mu_f32 = finite_float32(mu, "material.mu", material["model"] not in ("water", "oil"))
    wall_friction_f32 = finite_float32(wall_friction, "wallFriction")
    gradient_scale_f32 = finite_float32(gradient_scale, "grid gradient scale", True)
    domain_width_f32 = finite_float32(cells_x * cell_size_f32, "GPU grid width", True)
    domain_height_f32 = finite_float32(cells_y * cell_size_f32, "GPU grid height", True)

    arrays = as_particle_arrays(particles)
    n = len(arrays)
    capacity = config.get("capacity")
    if capacity is None:
        capacity = n
    elif not _is_safe_integer(capacity) or capacity < 1:
        raise RangeError("capacity must be a positive safe integer")
    capacity = int(capacity)
    if capacity < n or capacity > UINT32_MAX:
        raise RangeError("capacity must be at least the initial particle count and fit the GPU layout")
    if capacity * 9 > INT32_MAX:
        raise RangeError("particle stencil entries exceed the linked-list index range")

    # materials of each particle (validated once per distinct material)
    mats = [validate_material(m, "particles material") for m in arrays.materials]
    all_mats = mats + [material]
    mat_index = np.where(arrays.material >= 0, arrays.material, len(mats)).astype(np.int64)
    model_of = np.array([MODEL_CODES[m["model"]] for m in all_mats], dtype=np.uint32)
    lam_of = np.array([m["lambda"] for m in all_mats])
    mu_of = np.array([m["mu"] for m in all_mats])
    is_liquid_of = np.array([m["model"] in ("water", "oil") for m in all_mats])
    density_of = np.array([m.get("density", 0.0) if m["model"] in ("water", "oil") else 0.0 for m in all_mats])
    param_of = np.array([
        m["frictionCoefficient"] if m["model"] == "powder" else
        (m["equationOfState"]["exponent"] if m["model"] in ("water", "oil") and m.get("equationOfState") else 0.0)
        for m in all_mats])
    model = model_of[mat_index]
    liquid = is_liquid_of[mat_index]

    plastic = np.where(np.isnan(arrays.plastic_volume), 1.0, arrays.plastic_volume)
    volume = np.where(np.isnan(arrays.volume), particle_volume_f32, arrays.volume)
    damage = np.where(np.isnan(arrays.damage), 0.0, arrays.damage)
    F = arrays.F
    det = F[:, 0] * F[:, 3] - F[:, 1] * F[:, 2]
    with np.errstate(over="ignore", invalid="ignore"):
        f32 = lambda a: a.astype(np.float32)  # noqa: E731
        packed = np.zeros((n, PARTICLE_FLOATS), dtype=np.float32)
        packed[:, 0] = f32(arrays.px)
        packed[:, 1] = f32(arrays.py)
        packed[:, 2] = f32(arrays.vx)
        packed[:, 3] = f32(arrays.vy)
        packed[:, 4:8] = f32(arrays.C)
        packed[:, 8:12] = f32(F)
        packed[:, 12] = f32(plastic)
        packed[:, 14] = f32(lam_of[mat_index])
        packed[:, 15] = f32(mu_of[mat_index])
        density = np.where(liquid, density_of[mat_index], 0.0)
        packed[:, 16] = f32(density)
        packed[:, 17] = f32(volume)
        param = np.where(model == MODEL_CODES["neo-hookean"], damage, param_of[mat_index])
        packed[:, 18] = f32(param)
        packed_mass = np.where(liquid, packed[:, 16] * packed[:, 17], np.float32(particle_mass_f32)).astype(np.float32)
        pdet = (packed[:, 8] * packed[:, 11]).astype(np.float32) - (packed[:, 9] * packed[:, 10]).astype(np.float32)
        pdet = pdet.astype(np.float32)

    def f32_bad(v64, v32, positive=False):
        bad = ~np.isfinite(v32) | (np.abs(v64) > MAX_FLOAT32) | ((v64 != 0) & (v32 == 0))
        if positive:
            bad |= v32 <= 0
        return bad

    bad = np.zeros(n, dtype=bool)
    bad |= (volume <= 0) | (damage < 0) | (damage > 1)
    bad |= ~np.isnan(arrays.damage) & (model != MODEL_CODES["neo-hookean"])
    bad |= (plastic < SNOW_PLASTICITY["minPlasticVolume"]) | (plastic > SNOW_PLASTICITY["maxPlasticVolume"])
    bad |= (arrays.px < 0) | (arrays.px > domain_width) | (arrays.py < 0) | (arrays.py > domain_height)
    bad |= ~np.isfinite(det) | (det <= 0)
    for col, v64 in ((0, arrays.px), (1, arrays.py), (2, arrays.vx), (3, arrays.vy)):
        bad |= f32_bad(v64, packed[:, col])
    for k in range(4):
        bad |= f32_bad(arrays.C[:, k], packed[:, 4 + k]) | f32_bad(F[:, k], packed[:, 8 + k])
    bad |= f32_bad(plastic, packed[:, 12], True) | f32_bad(volume, packed[:, 17], True)
    bad |= liquid & f32_bad(density, packed[:, 16], True)
    bad |= f32_bad(param, packed[:, 18])
    bad |= ~np.isfinite(packed_mass) | (packed_mass <= 0)
    bad |= ~np.isfinite(pdet) | (pdet <= 0)
    bad |= (packed[:, 0] < 0) | (packed[:, 0] > domain_width_f32) | (packed[:, 1] < 0) | (packed[:, 1] > domain_height_f32)
    first = _first_bad(bad)
    if first is not None:
        _raise_particle_error(first, arrays, all_mats[mat_index[first]], particle_volume_f32, particle_mass_f32,
                              domain_width, domain_height, domain_width_f32, domain_height_f32)

    words = packed.view(np.uint32)
    words[:, 13] = model
    words[:, 19] = np.where(arrays.bonded_vertex >= 0, arrays.bonded_vertex.astype(np.int64) + 1, 0).astype(np.uint32)
    object_ids = arrays.object_id.astype(np.uint32)

    # object ranges must be contiguous (layout.ts:440-454)
    object_ranges = []
    if n:
        change = np.flatnonzero(np.diff(arrays.object_id) != 0) + 1
        starts = np.concatenate(([0], change))
        ends = np.concatenate((change, [n]))
        seen = set()
        for s, e in zip(starts, ends):
            oid = int(arrays.object_id[s])
            if oid in seen:
                raise RangeError(f"particles with objectId {oid} must be contiguous for GPU cloning")
            seen.add(oid)
            object_ranges.append({"objectId": oid, "start": int(s), "count": int(e - s)})

    # bonded triangle bodies (layout.ts:457-496)
    body_starts = []
    for rng in object_ranges:
        seg = arrays.bonded_vertex[rng["start"]:rng["start"] + rng["count"]]
        if not np.any(seg >= 0):
            continue
        if bond_rest_length is None:
            raise RangeError(f"object {rng['objectId']} uses bonded triangles but bondRestLength is missing")
        if rng["count"] % 3 != 0:
            raise RangeError(f"bonded object {rng['objectId']} must contain complete three-particle triangles")
        expected = np.arange(rng["count"]) % 3
        if np.any(seg != expected):
            raise RangeError(f"bonded object {rng['objectId']} must store contiguous vertices 0, 1, and 2")
        if np.any(liquid[rng["start"]:rng["start"] + rng["count"]]):
            raise RangeError("bonded triangle vertices must use a solid material")
        body_starts.extend(range(rng["start"], rng["start"] + rng["count"], 3))
    if body_starts and bond_rest_length_f32 <= 0:
        raise RangeError("bondRestLength must remain positive in float32")

    bonds = config.get("fractureBonds") or []
    fb_packed, topology = pack_fracture_bonds(bonds, arrays, model, n)

    validated_config = {
        "grid": {"cellsX": cells_x, "cellsY": cells_y, "cellSize": cell_size},
        "particleMass": particle_mass,
        "particleVolume": particle_volume,
        "bondStiffness": bond_stiffness,
        "material": material,
        "wallFriction": wall_friction,
        "capacity": capacity,
    }
    if bond_rest_length is not None:
        validated_config["bondRestLength"] = bond_rest_length
    if bond_reference_dt is not None:
        validated_config["bondReferenceDt"] = bond_reference_dt
    if config.get("fractureBonds") is not None:
        validated_config["fractureBonds"] = bonds
    return ValidatedInput(
        config=validated_config, particle_count=n, particle_capacity=capacity, packed_particles=packed,
        packed_object_ids=object_ids, bonded_body_starts=np.asarray(body_starts, dtype=np.uint32),
        packed_fracture_bonds=fb_packed, packed_fracture_bond_topology=topology,
        fracture_bond_count=len(bonds), fracture_bond_incidence_count=2 * len(bonds), object_ranges=object_ranges,
        domain_width=domain_width, domain_height=domain_height, domain_width_f32=domain_width_f32,
        domain_height_f32=domain_height_f32, cell_size_f32=cell_size_f32, particle_mass_f32=particle_mass_f32,
        particle_volume_f32=particle_volume_f32, bond_rest_length_f32=bond_rest_length_f32,
        bond_stiffness_f32=bond_stiffness_f32, bond_reference_dt_f32=bond_reference_dt_f32, lambda_f32=lambda_f32,
        mu_f32=mu_f32, wall_friction_f32=wall_friction_f32, gradient_scale=gradient_scale,
        gradient_scale_f32=gradient_scale_f32)


def _raise_particle_error(i, a: ParticleArrays, m, pv32, pm32, dw, dh, dw32, dh32):
    """Re-checks particle i in the order of layout.ts:284-438."""
    plastic = 1.0 if np.isnan(a.plastic_volume[i]) else float(a.plastic_volume[i])
    volume = pv32 if np.isnan(a.volume[i]) else float(a.volume[i])
    damage = 0.0 if np.isnan(a.damage[i]) else float(a.damage[i])
    if volume <= 0:
        raise RangeError(f"particles[{i}].volume must be greater than zero")
    if damage < 0 or damage > 1:
        raise RangeError(f"particles[{i}].damage must be between zero and one")
    if not np.isnan(a.damage[i]) and m["model"] != "neo-hookean":
        raise RangeError(f"particles[{i}].damage is only valid for neo-hookean solids")
    if plastic < SNOW_PLASTICITY["minPlasticVolume"] or plastic > SNOW_PLASTICITY["maxPlasticVolume"]:
        raise RangeError(f"particles[{i}].plasticVolume must be between 0.6 and 20")
    if a.px[i] < 0 or a.px[i] > dw or a.py[i] < 0 or a.py[i] > dh:
        raise RangeError(f"particles[{i}].position must be inside the grid domain")
    F = a.F[i]
    det = F[0] * F[3] - F[1] * F[2]
    if not math.isfinite(det) or det <= 0:
        raise RangeError(f"particles[{i}].F must have a finite positive determinant")
    liquid = m["model"] in ("water", "oil")
    density = m.get("density", 0.0) if liquid else 0.0
    param = (m["frictionCoefficient"] if m["model"] == "powder" else damage if m["model"] == "neo-hookean"
             else (m["equationOfState"]["exponent"] if liquid and m.get("equationOfState") else 0.0))
    vals = [finite_float32(a.px[i], f"particles[{i}].position.x"), finite_float32(a.py[i], f"particles[{i}].position.y"),
            finite_float32(a.vx[i], f"particles[{i}].velocity.x"), finite_float32(a.vy[i], f"particles[{i}].velocity.y")]
    for k, key in enumerate(("m00", "m01", "m10", "m11")):
        finite_float32(a.C[i, k], f"particles[{i}].C.{key}")
    f32F = [finite_float32(a.F[i, k], f"particles[{i}].F.{key}") for k, key in enumerate(("m00", "m01", "m10", "m11"))]
    finite_float32(plastic, f"particles[{i}].plasticVolume", True)
    finite_float32(m["lambda"], f"particles[{i}].material.lambda")
    finite_float32(m["mu"], f"particles[{i}].material.mu", not liquid)
    pd = finite_float32(density, f"particles[{i}].material.density", liquid)
    pvol = finite_float32(volume, f"particles[{i}].volume", True)
    finite_float32(param, f"particles[{i}].material parameter")
    mass = fround(pd * pvol) if liquid else pm32
    if not math.isfinite(mass) or mass <= 0:
        raise RangeError(f"particles[{i}] mass is outside the supported float32 range")
    pdet = fround(fround(f32F[0] * f32F[3]) - fround(f32F[1] * f32F[2]))
    if not math.isfinite(pdet) or pdet <= 0:
        raise RangeError(f"particles[{i}].F must retain a finite positive determinant in float32")
    if vals[0] < 0 or vals[0] > dw32 or vals[1] < 0 or vals[1] > dh32:
        raise RangeError(f"particles[{i}].position is outside the float32 GPU grid domain")
    raise RangeError(f"particles[{i}] is outside the supported float32 range")


def pack_fracture_bonds(bonds, arrays: ParticleArrays, model: np.ndarray, n: int):
    """Fracture bond graph validation (src/lib/mpm/reference/solid-bonds.ts:12-70)
    and packing (layout.ts:498-564): 6 words per bond and CSR incidence."""
    if not isinstance(bonds, (list, tuple)):
        raise TypeError("fractureBonds must be an array")
    nb = len(bonds)
    packed = np.zeros((nb, 6), dtype=np.uint32)
    floats = packed.view(np.float32)
    seen = set()
    offsets = np.zeros(n + 1, dtype=np.int64)
    for b, bond in enumerate(bonds):
        if not isinstance(bond, dict):
            raise TypeError(f"fractureBonds[{b}] must be an object")
        for key in ("firstParticle", "secondParticle"):
            v = bond.get(key)
            if not _is_safe_integer(v) or v < 0 or v >= n:
                raise RangeError(f"fractureBonds[{b}].{key} must identify an existing particle")
        first, second = int(bond["firstParticle"]), int(bond["secondParticle"])
        if first == second:
            raise RangeError(f"fractureBonds[{b}] must connect two distinct particles")
        rest, strain = bond.get("restLength"), bond.get("failureStrain")
        if not isinstance(rest, (int, float)) or not math.isfinite(rest) or rest <= 0:
            raise RangeError(f"fractureBonds[{b}].restLength must be positive and finite")
        if not isinstance(strain, (int, float)) or not math.isfinite(strain) or strain <= 0:
            raise RangeError(f"fractureBonds[{b}].failureStrain must be positive and finite")
        damage = bond.get("damage", 0.0) or 0.0
        if not math.isfinite(damage) or damage < 0 or damage > 1:
            raise RangeError(f"fractureBonds[{b}].damage must be between zero and one")
        broken = bond.get("broken")
        if broken is not None and not isinstance(broken, bool):
            raise TypeError(f"fractureBonds[{b}].broken must be a boolean")
        if arrays.object_id[first] != arrays.object_id[second]:
            raise RangeError(f"fractureBonds[{b}] must connect particles of one object")
        if arrays.bonded_vertex[first] >= 0 or arrays.bonded_vertex[second] >= 0:
            raise RangeError(f"fractureBonds[{b}] cannot reuse bonded triangle vertices")
        if model[first] != 0 or model[second] != 0:
            raise RangeError(f"fractureBonds[{b}] endpoints must be neo-hookean solids")
        pair = (min(first, second), max(first, second))
        if pair in seen:
            raise RangeError(f"fractureBonds[{b}] duplicates an existing particle pair")
        seen.add(pair)
        packed[b, 0], packed[b, 1] = first, second
        floats[b, 2] = finite_float32(rest, f"fractureBonds[{b}].restLength", True)
        floats[b, 3] = finite_float32(strain, f"fractureBonds[{b}].failureStrain", True)
        floats[b, 4] = finite_float32(1.0 if broken else damage, f"fractureBonds[{b}].damage")
        packed[b, 5] = 1 if broken else 0
        offsets[first + 1] += 1
        offsets[second + 1] += 1
    if nb == 0:
        return packed, np.zeros(0, dtype=np.uint32)
    offsets = np.cumsum(offsets)
    topology = np.zeros(n + 1 + 2 * nb, dtype=np.uint32)
    topology[:n + 1] = offsets
    cursors = offsets[:n].copy()
    for b, bond in enumerate(bonds):
        for end in (int(bond["firstParticle"]), int(bond["secondParticle"])):
            topology[n + 1 + cursors[end]] = b
            cursors[end] += 1
    return packed, topology


def unpack_particles(packed: np.ndarray, object_ids: np.ndarray) -> list:
    """unpackParticles, src/lib/mpm/kernels/solver.ts:3148-3226."""
    from .materials import decode_mpm_constitutive_model
    words = packed.view(np.uint32)
    out = []
    for i in range(packed.shape[0]):
        if words[i, 13] == UINT32_MAX:
            continue
        model = decode_mpm_constitutive_model(int(words[i, 13]))
        marker = int(words[i, 19])
        if marker > 3:
            raise RangeError(f"GPU particle {i} has an invalid bonded triangle marker.")
        v = [float(x) for x in packed[i]]
        if model in ("water", "oil"):
            material = {"model": model, "lambda": v[14], "mu": 0.0, "density": v[16]}
            if v[18] > 0:
                material["equationOfState"] = {"model": "tait", "exponent": v[18]}
        elif model == "powder":
            material = {"model": model, "lambda": v[14], "mu": v[15], "frictionCoefficient": v[18]}
        else:
            material = {"model": model, "lambda": v[14], "mu": v[15]}
        p = {
            "position": {"x": v[0], "y": v[1]},
            "velocity": {"x": v[2], "y": v[3]},
            "C": {"m00": v[4], "m01": v[5], "m10": v[6], "m11": v[7]},
            "F": {"m00": v[8], "m01": v[9], "m10": v[10], "m11": v[11]},
            "plasticVolume": v[12],
            "volume": v[17],
            "material": material,
            "objectId": int(object_ids[i]),
        }
        if model == "neo-hookean" and v[18] > 0:
            p["damage"] = v[18]
        if marker:
            p["bondedTriangleVertex"] = marker - 1
        out.append(p)
    return out


def pack_step_parameters(state: ValidatedInput, dt: float, gravity: dict, cfl_guard=None, bond_reference_dt=None):
    """The checks of packMpmMlsGpuStepParameters (layout.ts:896-949).  Returns
    the float32 values the C ABI receives."""
    step_dt = _finite_number(dt, "dt")
    if step_dt <= 0:
        raise RangeError("dt must be greater than zero")
    dt32 = finite_float32(step_dt, "dt", True)
    if not isinstance(gravity, dict):
        raise TypeError("gravity must be an object")
    gx = finite_float32(_finite_number(gravity.get("x"), "gravity.x"), "gravity.x")
    gy = finite_float32(_finite_number(gravity.get("y"), "gravity.y"), "gravity.y")
    wave = velocity = 0.0
    if cfl_guard is not None:
        wave = finite_float32(cfl_guard["waveSpeedBound"], "cflGuard.waveSpeedBound")
        velocity = finite_float32(cfl_guard["velocityBound"], "cflGuard.velocityBound")
    bref = finite_float32(bond_reference_dt if bond_reference_dt is not None else (
        state.bond_reference_dt_f32 if state.bond_reference_dt_f32 is not None else dt32), "bondReferenceDt", True)
    stress_scale = -step_dt * state.config["particleVolume"] * state.gradient_scale
    if not math.isfinite(stress_scale):
        raise RangeError("dt, particleVolume, and grid.cellSize produce a non-finite stress scale")
    finite_float32(stress_scale, "stress scale")
    return dt32, gx, gy, wave, velocity, bref
