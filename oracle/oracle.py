"""ctypes wrapper of the FP64 CPU oracle (oracle/libmpm_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker.  The product path never imports
this module.  The oracle restates src/lib/mpm/reference/solver.ts `stepMpm`
of 7korobi/powder-play (see oracle/mpm_oracle.h for the citation map).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "libmpm_oracle.so")

MODEL_CODES = {"neo-hookean": 0, "snow": 1, "water": 2, "oil": 3, "powder": 4, "fixed-corotated": 5}

PARTICLE_DTYPE = np.dtype([
    ("px", "f8"), ("py", "f8"), ("vx", "f8"), ("vy", "f8"),
    ("c00", "f8"), ("c01", "f8"), ("c10", "f8"), ("c11", "f8"),
    ("f00", "f8"), ("f01", "f8"), ("f10", "f8"), ("f11", "f8"),
    ("damage", "f8"), ("plastic_volume", "f8"), ("volume", "f8"),
    ("material", "i4"), ("object_id", "i4"), ("bonded_vertex", "i4"), ("has_damage", "i4"),
], align=True)
MATERIAL_DTYPE = np.dtype([
    ("model", "i4"), ("tait", "i4"), ("lambda_", "f8"), ("mu", "f8"), ("density", "f8"), ("friction", "f8"),
    ("exponent", "f8"),
], align=True)
BOND_DTYPE = np.dtype([
    ("first", "i4"), ("second", "i4"), ("rest_length", "f8"), ("failure_strain", "f8"), ("damage", "f8"),
    ("broken", "i4"), ("pad", "i4"),
], align=True)


class OrcConfig(ctypes.Structure):
    _fields_ = [
        ("dt", ctypes.c_double), ("cells_x", ctypes.c_int32), ("cells_y", ctypes.c_int32),
        ("cell_size", ctypes.c_double), ("particle_mass", ctypes.c_double), ("particle_volume", ctypes.c_double),
        ("has_bond_rest_length", ctypes.c_int32), ("material", ctypes.c_int32),
        ("bond_rest_length", ctypes.c_double), ("bond_stiffness", ctypes.c_double),
        ("bond_reference_dt", ctypes.c_double), ("gx", ctypes.c_double), ("gy", ctypes.c_double),
        ("wall_friction", ctypes.c_double), ("n_bonds", ctypes.c_int32), ("has_fracture_bonds", ctypes.c_int32),
    ]


class OrcDiag(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in (
        "input_mass", "grid_mass", "output_mass", "input_mx", "input_my", "grid_mx", "grid_my", "output_mx",
        "output_my")]


class OrcAdjScene(ctypes.Structure):
    _fields_ = [("cells_x", ctypes.c_int32), ("cells_y", ctypes.c_int32)] + [
        (k, ctypes.c_double) for k in ("dx", "dt", "gx", "gy", "solid_mass", "wall_friction", "rho", "gamma", "tait",
                                       "lambda_s", "mu_s")]


class OracleError(ValueError):
    """A RangeError/TypeError raised by the restated reference step."""


_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIBRARY


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBRARY):
        build()
    lib = ctypes.CDLL(LIBRARY)
    vp = ctypes.c_void_p
    lib.orc_step.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(OrcConfig), vp, vp, ctypes.c_int32, vp, vp,
                             ctypes.POINTER(OrcDiag), ctypes.c_char_p, ctypes.c_int32]
    lib.orc_step.restype = ctypes.c_int
    lib.orc_run.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(OrcConfig), vp, ctypes.c_int32, vp, ctypes.c_int32,
                            ctypes.c_char_p, ctypes.c_int32]
    lib.orc_run.restype = ctypes.c_int32
    lib.orc_triangle_field.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(OrcConfig), vp, ctypes.c_int32, vp, vp, vp,
                                       vp, ctypes.c_char_p, ctypes.c_int32]
    lib.orc_triangle_field.restype = ctypes.c_int
    lib.emu_fixed_point_scatter.argtypes = [ctypes.c_int32] + [vp] * 7 + [ctypes.c_float] * 3 + [ctypes.c_int32] * 3 + [vp]
    lib.emu_fixed_point_scatter.restype = ctypes.c_uint32
    lib.orc_adjoint_run.argtypes = [ctypes.POINTER(OrcAdjScene), ctypes.c_int32] + [vp] * 7 + [ctypes.c_int32] + [vp] * 4
    lib.orc_adjoint_run.restype = ctypes.c_int
    for name in ("orc_sizeof_particle", "orc_sizeof_material", "orc_sizeof_bond", "orc_sizeof_config"):
        getattr(lib, name).restype = ctypes.c_int32
    assert lib.orc_sizeof_particle() == PARTICLE_DTYPE.itemsize
    assert lib.orc_sizeof_material() == MATERIAL_DTYPE.itemsize
    assert lib.orc_sizeof_bond() == BOND_DTYPE.itemsize
    assert lib.orc_sizeof_config() == ctypes.sizeof(OrcConfig)
    _lib = lib
    return lib


def _material_record(m: dict):
    rec = np.zeros((), dtype=MATERIAL_DTYPE)
    rec["model"] = MODEL_CODES[m.get("model") or "neo-hookean"]
    rec["lambda_"] = m["lambda"]
    rec["mu"] = m.get("mu", 0.0)
    rec["density"] = m.get("density", 0.0)
    rec["friction"] = m.get("frictionCoefficient", 0.0)
    eos = m.get("equationOfState")
    if eos:
        rec["tait"] = 1
        rec["exponent"] = eos["exponent"]
    return rec


class OracleState:
    """Particles and materials in oracle layout, built from a ParticleArrays
    (powder-play_b200/mpm_b200/layout.py) and a step config dict."""

    def __init__(self, arrays, config: dict):
        self.materials = list(arrays.materials) + [config["material"]]
        self.mats = np.array([_material_record(m) for m in self.materials], dtype=MATERIAL_DTYPE)
        self.default_material = len(self.materials) - 1
        n = len(arrays)
        p = np.zeros(n, dtype=PARTICLE_DTYPE)
        p["px"], p["py"], p["vx"], p["vy"] = arrays.px, arrays.py, arrays.vx, arrays.vy
        for k, name in enumerate(("c00", "c01", "c10", "c11")):
            p[name] = arrays.C[:, k]
        for k, name in enumerate(("f00", "f01", "f10", "f11")):
            p[name] = arrays.F[:, k]
        p["has_damage"] = ~np.isnan(arrays.damage)
        p["damage"] = np.nan_to_num(arrays.damage, nan=0.0)
        p["plastic_volume"] = np.nan_to_num(arrays.plastic_volume, nan=1.0)
        p["volume"] = np.nan_to_num(arrays.volume, nan=0.0)
        p["material"] = arrays.material
        p["object_id"] = arrays.object_id.astype(np.int32)
        p["bonded_vertex"] = arrays.bonded_vertex.astype(np.int32)
        self.particles = p
        bonds = config.get("fractureBonds")
        self.has_bonds = bonds is not None
        self.bonds = np.zeros(len(bonds or []), dtype=BOND_DTYPE)
        for b, bond in enumerate(bonds or []):
            self.bonds[b] = (bond["firstParticle"], bond["secondParticle"], bond["restLength"],
                             bond["failureStrain"], 1.0 if bond.get("broken") else bond.get("damage", 0.0) or 0.0,
                             1 if bond.get("broken") else 0, 0)

    def config_struct(self, config: dict) -> OrcConfig:
        c = OrcConfig()
        c.dt = config["dt"]
        c.cells_x = int(config["grid"]["cellsX"])
        c.cells_y = int(config["grid"]["cellsY"])
        c.cell_size = config["grid"]["cellSize"]
        c.particle_mass = config["particleMass"]
        c.particle_volume = config["particleVolume"]
        c.has_bond_rest_length = 1 if config.get("bondRestLength") is not None else 0
        c.bond_rest_length = config.get("bondRestLength") or 0.0
        c.bond_stiffness = 0.35 if config.get("bondStiffness") is None else config["bondStiffness"]
        c.bond_reference_dt = config.get("bondReferenceDt") or 0.0
        c.material = self.default_material
        c.gx = config["gravity"]["x"]
        c.gy = config["gravity"]["y"]
        c.wall_friction = config.get("wallFriction") or 0.0
        c.n_bonds = len(self.bonds)
        c.has_fracture_bonds = 1 if self.has_bonds else 0
        return c

    def step(self, config: dict) -> dict:
        """One stepMpm; updates the state in place and returns diagnostics."""
        lib = load()
        c = self.config_struct(config)
        out = np.zeros_like(self.particles)
        bonds_out = self.bonds.copy()
        diag = OrcDiag()
        err = ctypes.create_string_buffer(512)
        rc = lib.orc_step(self.mats.ctypes.data, len(self.mats), ctypes.byref(c), self.particles.ctypes.data,
                          out.ctypes.data, len(self.particles), self.bonds.ctypes.data if len(self.bonds) else None,
                          bonds_out.ctypes.data if len(self.bonds) else None, ctypes.byref(diag), err, 512)
        if rc != 0:
            raise OracleError(err.value.decode())
        self.particles = out
        self.bonds = bonds_out
        return {k: getattr(diag, k) for k, _ in OrcDiag._fields_}

    def run(self, config: dict, steps: int) -> int:
        lib = load()
        c = self.config_struct(config)
        err = ctypes.create_string_buffer(512)
        done = lib.orc_run(self.mats.ctypes.data, len(self.mats), ctypes.byref(c), self.particles.ctypes.data,
                           len(self.particles), self.bonds.ctypes.data if len(self.bonds) else None, steps, err, 512)
        if done != steps:
            raise OracleError(err.value.decode())
        return done

    def triangle_field(self, config: dict) -> dict:
        """The bonded-triangle field of the current particles, dense over the
        halo nodes: sd, body (first-vertex index, -1: none), normal, bary."""
        lib = load()
        c = self.config_struct(config)
        h, w = int(config["grid"]["cellsY"]) + 3, int(config["grid"]["cellsX"]) + 3
        sd = np.zeros(h * w)
        body = np.zeros(h * w, dtype=np.int32)
        normal = np.zeros((h * w, 2))
        bary = np.zeros((h * w, 3))
        err = ctypes.create_string_buffer(512)
        rc = lib.orc_triangle_field(self.mats.ctypes.data, len(self.mats), ctypes.byref(c),
                                    self.particles.ctypes.data, len(self.particles), sd.ctypes.data,
                                    body.ctypes.data, normal.ctypes.data, bary.ctypes.data, err, 512)
        if rc != 0:
            raise OracleError(err.value.decode())
        return {"sd": sd.reshape(h, w), "body": body.reshape(h, w), "normal": normal.reshape(h, w, 2),
                "bary": bary.reshape(h, w, 3)}

    def positions(self) -> np.ndarray:
        return np.stack([self.particles["px"], self.particles["py"]], axis=1)

    def velocities(self) -> np.ndarray:
        return np.stack([self.particles["vx"], self.particles["vy"]], axis=1)

    def affine(self) -> np.ndarray:
        return np.stack([self.particles[k] for k in ("c00", "c01", "c10", "c11")], axis=1)

    def deformation(self) -> np.ndarray:
        return np.stack([self.particles[k] for k in ("f00", "f01", "f10", "f11")], axis=1)


def emulate_fixed_point_scatter(packed: np.ndarray, affine: np.ndarray, cell_size: float, particle_mass: float,
                                particle_volume: float, cells_x: int, cells_y: int, shift: int = 24):
    """Integer words (node_count, 11) of the fixed-point scatter for 20-word
    packed records and the GPU's prepared affines, plus the range flags."""
    lib = load()
    packed = np.ascontiguousarray(packed, dtype=np.float32)
    n = packed.shape[0]
    pos = np.ascontiguousarray(packed[:, 0:2])
    vel = np.ascontiguousarray(packed[:, 2:4])
    F = np.ascontiguousarray(packed[:, 8:12])
    vol = np.ascontiguousarray(packed[:, 17])
    model = np.ascontiguousarray(packed.view(np.uint32)[:, 13])
    density = np.ascontiguousarray(packed[:, 16])
    aff = np.ascontiguousarray(affine, dtype=np.float32)
    words = np.zeros(((cells_x + 3) * (cells_y + 3), 11), dtype=np.int32)
    flags = lib.emu_fixed_point_scatter(n, pos.ctypes.data, vel.ctypes.data, F.ctypes.data, vol.ctypes.data,
                                        model.ctypes.data, density.ctypes.data, aff.ctypes.data, cell_size,
                                        particle_mass, particle_volume, cells_x, cells_y, shift, words.ctypes.data)
    return words, int(flags)


def packed_state(packed: np.ndarray) -> dict:
    """Splits 20-word GPU records into float64 columns for comparisons."""
    p = packed.astype(np.float64)
    return {"position": p[:, 0:2], "velocity": p[:, 2:4], "C": p[:, 4:8], "F": p[:, 8:12], "plastic": p[:, 12]}


def js_hypot(x, y):
    return math.hypot(x, y)


def adjoint_fp64(scene: dict, x0, v0, C0, F0, vol, liquid, target, steps: int):
    """The FP64 adjoint of the differentiable form (oracle/adjoint_fp64.c) for
    one scene: returns (loss, gradient wrt v0 (n, 2), gradient wrt (tait,
    lambda_s, mu_s), x(T) (n, 2))."""
    lib = load()
    s = OrcAdjScene(**scene)
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
    x0, v0, C0, F0, vol, target = map(f64, (x0, v0, C0, F0, vol, target))
    liquid = np.ascontiguousarray(liquid, dtype=np.int32)
    n = len(vol)
    loss = ctypes.c_double()
    gv = np.zeros((n, 2), dtype=np.float64)
    gp = np.zeros(3, dtype=np.float64)
    xt = np.zeros((n, 2), dtype=np.float64)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    rc = lib.orc_adjoint_run(ctypes.byref(s), n, p(x0), p(v0), p(C0), p(F0), p(vol), p(liquid), p(target), steps,
                             ctypes.byref(loss), p(gv), p(gp), p(xt))
    if rc != 0:
        raise OracleError(f"the FP64 adjoint stopped ({rc})")
    return loss.value, gv, gp, xt



def current_area_fp64(px, py, F, volume, phase, cells_x: int, cells_y: int, cell_size: float) -> np.ndarray:
    """FP64 restatement of gatherCurrentArea (src/lib/mpm/reference/occupancy.ts:70-128,
    particleStencil / quadraticWeights :283-303) on a dense halo field.

    phase: 0 water, 1 oil, anything else ignored (occupancy.ts:223).  Returns
    (cells_y + 3, cells_x + 3, 2): node (x, y) at [y + 1, x + 1], its water
    and oil current area V det(F) w / cellSize^2, added particle by particle
    in stencil order (oy, then ox) like the reference's loop.  The GPU field
    of gatherSurfaceOccupancy (shaders.ts:770-772) is the display area, twice
    this.  Raises OracleError for the inputs the reference rejects
    (occupancy.ts:178-230)."""
    px = np.asarray(px, np.float64)
    py = np.asarray(py, np.float64)
    F = np.asarray(F, np.float64).reshape(-1, 4)
    volume = np.asarray(volume, np.float64)
    phase = np.asarray(phase)
    if not (cell_size > 0):
        raise OracleError("grid.cellSize must be greater than zero")
    width, height = cells_x * cell_size, cells_y * cell_size
    if np.any((px < 0) | (px > width) | (py < 0) | (py > height)):
        raise OracleError("position must be inside the grid domain")
    jac = F[:, 0] * F[:, 3] - F[:, 1] * F[:, 2]
    if np.any(~np.isfinite(jac) | (jac <= 0)):
        raise OracleError("F must have a finite positive determinant")
    liquid = (phase == 0) | (phase == 1)
    area = volume * jac
    field = np.zeros(((cells_y + 3) * (cells_x + 3), 2), np.float64)
    if not np.any(liquid):
        return field.reshape(cells_y + 3, cells_x + 3, 2)
    gx, gy = px[liquid] / cell_size, py[liquid] / cell_size
    bx, by = np.floor(gx - 0.5), np.floor(gy - 0.5)
    fx, fy = gx - bx, gy - by

    def weights(f):
        return np.stack([0.5 * (1.5 - f) ** 2, 0.75 - (f - 1) ** 2, 0.5 * (f - 0.5) ** 2], axis=1)

    wx, wy = weights(fx), weights(fy)
    cell_area = cell_size * cell_size
    node_w = cells_x + 3
    index, value = [], []
    for oy in range(3):
        for ox in range(3):
            index.append((by + oy + 1) * node_w + (bx + ox + 1))
            value.append(wx[:, ox] * wy[:, oy] * area[liquid] / cell_area)
    index = np.stack(index, axis=1).astype(np.int64)  # particle-major, then oy, ox
    value = np.stack(value, axis=1)
    channel = np.repeat(phase[liquid].astype(np.int64)[:, None], 9, axis=1)
    np.add.at(field, (index.ravel(), channel.ravel()), value.ravel())
    return field.reshape(cells_y + 3, cells_x + 3, 2)
