"""Scenes of the reference and the seeded synthetic workloads built on them.

* `create_si_fluid_scene` -- src/lib/mpm/scenes/si-fluid.ts:39-79 (the
  reference SI Tait water tank, 1,600 particles on a 40x40 grid).
* `create_si_tank_scene` -- the 1,600-particle SI tank on an 80x80 grid with
  seeded jitter (40x40 lattice at 1.25 mm in a 50 mm block, Tait gamma 7,
  c = 20 m/s, y-up gravity).
* `create_mpm_gate4_scene` / `create_mpm_gate4_step_config` --
  src/lib/mpm/scenes/gate4.ts:134-357 (LCG seeds, draw order, bonds).
* `create_dam_break_scene` -- the 1,000,000-particle two-phase water/oil dam
  break on a 1024x2048 grid (cellSize 10, gravity 90, Gate-4 liquids).
* `create_mpm_emitter_particles` -- src/lib/mpm/scenes/emitter.ts:49-129 (the
  particles of an interactive emitter batch).
* `create_batched_tank_scenes` -- independent SI Tait water tanks of uneven
  particle counts and grids for the batched solver.
* `create_adjoint_scenes` -- water + fixed-corotated solid scenes, their
  initial velocities and target displacement fields for the differentiable
  form.

All seeded randomness uses the reference's LCG (gate4.ts:134-144) so that a
seed names the same scene in every language.
"""
from __future__ import annotations

import math

import numpy as np

from .errors import RangeError
from .layout import ParticleArrays
from .materials import MPM_SI_BOX_DOMAIN
from .tait_eos import create_mpm_tait_liquid_material, derive_tait_pressure_coefficient_pa

UINT32_RANGE = 0x1_0000_0000


class SeededRandom:
    """createSeededRandom, gate4.ts:134-144 (Numerical Recipes LCG)."""

    def __init__(self, seed: int):
        if not isinstance(seed, int) or seed < 0 or seed >= UINT32_RANGE:
            raise ValueError("The scene seed must be an unsigned 32-bit integer.")
        self.state = seed

    def __call__(self) -> float:
        self.state = (self.state * 1_664_525 + 1_013_904_223) & 0xFFFFFFFF
        return self.state / UINT32_RANGE

    def many(self, count: int) -> np.ndarray:
        return np.array([self() for _ in range(count)], dtype=np.float64)


def lcg_sequence(seed: int, count: int) -> np.ndarray:
    """`count` successive LCG draws, vectorised by jumping the recurrence a
    block at a time (all products fit in uint64 before the mod 2^32)."""
    a, c, m = 1_664_525, 1_013_904_223, 1 << 32
    block = 1 << 12
    mults = np.empty(block, dtype=np.uint64)
    adds = np.empty(block, dtype=np.uint64)
    am, ad = 1, 0
    for k in range(block):
        am, ad = (am * a) % m, (ad * a + c) % m
        mults[k], adds[k] = am, ad
    out = np.empty(count, dtype=np.float64)
    state = np.uint64(seed)
    for start in range(0, count, block):
        n = min(block, count - start)
        states = (mults[:n] * state + adds[:n]) % np.uint64(m)
        out[start:start + n] = states.astype(np.float64) / UINT32_RANGE
        state = states[n - 1]
    return out


SI_FLUID_GRID_CELLS = 40
SI_FLUID_PARTICLE_SPACING_M = 0.0025
SI_FLUID_FILL_HEIGHT_M = 0.05
SI_FLUID_EFFECTIVE_SOUND_SPEED_M_PER_S = 20.0
SI_FLUID_COURANT_LIMIT = 0.3
SI_FLUID_FIXED_STEP_SECONDS = 1 / 120
SI_FLUID_MAX_MICROSTEPS_PER_BATCH = 512
SI_FLUID_WALL_FRICTION = 1.0
SI_TAIT_WATER_PARAMETERS = {
    "referenceDensityKgPerM3": 998.2,
    "exponent": 7.15,
    "pressureCoefficientPa": derive_tait_pressure_coefficient_pa(998.2, 7.15, SI_FLUID_EFFECTIVE_SOUND_SPEED_M_PER_S),
    "ambientPressurePa": 101_325.0,
}


def create_si_fluid_scene():
    """createSiFluidScene, si-fluid.ts:39-79 -> (ParticleArrays, config)."""
    material = create_mpm_tait_liquid_material(SI_TAIT_WATER_PARAMETERS, MPM_SI_BOX_DOMAIN["extrusionDepthM"])
    area = SI_FLUID_PARTICLE_SPACING_M ** 2
    columns = math.floor(MPM_SI_BOX_DOMAIN["innerWidthM"] / SI_FLUID_PARTICLE_SPACING_M)
    rows = math.floor(SI_FLUID_FILL_HEIGHT_M / SI_FLUID_PARTICLE_SPACING_M)
    n = rows * columns
    p = ParticleArrays.empty(n)
    r, c = np.divmod(np.arange(n), columns)
    p.px[:] = (c + 0.5) * SI_FLUID_PARTICLE_SPACING_M
    p.py[:] = MPM_SI_BOX_DOMAIN["innerHeightM"] - SI_FLUID_FILL_HEIGHT_M + (r + 0.5) * SI_FLUID_PARTICLE_SPACING_M
    p.volume[:] = area
    grid = {"cellsX": SI_FLUID_GRID_CELLS, "cellsY": SI_FLUID_GRID_CELLS,
            "cellSize": MPM_SI_BOX_DOMAIN["innerWidthM"] / SI_FLUID_GRID_CELLS}
    config = {"grid": grid, "particleMass": material["density"] * area, "particleVolume": area,
              "material": material, "wallFriction": SI_FLUID_WALL_FRICTION}
    return p, config


def create_si_tank_scene(seed: int = 1):
    """The SI tank workload: 80x80 grid over 0.2 m (dx 2.5 mm), 40x40 lattice at
    1.25 mm filling [0, 50 mm]^2, jitter U(+-0.1 dx), rho 1000 kg/m^3 with 0.02 m
    extrusion, Tait gamma 7, c 20 m/s, gravity (0, -9.81), no-slip walls."""
    depth = MPM_SI_BOX_DOMAIN["extrusionDepthM"]
    tait = {"referenceDensityKgPerM3": 1000.0, "exponent": 7.0,
            "pressureCoefficientPa": derive_tait_pressure_coefficient_pa(1000.0, 7.0, 20.0)}
    material = create_mpm_tait_liquid_material(tait, depth)
    dx = 0.2 / 80
    spacing = 0.00125
    side = 40
    n = side * side
    rnd = lcg_sequence(seed, 2 * n)
    p = ParticleArrays.empty(n)
    r, c = np.divmod(np.arange(n), side)
    p.px[:] = (c + 0.5) * spacing + (rnd[0::2] * 2 - 1) * 0.1 * dx
    p.py[:] = (r + 0.5) * spacing + (rnd[1::2] * 2 - 1) * 0.1 * dx
    area = spacing * spacing
    p.volume[:] = area
    config = {"grid": {"cellsX": 80, "cellsY": 80, "cellSize": dx}, "particleMass": material["density"] * area,
              "particleVolume": area, "material": material, "wallFriction": 1.0}
    return p, config


SI_TANK_GRAVITY = {"x": 0.0, "y": -9.81}
SI_TANK_FIXED_STEP_SECONDS = 1 / 120

# ----------------------------------------------------------------- gate 4 --

GATE4_GRID = {"cellsX": 220, "cellsY": 150, "cellSize": 10}
GATE4_SCENE_SEED = 0x4D504D34
GATE4_FIXED_STEP_SECONDS = 1 / 240
GATE4_DEFAULT_GRAVITY = {"x": 0.0, "y": 90.0}
GATE4_LIQUID_PARTICLE_SPACING = 18
GATE4_PARTICLE_AREA = 100
GATE4_LIQUID_PARTICLE_DIAMETER = 20
GATE4_LIQUID_PARTICLE_AREA = GATE4_LIQUID_PARTICLE_DIAMETER ** 2
GATE4_LIQUID_BULK_MODULUS_SCALE = 4
GATE4_SOLID_PARTICLE_MASS = 4
GATE4_PEBBLE_COUNT = 50
GATE4_PEBBLE_COLUMNS = 8
GATE4_PEBBLE_ROWS = math.ceil(GATE4_PEBBLE_COUNT / GATE4_PEBBLE_COLUMNS)
GATE4_PEBBLE_SPACING = 150
GATE4_FRACTURE_COLUMNS, GATE4_FRACTURE_ROWS, GATE4_FRACTURE_SPACING = 6, 4, 20
GATE4_FRACTURE_FAILURE_STRAIN = 0.12
GATE4_PEBBLE_EDGE_LENGTH = GATE4_GRID["cellsX"] * GATE4_GRID["cellSize"] * 0.005 * 12
GATE4_WATER_MATERIAL = {"lambda": 40_000 * GATE4_LIQUID_BULK_MODULUS_SCALE, "mu": 0.0, "model": "water", "density": 0.02}
GATE4_OIL_MATERIAL = {"lambda": 30_000 * GATE4_LIQUID_BULK_MODULUS_SCALE, "mu": 0.0, "model": "oil", "density": 0.016}
GATE4_PEBBLE_MATERIAL = {"lambda": 20.0, "mu": 10.0, "model": "neo-hookean"}


def create_mpm_gate4_scene(seed: int = GATE4_SCENE_SEED, liquid_particle_diameter: float = 20,
                           liquid_particle_area: float | None = None, y_shift: float = 0.0):
    """createMpmGate4Scene, gate4.ts:191-339 -> (ParticleArrays, fractureBonds,
    parityProbeIndices).  `liquid_particle_area` and `y_shift` give the
    enlarged variant (220x600 grid, liquid area 1,600, +4,500 in y)."""
    if not (10 <= liquid_particle_diameter <= 21):
        raise ValueError("liquidParticleDiameter must be between 10 and 21.")
    area = liquid_particle_area if liquid_particle_area is not None else liquid_particle_diameter ** 2
    random = SeededRandom(seed)
    rows_out = []
    probes = []
    objects = [
        (1, 100, 640, 50, 40, 0, 25, GATE4_WATER_MATERIAL, 64),
        (2, 100, 100, 50, 30, 29, 25, GATE4_OIL_MATERIAL, 64),
    ]
    mats = [GATE4_WATER_MATERIAL, GATE4_OIL_MATERIAL, GATE4_PEBBLE_MATERIAL]
    for oid, sx, sy, cols, rows, prow, pcol, mat, vmax in objects:
        start = len(rows_out)
        for r in range(rows):
            for c in range(cols):
                vx = (random() * 2 - 1) * vmax
                vy = (random() * 2 - 1) * vmax
                rows_out.append((sx + c * GATE4_LIQUID_PARTICLE_SPACING, sy + r * GATE4_LIQUID_PARTICLE_SPACING + y_shift,
                                 vx, vy, oid, -1, area, mats.index(mat)))
        probes.append(start + prow * cols + pcol)
    parity_pebble = (GATE4_PEBBLE_ROWS // 2) * GATE4_PEBBLE_COLUMNS + GATE4_PEBBLE_COLUMNS // 2
    edge = GATE4_PEBBLE_EDGE_LENGTH
    for k in range(GATE4_PEBBLE_COUNT):
        row = k // GATE4_PEBBLE_COLUMNS
        row_start = row * GATE4_PEBBLE_COLUMNS
        in_row = min(GATE4_PEBBLE_COLUMNS, GATE4_PEBBLE_COUNT - row_start)
        column = k - row_start + (GATE4_PEBBLE_COLUMNS - in_row) * 0.5
        cx = 700 + (column - (GATE4_PEBBLE_COLUMNS - 1) / 2) * GATE4_PEBBLE_SPACING
        cy = 569 + (row - (GATE4_PEBBLE_ROWS - 1) / 2) * GATE4_PEBBLE_SPACING + y_shift
        verts = [(cx - edge * 0.5, cy - edge / (2 * math.sqrt(3))), (cx + edge * 0.5, cy - edge / (2 * math.sqrt(3))),
                 (cx, cy + edge / math.sqrt(3))]
        start = len(rows_out)
        for v, (x, y) in enumerate(verts):
            vx = (random() * 2 - 1) * 240
            vy = (random() * 2 - 1) * 240
            rows_out.append((x, y, vx, vy, 3 + k, v, GATE4_PARTICLE_AREA, 2))
        if k == parity_pebble:
            probes.append(start + 2)
    fstart = len(rows_out)
    fvx = (random() * 2 - 1) * 80
    fvy = (random() * 2 - 1) * 80
    for r in range(GATE4_FRACTURE_ROWS):
        for c in range(GATE4_FRACTURE_COLUMNS):
            x = 1520 + (c - (GATE4_FRACTURE_COLUMNS - 1) / 2) * GATE4_FRACTURE_SPACING
            y = 1380 + (r - (GATE4_FRACTURE_ROWS - 1) / 2) * GATE4_FRACTURE_SPACING + y_shift
            rows_out.append((x, y, fvx, fvy, 3 + GATE4_PEBBLE_COUNT, -1, GATE4_PARTICLE_AREA, 2))
    bonds = []
    idx = lambda r, c: fstart + r * GATE4_FRACTURE_COLUMNS + c  # noqa: E731
    for r in range(GATE4_FRACTURE_ROWS):
        for c in range(GATE4_FRACTURE_COLUMNS):
            first = idx(r, c)
            if c + 1 < GATE4_FRACTURE_COLUMNS:
                bonds.append({"firstParticle": first, "secondParticle": first + 1,
                              "restLength": GATE4_FRACTURE_SPACING, "failureStrain": GATE4_FRACTURE_FAILURE_STRAIN})
            if r + 1 < GATE4_FRACTURE_ROWS:
                bonds.append({"firstParticle": first, "secondParticle": first + GATE4_FRACTURE_COLUMNS,
                              "restLength": GATE4_FRACTURE_SPACING, "failureStrain": GATE4_FRACTURE_FAILURE_STRAIN})
            if r + 1 < GATE4_FRACTURE_ROWS and c + 1 < GATE4_FRACTURE_COLUMNS:
                bonds.append({"firstParticle": first, "secondParticle": first + GATE4_FRACTURE_COLUMNS + 1,
                              "restLength": GATE4_FRACTURE_SPACING * math.sqrt(2),
                              "failureStrain": GATE4_FRACTURE_FAILURE_STRAIN})
    n = len(rows_out)
    arr = np.array(rows_out, dtype=np.float64)
    p = ParticleArrays.empty(n)
    p.px[:], p.py[:], p.vx[:], p.vy[:] = arr[:, 0], arr[:, 1], arr[:, 2], arr[:, 3]
    p.object_id[:] = arr[:, 4].astype(np.int64)
    p.bonded_vertex[:] = arr[:, 5].astype(np.int8)
    p.volume[:] = arr[:, 6]
    p.plastic_volume[:] = 1.0
    p.material[:] = arr[:, 7].astype(np.int32)
    p.materials = mats
    return p, bonds, probes


def create_mpm_cpu_parity_sample(particles, probe_indices, grid_cell_size: float) -> dict:
    """createMpmCpuParitySample (src/lib/mpm/scenes/gate4.ts:359-467): the
    particles a CPU step needs to reproduce the probes' step -- every
    particle within 20 cells of a probe, every bonded triangle whose box lies
    within 22 cells of a probe with the particles within 20 cells of that box,
    and the whole triangle of every bonded vertex taken -- in source order.
    Returns {"particles": ParticleArrays, "sourceIndices": [...],
    "probeSampleIndices": [...]} with the reference's errors."""
    probes = list(probe_indices)
    if not probes:
        raise RangeError("At least one CPU/GPU parity probe is required.")
    if not (math.isfinite(grid_cell_size) and grid_cell_size > 0):
        raise RangeError("gridCellSize must be a positive finite number.")
    n = len(particles)
    for index in probes:
        if not isinstance(index, (int, np.integer)) or index < 0 or index >= n:
            raise RangeError("CPU/GPU parity probe indices must identify input particles.")
    px, py = np.asarray(particles.px, np.float64), np.asarray(particles.py, np.float64)
    vertex = np.asarray(particles.bonded_vertex, np.int64)  # -1: not a bonded vertex
    qx, qy = px[probes], py[probes]
    radius = grid_cell_size * 20
    source = np.zeros(n, bool)
    for x, y in zip(qx, qy):
        source |= (np.abs(px - x) <= radius) & (np.abs(py - y) <= radius)
    contact = radius + 2 * grid_cell_size

    def body_ok(start):
        return start + 3 <= n and all(vertex[start + v] == v for v in range(3))

    for start in np.flatnonzero(vertex == 0):
        start = int(start)
        if not body_ok(start):
            raise RangeError(f"Bonded triangle at particle {start} is incomplete.")
        bx, by = px[start:start + 3], py[start:start + 3]
        x0, x1, y0, y1 = bx.min(), bx.max(), by.min(), by.max()
        if not np.any((qx >= x0 - contact) & (qx <= x1 + contact) & (qy >= y0 - contact) & (qy <= y1 + contact)):
            continue
        source[start:start + 3] = True
        source |= (px >= x0 - radius) & (px <= x1 + radius) & (py >= y0 - radius) & (py <= y1 + radius)
    for index in np.flatnonzero(source & (vertex >= 0)):
        start = int(index - vertex[index])
        if start < 0 or not body_ok(start):
            raise RangeError(f"Bonded triangle at particle {start} is incomplete.")
        source[start:start + 3] = True
    ordered = np.flatnonzero(source)
    position = {int(s): k for k, s in enumerate(ordered)}
    probe_samples = []
    for index in probes:
        if int(index) not in position:
            raise RuntimeError(f"CPU/GPU parity probe {index} is missing from its local sample.")
        probe_samples.append(position[int(index)])
    return {"particles": particles.take(ordered), "sourceIndices": [int(s) for s in ordered],
            "probeSampleIndices": probe_samples}


def create_mpm_gate4_step_config(gravity=None, dt=GATE4_FIXED_STEP_SECONDS, fracture_bonds=None, grid=None):
    """createMpmGate4StepConfig, gate4.ts:341-357."""
    cfg = {"dt": dt, "bondReferenceDt": GATE4_FIXED_STEP_SECONDS, "grid": dict(grid or GATE4_GRID),
           "particleMass": GATE4_SOLID_PARTICLE_MASS, "particleVolume": GATE4_PARTICLE_AREA,
           "bondRestLength": GATE4_PEBBLE_EDGE_LENGTH, "material": GATE4_PEBBLE_MATERIAL,
           "gravity": dict(gravity or GATE4_DEFAULT_GRAVITY)}
    if fracture_bonds is not None:
        cfg["fractureBonds"] = fracture_bonds
    return cfg


# -------------------------------------------------------------- dam break --

DAM_BREAK_GRID = {"cellsX": 1024, "cellsY": 2048, "cellSize": 10}
DAM_BREAK_GRAVITY = {"x": 0.0, "y": 90.0}
DAM_BREAK_FIXED_STEP_SECONDS = 1 / 240


def create_dam_break_scene(particles_per_phase: int = 500_000, columns: int = 500, grid=None):
    """Two stacked liquid blocks (y-down, gravity +y): water on the floor, oil
    above it, both at the left wall; 2x2 particles per 10-unit cell (spacing 5,
    area 25), zero velocity, Gate-4 liquid materials (legacy linear EOS,
    lambda 160,000 / 120,000, density 0.02 / 0.016)."""
    grid = dict(grid or DAM_BREAK_GRID)
    spacing = grid["cellSize"] / 2
    rows = particles_per_phase // columns
    if rows * columns != particles_per_phase:
        raise ValueError("particles_per_phase must be a multiple of columns")
    height = grid["cellsY"] * grid["cellSize"]
    margin = 2 * grid["cellSize"]
    n = 2 * particles_per_phase
    p = ParticleArrays.empty(n)
    k = np.arange(particles_per_phase)
    r, c = np.divmod(k, columns)
    x = margin + (c + 0.5) * spacing
    water_y = height - margin - (r + 0.5) * spacing
    oil_y = height - margin - rows * spacing - (r + 0.5) * spacing
    if oil_y.min() < 0 or x.max() > grid["cellsX"] * grid["cellSize"]:
        raise ValueError("the dam-break blocks do not fit the grid")
    p.px[:particles_per_phase], p.py[:particles_per_phase] = x, water_y
    p.px[particles_per_phase:], p.py[particles_per_phase:] = x, oil_y
    p.object_id[:particles_per_phase] = 1
    p.object_id[particles_per_phase:] = 2
    p.volume[:] = spacing * spacing
    p.plastic_volume[:] = 1.0
    p.materials = [GATE4_WATER_MATERIAL, GATE4_OIL_MATERIAL]
    p.material[:particles_per_phase] = 0
    p.material[particles_per_phase:] = 1
    mass = GATE4_WATER_MATERIAL["density"] * spacing * spacing
    config = {"grid": grid, "particleMass": mass, "particleVolume": spacing * spacing,
              "material": GATE4_WATER_MATERIAL, "wallFriction": 0.0}
    return p, config


# ------------------------------------------------------------ batched tanks --

BATCHED_TANK_DOMAIN_M = 0.2
BATCHED_TANK_GRAVITY = {"x": 0.0, "y": -9.81}
BATCHED_TANK_MAX_FILL_HEIGHT = 0.6  # of the box


def batched_tank_scene_specs(count: int = 512, seed: int = 0x4D504D42, particles=(1_000, 64_000), sides=(64, 512),
                             first: int = 0) -> list:
    """(particle count N, grid side S) of scenes first .. first + count - 1
    of create_batched_tank_scenes, without building their particles (the
    first two draws of each scene's LCG)."""
    out = []
    for k in range(first, first + count):
        rnd = SeededRandom((seed + k * 0x9E3779B9) % UINT32_RANGE)
        log_lo, log_hi = math.log(particles[0]), math.log(particles[1])
        n = int(round(math.exp(log_lo + rnd() * (log_hi - log_lo))))
        side = min(int(sides[0] + math.floor(rnd() * (sides[1] - sides[0] + 1))), sides[1])
        out.append((n, side))
    return out


def create_batched_tank_scenes(count: int = 512, seed: int = 0x4D504D42, particles=(1_000, 64_000),
                               sides=(64, 512), first: int = 0, indices=None):
    """`count` independent SI Tait water tanks (rho 1000 kg/m^3, gamma 7,
    c = 20 m/s, 0.02 m extrusion, no-slip walls, at rest under y-up gravity
    9.81 m/s^2), each a 0.2 m square box.  Scene k (k = first, ..., first +
    count - 1) draws from the LCG seeded with (seed + k * 0x9E3779B9) mod
    2^32: its particle count N log-uniform in
    `particles`, its grid side S uniform in `sides` (S x S cells, dx = 0.2 m /
    S), the width of its block (a quarter to 0.6 of the box) and the block's
    place.  The block is a lattice at dx / 2 (2 x 2 particles per cell) where
    N of them fit under 0.6 of the box height, else at the finer spacing that
    fits; each particle is jittered by U(+-0.1) spacing.  `indices`, when
    given, replaces first .. first + count - 1 by those scene numbers.
    Returns [(particles, config), ...]."""
    depth = MPM_SI_BOX_DOMAIN["extrusionDepthM"]
    tait = {"referenceDensityKgPerM3": 1000.0, "exponent": 7.0,
            "pressureCoefficientPa": derive_tait_pressure_coefficient_pa(1000.0, 7.0, 20.0)}
    material = create_mpm_tait_liquid_material(tait, depth)
    size = BATCHED_TANK_DOMAIN_M
    top = BATCHED_TANK_MAX_FILL_HEIGHT * size
    out = []
    for k in (range(first, first + count) if indices is None else indices):
        rnd = SeededRandom((seed + k * 0x9E3779B9) % UINT32_RANGE)
        log_lo, log_hi = math.log(particles[0]), math.log(particles[1])
        n = int(round(math.exp(log_lo + rnd() * (log_hi - log_lo))))
        side = min(int(sides[0] + math.floor(rnd() * (sides[1] - sides[0] + 1))), sides[1])
        dx = size / side
        width = size * (0.25 + 0.35 * rnd())

        def height(spacing):
            return math.ceil(n / max(1, math.floor(width / spacing))) * spacing

        spacing = dx / 2
        if height(spacing) > top:
            spacing = math.sqrt(width * top / n)
            while height(spacing) > top:
                spacing *= 0.99
        columns = max(1, math.floor(width / spacing))
        rows = math.ceil(n / columns)
        x0 = (size - columns * spacing) * rnd()
        y0 = (size - rows * spacing) * 0.5 * rnd()
        jitter = lcg_sequence(rnd.state, 2 * n)
        r, c = np.divmod(np.arange(n), columns)
        p = ParticleArrays.empty(n)
        p.px[:] = x0 + (c + 0.5) * spacing + (jitter[0::2] * 2 - 1) * 0.1 * spacing
        p.py[:] = y0 + (r + 0.5) * spacing + (jitter[1::2] * 2 - 1) * 0.1 * spacing
        area = spacing * spacing
        p.volume[:] = area
        config = {"grid": {"cellsX": side, "cellsY": side, "cellSize": dx},
                  "particleMass": material["density"] * area, "particleVolume": area, "material": material,
                  "wallFriction": 1.0}
        out.append((p, config))
    return out


# ------------------------------------------------------- adjoint scenes --

ADJOINT_GRAVITY = {"x": 0.0, "y": 90.0}
ADJOINT_TAIT_WATER = {"lambda": 22_857.0, "mu": 0.0, "model": "water", "density": 0.02,
                      "equationOfState": {"model": "tait", "exponent": 7.0}}
ADJOINT_SOLID = {"lambda": 20.0, "mu": 10.0, "model": "fixed-corotated"}


def _normal_pairs(rnd: SeededRandom, count: int) -> np.ndarray:
    """`count` standard normal draws by Box-Muller over the seeded LCG."""
    u = lcg_sequence(rnd.state, 2 * ((count + 1) // 2))
    u1 = np.maximum(u[0::2], 1e-12)
    r = np.sqrt(-2.0 * np.log(u1))
    z = np.concatenate([r * np.cos(2 * np.pi * u[1::2]), r * np.sin(2 * np.pi * u[1::2])])
    return z[:count]


def create_adjoint_scenes(count: int = 64, seed: int = 0x4D504D41, water_columns: int = 96, water_rows: int = 128,
                          solid_side: int = 64, cells: int = 256, velocity_sigma: float = 10.0,
                          target_amplitude: float = 20.0, first: int = 0):
    """`count` scenes for the differentiable form, in Gate-4 world units
    (cellSize 10, gravity 90 along +y): a block of water_columns x water_rows
    Tait water particles (density 0.02, gamma 7, pressure coefficient
    22,857: the linear EOS's 2,828 sound speed) and a block of solid_side^2
    fixed-corotated solid particles (lambda 20, mu 10, density 0.02), both at
    2 x 2 particles per cell (spacing 5, area 25), on a cells x cells grid.
    Scene k (k = first, ..., first + count - 1) draws from the LCG seeded with
    (seed + k * 0x9E3779B9) mod 2^32: the blocks' places, initial velocities N(0, velocity_sigma^2) per
    component, and a target displacement field d(x) = A (sin(2 pi k1 x / L +
    p1), cos(2 pi k2 y / L + p2)) with A = target_amplitude.  Returns
    [(particles, config, targets (n, 2))]; the defaults give 64 scenes of
    12,288 + 4,096 particles on 256 x 256 grids."""
    dx, spacing = 10.0, 5.0
    size = cells * dx
    area = spacing * spacing
    out = []
    for k in range(first, first + count):
        rnd = SeededRandom((seed + k * 0x9E3779B9) % UINT32_RANGE)
        ww, wh = water_columns * spacing, water_rows * spacing
        sw = solid_side * spacing
        margin = 4 * dx
        wx0 = margin + rnd() * (size / 2 - ww - 2 * margin)
        wy0 = margin + rnd() * (size - wh - 2 * margin)
        sx0 = size / 2 + margin + rnd() * (size / 2 - sw - 2 * margin)
        sy0 = margin + rnd() * (size - sw - 2 * margin)
        nw, ns = water_columns * water_rows, solid_side * solid_side
        n = nw + ns
        p = ParticleArrays.empty(n)
        r, c = np.divmod(np.arange(nw), water_columns)
        p.px[:nw] = wx0 + (c + 0.5) * spacing
        p.py[:nw] = wy0 + (r + 0.5) * spacing
        r, c = np.divmod(np.arange(ns), solid_side)
        p.px[nw:] = sx0 + (c + 0.5) * spacing
        p.py[nw:] = sy0 + (r + 0.5) * spacing
        z = _normal_pairs(rnd, 2 * n) * velocity_sigma
        rnd.state = (rnd.state * 1_664_525 + 1_013_904_223) & 0xFFFFFFFF  # past the normal draws
        p.vx[:] = z[:n]
        p.vy[:] = z[n:]
        p.volume[:] = area
        p.materials = [ADJOINT_TAIT_WATER, ADJOINT_SOLID]
        p.material[:nw] = 0
        p.material[nw:] = 1
        p.object_id[:nw] = 1
        p.object_id[nw:] = 2
        k1, k2 = 1 + int(rnd() * 3), 1 + int(rnd() * 3)
        p1, p2 = 2 * np.pi * rnd(), 2 * np.pi * rnd()
        targets = np.stack([p.px + target_amplitude * np.sin(2 * np.pi * k1 * p.px / size + p1),
                            p.py + target_amplitude * np.cos(2 * np.pi * k2 * p.py / size + p2)], axis=1)
        config = {"grid": {"cellsX": cells, "cellsY": cells, "cellSize": dx}, "particleMass": 0.02 * area,
                  "particleVolume": area, "material": ADJOINT_SOLID, "wallFriction": 0.0}
        out.append((p, config, targets))
    return out


# ---------------------------------------------------------------- emitter --

MAX_MPM_EMITTER_PARTICLES = 100_000
_GOLDEN_ANGLE = math.pi * (3 - math.sqrt(5))
_EMITTER_MATERIALS = {
    "water": dict(GATE4_WATER_MATERIAL),
    "oil": dict(GATE4_OIL_MATERIAL),
    "neo-hookean": {"lambda": 20.0, "mu": 10.0, "model": "neo-hookean"},
}


def create_mpm_emitter_particles(config: dict) -> list:
    """createMpmEmitterParticles, emitter.ts:49-129: `count` particles in a
    jittered rectangle lattice or a golden-angle disc around `center`, with
    the seeded LCG's draws in the reference's order."""
    count = config.get("count")
    if not isinstance(count, int) or isinstance(count, bool) or count < 1:
        raise RangeError("count must be a positive safe integer")
    if count > MAX_MPM_EMITTER_PARTICLES:
        raise RangeError(f"count must not exceed {MAX_MPM_EMITTER_PARTICLES}")
    seed = config.get("seed")
    if not isinstance(seed, int) or isinstance(seed, bool) or seed < 0 or seed > 0xFFFFFFFF:
        raise RangeError("seed must be an unsigned 32-bit integer")
    shape = config.get("shape")
    if shape not in ("rectangle", "circle"):
        raise RangeError("shape must be rectangle or circle")
    material = config.get("material")
    if material not in _EMITTER_MATERIALS:
        raise RangeError("material must be water, oil, or neo-hookean")

    def vector(v, name):
        if not isinstance(v, dict):
            raise TypeError(f"{name} must be a vector")
        if not all(isinstance(v.get(k), (int, float)) and math.isfinite(v.get(k)) for k in ("x", "y")):
            raise RangeError(f"{name} components must be finite")
        return float(v["x"]), float(v["y"])

    def positive(v, name):
        if not isinstance(v, (int, float)) or not math.isfinite(v) or v <= 0:
            raise RangeError(f"{name} must be a positive finite number")
        return float(v)

    cx, cy = vector(config.get("center"), "center")
    vx, vy = vector(config.get("velocity"), "velocity")
    grid = config.get("grid")
    if not isinstance(grid, dict):
        raise TypeError("grid must be an object")
    if not all(isinstance(grid.get(k), int) and grid.get(k) >= 1 for k in ("cellsX", "cellsY")):
        raise RangeError("grid cell counts must be positive safe integers")
    cell = positive(grid.get("cellSize"), "grid.cellSize")
    spacing = positive(config.get("spacing"), "spacing")
    volume = positive(config.get("particleVolume", 25), "particleVolume")
    width, height = grid["cellsX"] * cell, grid["cellsY"] * cell
    if cx < 0 or cx > width or cy < 0 or cy > height:
        raise RangeError("center must be inside the simulation domain")
    random = SeededRandom(seed)
    columns = math.ceil(math.sqrt(count))
    rows = math.ceil(count / columns)
    radius = spacing * math.sqrt(count / math.pi)
    angular_offset = random() * math.pi * 2
    out = []
    for index in range(count):
        if shape == "circle":
            radial = math.sqrt((index + 0.5) / count)
            angle = angular_offset + index * _GOLDEN_ANGLE
            jitter = (random() - 0.5) * spacing * 0.12
            distance = max(0.0, radial * radius + jitter)
            x, y = cx + math.cos(angle) * distance, cy + math.sin(angle) * distance
        else:
            column, row = index % columns, index // columns
            x = cx + (column - (columns - 1) * 0.5) * spacing + (random() - 0.5) * spacing * 0.12
            y = cy + (row - (rows - 1) * 0.5) * spacing + (random() - 0.5) * spacing * 0.12
        if x < 0 or x > width or y < 0 or y > height:
            raise RangeError(f"emitted particle {index} would be outside the simulation domain")
        out.append({"position": {"x": x, "y": y}, "velocity": {"x": vx, "y": vy},
                    "C": {"m00": 0.0, "m01": 0.0, "m10": 0.0, "m11": 0.0},
                    "F": {"m00": 1.0, "m01": 0.0, "m10": 0.0, "m11": 1.0}, "plasticVolume": 1.0,
                    "volume": volume, "material": dict(_EMITTER_MATERIALS[material])})
    return out

