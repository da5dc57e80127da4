"""The default path's substep variants and the barrier wait limit.

A substep runs either as ONE cooperative launch of persistent CTAs
(k_substep: tile allocation, bucketing, P2G, grid update + G2P, with grid
barriers between the phases) or as four launches of the same device code, so
the two forms must agree bit for bit, whatever the persistent grid; so must
G2P's water-and-oil instantiation and its general one on a scene of water
and oil, and the two ways of handing prepareParticle's results to P2G
(records written by G2P, or each particle prepared in P2G).  The
narrow P2G stage (384 particles) changes only how a crowded tile is cut into
chunks, so it must stay within the oracle tolerances.  A CTA that leaves
before the first barrier without arriving makes the others' waits run out:
the launch must then report status flag 1 << 20 and return instead of
hanging, and the solver must step normally once its particles are written
back.
"""
import numpy as np
import pytest

from mpm_b200 import create_mpm_batched_gpu_solver, create_mpm_mls_gpu_solver
from mpm_b200.errors import decode_numerical_error, is_recoverable_cfl_error
from mpm_b200.layout import ParticleArrays, particles_from_dicts
from mpm_b200.scenes import (BATCHED_TANK_GRAVITY, DAM_BREAK_GRAVITY, GATE4_FIXED_STEP_SECONDS, SI_TANK_GRAVITY,
                             create_batched_tank_scenes, create_dam_break_scene, create_mpm_gate4_scene,
                             create_mpm_gate4_step_config, create_si_tank_scene)
from oracle import OracleState

from helpers import transfer_regression_fixture

pytestmark = pytest.mark.gpu

STATE_WORDS = slice(0, 12)  # x, v, C, F of the packed 20-word record
ERROR_BARRIER = 1 << 20
SMALL_DAM = {"cellsX": 256, "cellsY": 512, "cellSize": 10}


def _bits(packed):
    return np.ascontiguousarray(packed[:, STATE_WORDS]).view(np.uint32)


def _step(particles, config, variant, steps, dt, gravity, g2p_ctas=0):
    solver = create_mpm_mls_gpu_solver(particles, config)
    try:
        solver.set_substep_variant(**variant)
        if g2p_ctas:
            solver.set_launch_shape(g2p_ctas=g2p_ctas)
        chosen = solver.substep_variant()
        solver.step_batch(steps, dt, gravity)
        status = solver._read_compact()[2]
        packed, _ = solver.read_particles_packed()
    finally:
        solver.dispose()
    return packed, status, chosen


def test_one_launch_and_four_launches_agree_bitwise_on_a_dam_break():
    p, config = create_dam_break_scene(particles_per_phase=20_000, columns=200, grid=SMALL_DAM)
    dt = 1.0 / 1200.0
    runs = {}
    for name, variant in {"one": dict(fused=True, stage_capacity=640),
                          "one_148": dict(fused=True, stage_capacity=640, substep_ctas=148),
                          "four": dict(fused=False, stage_capacity=640),
                          "four_general": dict(fused=False, stage_capacity=640, liquid_kernels=False),
                          "one_general": dict(fused=True, stage_capacity=640, liquid_kernels=False),
                          "four_records": dict(fused=False, stage_capacity=640, p2g_records=True),
                          "four_records_general": dict(fused=False, stage_capacity=640, p2g_records=True,
                                                       liquid_kernels=False),
                          "one_narrow": dict(fused=True, stage_capacity=384),
                          "four_narrow": dict(fused=False, stage_capacity=384)}.items():
        packed, status, chosen = _step(p, config, variant, 24, dt, DAM_BREAK_GRAVITY)
        assert status[0] == 0, name
        assert chosen["fused"] == variant["fused"] and chosen["stageCapacity"] == variant["stage_capacity"]
        # water and oil only: G2P runs its water-and-oil instantiation unless told not to
        assert chosen["liquidKernels"] == variant.get("liquid_kernels", True)
        # linear-EOS liquids: P2G prepares each particle unless records are asked for
        assert chosen["p2gRecords"] == variant.get("p2g_records", False)
        runs[name] = packed
    assert np.array_equal(_bits(runs["one"]), _bits(runs["four"]))
    assert np.array_equal(_bits(runs["four"]), _bits(runs["four_general"]))
    assert np.array_equal(_bits(runs["one"]), _bits(runs["one_general"]))
    assert np.array_equal(_bits(runs["four"]), _bits(runs["four_records"]))
    assert np.array_equal(_bits(runs["four"]), _bits(runs["four_records_general"]))
    assert np.array_equal(_bits(runs["one"]), _bits(runs["one_148"]))
    assert np.array_equal(_bits(runs["one_narrow"]), _bits(runs["four_narrow"]))
    # both stage capacities agree within the oracle tolerances (position 1e-3 dx)
    dx = config["grid"]["cellSize"]
    assert np.max(np.abs(runs["one"][:, 0:2].astype(np.float64) - runs["one_narrow"][:, 0:2])) <= 1e-3 * dx


@pytest.mark.parametrize("g2p_ctas", [7, 64])
def test_small_persistent_g2p_grids_agree_bitwise(g2p_ctas):
    # With one scene each G2P CTA copies the next tile's bucket range,
    # neighbour records, first bucket entries and status words in while the
    # current tile's particles move; a small persistent grid gives every CTA
    # many tiles, so most tiles run on prefetched data, among them tiles at
    # the edge of the fluid whose neighbours hold no record or only one
    # liquid's channel.  The water-and-oil and the general instantiation
    # must agree bit for bit there too.
    p, config = create_dam_break_scene(particles_per_phase=20_000, columns=200, grid=SMALL_DAM)
    dt = 1.0 / 1200.0
    liquid, status, chosen = _step(p, config, dict(fused=False), 24, dt, DAM_BREAK_GRAVITY, g2p_ctas=g2p_ctas)
    assert status[0] == 0 and chosen["liquidKernels"]
    general, status, chosen = _step(p, config, dict(fused=False, liquid_kernels=False), 24, dt, DAM_BREAK_GRAVITY,
                                    g2p_ctas=g2p_ctas)
    assert status[0] == 0 and not chosen["liquidKernels"]
    assert np.array_equal(_bits(liquid), _bits(general))
    default, status, _ = _step(p, config, dict(fused=False), 24, dt, DAM_BREAK_GRAVITY)
    assert np.array_equal(_bits(liquid), _bits(default))


def _touched_nodes(px, py, dx):
    """Nodes with a positive quadratic weight from the particles at (px, py):
    the base node's stencil as the kernels form it (position * (1 / dx),
    base = floor(g - 0.5), f = g - base; float32), offsets 0 and 1 always
    and 2 where f > 0.5 (the third weight is 0.5 (f - 0.5)^2)."""
    inv = np.float32(1) / np.float32(dx)

    def axis(x):
        g = np.asarray(x, np.float32) * inv
        base = np.floor(g - np.float32(0.5))
        return base.astype(np.int64), (g - base) > np.float32(0.5)

    (bx, third_x), (by, third_y) = axis(px), axis(py)
    nodes = set()
    for ox in range(3):
        for oy in range(3):
            keep = np.ones(len(bx), bool)
            if ox == 2:
                keep &= third_x
            if oy == 2:
                keep &= third_y
            nodes.update(zip((bx[keep] + ox).tolist(), (by[keep] + oy).tolist()))
    return len(nodes)


def test_active_node_count_is_the_last_substeps_nodes_with_mass():
    # the default path counts, from the ring records of the last substep, the
    # nodes whose summed water / oil mass is positive: after one substep from
    # the uploaded state those are the nodes the particles' stencils weigh
    p, config = create_dam_break_scene(particles_per_phase=20_000, columns=200, grid=SMALL_DAM)
    solver = create_mpm_mls_gpu_solver(p, config)
    try:
        solver.step_batch(1, 1.0 / 1200.0, DAM_BREAK_GRAVITY)
        assert solver._read_compact()[2][0] == 0
        counts = solver.count_active_nodes()
    finally:
        solver.dispose()
    water, oil = p.material == 0, p.material == 1
    dx = config["grid"]["cellSize"]
    assert counts == (0, _touched_nodes(p.px[water], p.py[water], dx), _touched_nodes(p.px[oil], p.py[oil], dx))


def _crowded_tank(per_side):
    """The SI tank's water as a block of per_side^2 particles per cell over
    12 x 12 cells: its tiles hold far more than one stage (the crowded path of
    either capacity)."""
    _, config = create_si_tank_scene(seed=1)
    dx = config["grid"]["cellSize"]
    spacing = dx / per_side
    side = 12 * per_side
    r, c = np.divmod(np.arange(side * side), side)
    p = ParticleArrays.empty(side * side)
    p.px[:] = 12 * dx + (c + 0.5) * spacing
    p.py[:] = 12 * dx + (r + 0.5) * spacing
    p.volume[:] = spacing * spacing
    config = dict(config, particleMass=config["material"]["density"] * spacing * spacing,
                  particleVolume=spacing * spacing)
    return p, config


@pytest.mark.parametrize("per_side", [6, 10])
def test_crowded_tiles_match_the_oracle_in_every_variant(per_side):
    p, config = _crowded_tank(per_side)
    dt = 2e-5
    steps = 6
    dt32 = float(np.float32(dt))
    ref = OracleState(p, dict(config, dt=dt32, gravity=SI_TANK_GRAVITY))
    ref.run(dict(config, dt=dt32, gravity=SI_TANK_GRAVITY), steps)
    dx = config["grid"]["cellSize"]
    results = {}
    for fused, records in ((True, None), (False, True), (False, False)):
        for cap in (640, 384):
            packed, status, _ = _step(p, config, dict(fused=fused, stage_capacity=cap, p2g_records=records), steps,
                                      dt, SI_TANK_GRAVITY)
            assert status[0] == 0
            assert np.max(np.abs(packed[:, 0:2].astype(np.float64) - ref.positions())) <= 1e-3 * dx
            vel_err = np.abs(packed[:, 2:4].astype(np.float64) - ref.velocities()) / (1 + np.abs(ref.velocities()))
            assert np.max(vel_err) <= 1e-3
            results[(fused, records, cap)] = packed
    for cap in (640, 384):
        assert np.array_equal(_bits(results[(True, None, cap)]), _bits(results[(False, True, cap)]))
        assert np.array_equal(_bits(results[(True, None, cap)]), _bits(results[(False, False, cap)]))


def test_batched_scenes_agree_bitwise_in_one_launch_and_four():
    scenes = create_batched_tank_scenes(7, seed=5, particles=(200, 4000), sides=(20, 128))
    out = {}
    for fused, liquid, records in ((True, True, None), (False, True, None), (False, False, None),
                                   (False, True, False)):
        batch = create_mpm_batched_gpu_solver(scenes)
        try:
            batch.set_substep_variant(fused=fused, stage_capacity=640, liquid_kernels=liquid, p2g_records=records)
            chosen = batch.substep_variant()
            assert chosen["fused"] == fused and chosen["liquidKernels"] == liquid
            # several scenes: records by default (the one-launch form prepares in P2G)
            assert chosen["p2gRecords"] == (not fused and records is not False)
            dts = [2e-4 * (1 + 0.1 * k) for k in range(batch.scene_count)]
            batch.step_batch([4 + (k % 3) for k in range(batch.scene_count)], dts, BATCHED_TANK_GRAVITY)
            batch.step_batch([0 if k % 2 else 3 for k in range(batch.scene_count)], dts, BATCHED_TANK_GRAVITY)
            assert all(e is None for e in batch.check_numerical_status())
            out[(fused, liquid, records)] = [batch.read_particles_packed(k)[0] for k in range(batch.scene_count)]
        finally:
            batch.dispose()
    for other in ((False, True, None), (False, False, None), (False, True, False)):
        for k, (a, b) in enumerate(zip(out[(True, True, None)], out[other])):
            assert np.array_equal(_bits(a), _bits(b)), f"scene {k}, variant {other}"


def test_every_material_model_agrees_bitwise_with_and_without_records():
    # the reference's 45-particle five-model fixture (Neo-Hookean, snow, water,
    # oil, powder): P2G's general prepare path against the records G2P writes
    particles, config = transfer_regression_fixture()
    p = particles_from_dicts(particles)
    out = {}
    for records in (True, False):
        packed, status, chosen = _step(p, config, dict(fused=False, p2g_records=records), 16, 0.01,
                                       {"x": 0.0, "y": -0.5})
        assert status[0] == 0 and chosen["p2gRecords"] == records and not chosen["liquidKernels"]
        out[records] = packed
    assert np.array_equal(np.ascontiguousarray(out[True]).view(np.uint32),
                          np.ascontiguousarray(out[False]).view(np.uint32))


def test_bonded_bodies_and_fracture_agree_bitwise_with_and_without_records():
    # the multi-material scene: water, oil, bonded-triangle pebbles and a
    # fractured Neo-Hookean block (bodies take four launches and the general
    # G2P; their moved particles get their bucket keys, and records when
    # used, from the body pass)
    p, bonds, _ = create_mpm_gate4_scene()
    config = create_mpm_gate4_step_config(fracture_bonds=bonds)
    dt = GATE4_FIXED_STEP_SECONDS / 5
    out = {}
    for records in (True, False):
        packed, status, chosen = _step(p, config, dict(fused=False, p2g_records=records), 6, dt, config["gravity"])
        assert status[0] == 0 and not chosen["fused"] and not chosen["liquidKernels"]
        assert chosen["p2gRecords"] == records
        out[records] = packed
    assert np.array_equal(_bits(out[True]), _bits(out[False]))
    # and the damage word of the fractured block
    assert np.array_equal(out[True][:, 18].view(np.uint32), out[False][:, 18].view(np.uint32))


def test_a_barrier_wait_that_runs_out_reports_the_status_and_the_solver_recovers():
    particles, config = create_si_tank_scene(seed=1)
    dt = 2e-4
    solver = create_mpm_mls_gpu_solver(particles, config)
    try:
        solver.set_substep_variant(fused=True)
        assert solver.substep_variant()["fused"]
        start, _ = solver.read_particles_packed()
        # CTA 1 leaves before the first barrier: every other CTA's wait runs
        # out after 2 ms, and the launch (and the batch's next one) returns
        solver.set_barrier_limit(2_000_000, skip_cta=1)
        solver.step_batch(3, dt, SI_TANK_GRAVITY)
        _, _, status = solver._read_compact()
        assert status[0] & ERROR_BARRIER
        error = decode_numerical_error(status)
        assert "grid barrier" in str(error) and not is_recoverable_cfl_error(error)
        # the default limit, the status cleared and the particles written
        # back: the solver steps exactly like a fresh one
        solver.set_barrier_limit(1_000_000_000)
        solver._clear_status()
        solver.write_particles_packed(start)
        solver.step_batch(5, dt, SI_TANK_GRAVITY)
        assert solver._read_compact()[2][0] == 0
        got, _ = solver.read_particles_packed()
    finally:
        solver.dispose()
    fresh, status, _ = _step(particles, config, dict(fused=True), 5, dt, SI_TANK_GRAVITY)
    assert status[0] == 0
    assert np.array_equal(_bits(got), _bits(fresh))
