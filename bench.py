"""Benchmark: particle-substeps/s of the 2D MLS-MPM substep on B200.

Workload (default): the 1,000,000-particle two-phase water/oil dam break on a
1024x2048 grid (cellSize 10, gravity 90, 1/240 s macrosteps split by CFL 0.3),
gather P2G, FP32.  One step = one macrostep: a CFL-certified batch of
microsteps submitted through the reference-facing API
(`step_cfl_batch_adaptive`, the host loop of stepCflBatchAdaptive) with its
compact readback.

* value: particles x committed substeps / summed device time of the batches
  (CUDA events recorded on the solver's stream around each batch);
* e2e: the same count / wall time of the API calls (host CFL planning, the
  parameter upload from pinned memory, the graph launches and the 40-byte
  compact readback of each batch);
* roofline: the dominant kernel, from a kernel-by-kernel event-timed run of
  real substeps right after the timed region;
* cpu_baseline: the FP64 C restatement of the reference CPU step on a bounded
  sample of the same scene, single-threaded like the reference's worker.

`--impl reference` times that CPU restatement alone (the reference is
TypeScript; no JavaScript runtime exists on this image), one single-threaded
process per host core (replicas of the scene for the plain form, shares of
the scenes for the batched and differentiable forms).  Multi-GPU runs are
replicas: each rank steps its own copy of the scene (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "powder-play_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "particle-substeps/s on 1 B200, plain vs batched; adjoint/forward time ratio"
UNIT = "particle-substeps/s"
MACRO_DT = 1 / 240
MAX_MICROSTEPS = 256
L2_FLUSH_BYTES = 512 * 1024 * 1024


def _rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def reduce_over_ranks(dist, device, maxima, sums):
    """The maximum over ranks of each of `maxima` (times) and the sum over
    ranks of each of `sums` (work); one collective each, the same on every
    rank, no collective without a process group."""
    import torch
    t_max = torch.tensor(list(maxima), dtype=torch.float64, device=device)
    t_sum = torch.tensor(list(sums), dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
        dist.all_reduce(t_sum, op=dist.ReduceOp.SUM)
    return [float(v) for v in t_max], [float(v) for v in t_sum]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for name, value in zip(names[1:], r[5:9]):
                if value.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# the launch-shape tuner runs after the first warm-up step unless --no-autotune
AUTOTUNE = True


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def build_workload(name: str):
    from mpm_b200.scenes import (DAM_BREAK_GRAVITY, create_dam_break_scene, create_si_tank_scene, SI_TANK_GRAVITY)
    if name == "dam-break-1m":
        p, config = create_dam_break_scene()
        return p, config, DAM_BREAK_GRAVITY, {
            "workload": "two-phase water/oil dam break, 1,000,000 particles (500k water + 500k oil, 2x2 per "
                        "cell), 1024x2048 grid, cellSize 10, gravity 90, macrostep 1/240 s, CFL 0.3",
            "particles": len(p), "grid": "1024x2048", "macro_dt": MACRO_DT, "courant": 0.3}
    if name == "si-tank":
        p, config = create_si_tank_scene(seed=1)
        return p, config, SI_TANK_GRAVITY, {
            "workload": "SI Tait water tank, 1,600 particles, 80x80 grid (dx 2.5 mm), macrostep 1/120 s",
            "particles": len(p), "grid": "80x80", "macro_dt": 1 / 120, "courant": 0.3,
            "max_microsteps": 4096}  # its 20 m/s sound speed takes about 280 substeps per macrostep
    raise SystemExit(f"unknown workload {name}")


def plan_macrostep(solver, config, velocity, macro_dt, gravity, max_microsteps=MAX_MICROSTEPS):
    from mpm_b200 import calculate_mpm_cfl_microsteps
    from mpm_b200.cfl_bounds import calculate_mpm_cfl_velocity_bound
    gmag = math.hypot(gravity["x"], gravity["y"])
    bound = calculate_mpm_cfl_velocity_bound(velocity, macro_dt, gmag, 0, 0, 0, 0)
    bound = max(bound, solver._last_scheduled_velocity_bound or 0.0)
    plan = calculate_mpm_cfl_microsteps(macro_dt, config["grid"]["cellSize"], solver.cfl_bounds["waveSpeedBound"],
                                        bound, max_microsteps)
    return plan, bound


def cpu_baseline(particles, config, gravity, micro_dt, substeps: int) -> dict:
    """The FP64 C restatement of the reference CPU step (oracle/), timed on a
    bounded sample: `substeps` substeps of the full scene, one thread."""
    from oracle import OracleState
    state = OracleState(particles, dict(config, dt=micro_dt, gravity=gravity))
    cfg = dict(config, dt=micro_dt, gravity=gravity)
    t0 = time.perf_counter()
    state.run(cfg, substeps)
    elapsed = time.perf_counter() - t0
    n = len(particles)
    return {"value": n * substeps / elapsed, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{substeps} substeps of the full {n}-particle scene at dt {micro_dt:.3e} s "
                      f"({elapsed:.1f} s, C FP64 restatement of stepMpm, single thread)"}


def kernel_bytes(name: str, n: int, active: tuple) -> float:
    """Algorithmic bytes per launch of the substep kernels (the per-kernel
    split of 104 B per particle + 64 B per active channel-node)."""
    channel_nodes = float(sum(active))
    table = {
        # G2P: reads x, F, volume, material (32 B), writes x, v, C, F (48 B),
        # reads one 16 B grid record per active channel-node
        "k_g2p": n * 80.0 + channel_nodes * 16.0,
        # grid update + G2P: writes x, v, C, F (48 B); reads the sums, writes and
        # reads one velocity record per active channel-node (3 x 16 B)
        "k_g2p_tile": n * 48.0 + channel_nodes * 48.0,
        # P2G: the particle state it depends on, x, v, C, F, volume, material
        # (56 B; G2P hands it over as a prepared record), writes one 16 B sum
        # record per active channel-node
        "k_p2g_gather": n * 56.0 + channel_nodes * 16.0,
        # grid update: reads the sums, writes one 16 B velocity record
        "k_grid_from_parts": channel_nodes * 32.0,
        "k_grid_update": channel_nodes * 32.0,
        "k_prepare_scatter": n * 56.0 + channel_nodes * 16.0,
        "k_fixed_decode": channel_nodes * 16.0,
        # tile bucketing: reads x (8 B), writes key + rank (8 B); then reads
        # key + rank and writes the permutation (12 B)
        "k_tile_count": n * 16.0,
        "k_tile_scatter": n * 12.0,
        # the whole substep in one launch (allocation, bucketing, P2G, grid
        # update + G2P): the substep's 104 B per particle + 64 B per active
        # channel-node
        "k_substep": n * 104.0 + channel_nodes * 64.0,
    }
    return table.get(name, 0.0)


def dram_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu capture
    (profiles/dram_traffic.txt), or None when it has not been captured."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles", "dram_traffic.txt")
    try:
        with open(path) as fh:
            for line in fh:
                parts = line.split()
                if len(parts) == 2 and not line.startswith("#") and parts[0] == kernel:
                    return float(parts[1])
    except OSError:
        pass
    return None


# ------------------------------------------------------------ reference arm
#
# The reference's CPU step is single-threaded (a JavaScript worker), so the
# arm runs one copy of the FP64 restatement per host core, in processes
# started with `spawn` (no GPU is touched): replicas of the whole scene for
# the plain form, a share of the scenes per process for the batched and
# differentiable forms.  Throughput = the work of all processes / the wall
# time of the step in which they all run.

def _reference_plan(workload: str):
    """(jobs, meta): jobs = [(kind, payload)] of the whole workload, built
    identically in every process."""
    from mpm_b200 import calculate_mpm_cfl_microsteps, derive_mpm_mls_gpu_cfl_bounds
    if workload in ("dam-break-1m", "si-tank"):
        particles, config, gravity, meta = build_workload(workload)
        bounds = derive_mpm_mls_gpu_cfl_bounds(particles, config)
        plan = calculate_mpm_cfl_microsteps(meta["macro_dt"], config["grid"]["cellSize"], bounds["waveSpeedBound"],
                                            max(bounds["velocityBound"], 5.0), BATCHED_MAX_MICROSTEPS)
        micro = float(np.float32(plan["microDt"]))
        return [("step", (particles, dict(config, dt=micro, gravity=gravity)))], dict(meta, micro_dt=micro)
    if workload == "batched-512":
        from mpm_b200.scenes import BATCHED_TANK_GRAVITY, create_batched_tank_scenes
        scenes = create_batched_tank_scenes()
        jobs = []
        for particles, config in scenes:
            bounds = derive_mpm_mls_gpu_cfl_bounds(particles, config)
            plan = calculate_mpm_cfl_microsteps(MACRO_DT, config["grid"]["cellSize"], bounds["waveSpeedBound"],
                                                _batched_bound(bounds["velocityBound"], MACRO_DT, BATCHED_TANK_GRAVITY),
                                                BATCHED_MAX_MICROSTEPS)
            jobs.append(("step", (particles, dict(config, dt=float(np.float32(plan["microDt"])),
                                                  gravity=BATCHED_TANK_GRAVITY))))
        return jobs, {"workload": "batched: 512 independent SI Tait water tanks (see the b200 arm)",
                      "scenes": len(scenes), "particles": int(sum(len(p) for p, _ in scenes))}
    if workload == "adjoint-64":
        from mpm_b200.adjoint import fixed_cfl_dt
        from mpm_b200.scenes import ADJOINT_GRAVITY, create_adjoint_scenes
        jobs = []
        for particles, config, target in create_adjoint_scenes():
            dt = fixed_cfl_dt(particles, config, 90.0, 0.0)
            dt = float(np.float32(fixed_cfl_dt(particles, config, 90.0, ADJOINT_SUBSTEPS * dt)))
            jobs.append(("adjoint", (particles, config, target, dt)))
        return jobs, {"workload": "differentiable form: 64 scenes (see the b200 arm)", "scenes": len(jobs)}
    raise SystemExit(f"unknown workload {workload}")


def _job_cost(kind, payload) -> int:
    particles, config = payload[0], payload[1]
    from mpm_b200.sharding import scene_cost
    return scene_cost(len(particles), config["grid"]["cellsX"], config["grid"]["cellsY"])


def _reference_share(workload: str, worker: int, workers: int):
    """The jobs of process `worker`: the whole scene for the plain form (a
    replica), its cost-balanced share of the scenes otherwise."""
    jobs, _ = _reference_plan(workload)
    from oracle import OracleState
    from mpm_b200.sharding import shard_by_cost
    mine = []
    if len(jobs) == 1:
        picked = jobs
    else:
        share = shard_by_cost([_job_cost(kind, payload) for kind, payload in jobs], workers)[worker]
        picked = [jobs[k] for k in share]
    for kind, payload in picked:
        if kind == "step":
            particles, cfg = payload
            mine.append((kind, (OracleState(particles, cfg), cfg, len(particles))))
        else:
            mine.append((kind, payload))
    return mine


def _adjoint_inputs(particles, config, target, dt):
    from mpm_b200.layout import validate_mpm_mls_gpu_input
    from mpm_b200.scenes import ADJOINT_GRAVITY
    pk = validate_mpm_mls_gpu_input(particles, config).packed_particles
    liquid = pk[:, 13].view(np.uint32) == 2
    pk64 = pk.astype(np.float64)
    water, solid = pk64[liquid][0], pk64[~liquid][0]
    scene = {"cells_x": config["grid"]["cellsX"], "cells_y": config["grid"]["cellsY"],
             "dx": config["grid"]["cellSize"], "dt": dt, "gx": ADJOINT_GRAVITY["x"], "gy": ADJOINT_GRAVITY["y"],
             "solid_mass": float(np.float32(config["particleMass"])), "wall_friction": config["wallFriction"],
             "rho": float(water[16]), "gamma": float(water[18]), "tait": float(water[14]),
             "lambda_s": float(solid[14]), "mu_s": float(solid[15])}
    return (scene, pk64[:, 0:2], pk64[:, 2:4], pk64[:, 4:8], pk64[:, 8:12], pk64[:, 17], liquid.astype(np.int32),
            np.asarray(target, np.float32).astype(np.float64))


def _reference_sample(share, substeps: int):
    """One timed sample of a process's share: (seconds, particle-substeps)."""
    from oracle import adjoint_fp64
    work, t0 = 0, time.perf_counter()
    for kind, payload in share:
        if kind == "step":
            state, cfg, n = payload
            state.run(cfg, substeps)
            work += n * substeps
        else:
            particles, config, target, dt = payload
            adjoint_fp64(*_adjoint_inputs(particles, config, target, dt), substeps)
            work += len(particles) * substeps
    return time.perf_counter() - t0, work


def _reference_process(conn, workload: str, worker: int, workers: int):
    """A reference process: builds its share, then answers each step request
    (substeps) with (seconds, work) until it receives None."""
    try:
        share = _reference_share(workload, worker, workers)
        conn.send("ready")
        while True:
            substeps = conn.recv()
            if substeps is None:
                break
            conn.send(_reference_sample(share, substeps))
    except Exception as exc:  # reported to the parent, which fails the run
        conn.send(("error", repr(exc)))
    finally:
        conn.close()


def _reference_workers(workload: str, jobs: int) -> int:
    """One process per host core (at most one per scene when the workload
    has several), within the host memory (about 1 GB per replica of the
    1M-particle scene)."""
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    workers = min(cores, jobs) if jobs > 1 else cores
    if workload == "dam-break-1m":
        try:
            import psutil
            workers = min(workers, max(1, int(psutil.virtual_memory().available // (1 << 30)) - 4))
        except ImportError:
            pass
    return max(1, workers)


def run_reference(args):
    rank, _, world = _rank_info()
    if rank != 0:
        return
    import multiprocessing
    jobs, meta = _reference_plan(args.workload)
    workers = _reference_workers(args.workload, len(jobs))
    substeps = args.reference_substeps
    ctx = multiprocessing.get_context("spawn")
    pipes, procs = [], []
    for k in range(workers):
        parent, child = ctx.Pipe()
        proc = ctx.Process(target=_reference_process, args=(child, args.workload, k, workers), daemon=True)
        proc.start()
        child.close()
        pipes.append(parent)
        procs.append(proc)
    total_work, total_s = 0, 0.0
    try:
        for conn in pipes:
            msg = conn.recv()
            if msg != "ready":
                raise SystemExit(f"reference process failed: {msg}")
        for step in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            for conn in pipes:
                conn.send(substeps)
            results = [conn.recv() for conn in pipes]
            wall = time.perf_counter() - t0
            for r in results:
                if not isinstance(r, tuple) or r[0] == "error":
                    raise SystemExit(f"reference process failed: {r}")
            if step >= args.warmup:
                total_work += sum(w for _, w in results)
                total_s += wall
    finally:
        for conn in pipes:
            try:
                conn.send(None)
            except OSError:
                pass
        for proc in procs:
            proc.join(timeout=30)
    value = total_work / total_s
    adjoint = args.workload == "adjoint-64"
    unit = "particle-substeps/s (adjoint)" if adjoint else UNIT
    what = {"dam-break-1m": f"{workers} replicas of the full scene, {substeps} substeps each per step",
            "si-tank": f"{workers} replicas of the full scene, {substeps} substeps each per step",
            "batched-512": f"the 512 scenes shared by {workers} processes, {substeps} substeps of each scene per step",
            "adjoint-64": f"the 64 scenes shared by {workers} processes, {substeps} forward + adjoint substeps of "
                          "each scene per step (FP64 adjoint, oracle/adjoint_fp64.c)"}[args.workload]
    sample = (f"{what}; C FP64 restatement (oracle/), one single-threaded process per host core, "
              f"{total_s:.1f} s timed")
    line = {"metric": METRIC, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_s * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded scenes)",
            "impl": "reference", "config": dict(meta, p2g="CPU scatter (stepMpm restatement)", processes=workers),
            "cpu_baseline": {"value": value, "unit": unit, "cores": workers, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


BATCHED_MAX_MICROSTEPS = 4096
PLAIN_SAMPLE_SCENES = 16


def _batched_bound(velocity, macro_dt, gravity):
    from mpm_b200.cfl_bounds import calculate_mpm_cfl_velocity_bound
    return calculate_mpm_cfl_velocity_bound(velocity, macro_dt, math.hypot(gravity["x"], gravity["y"]), 0, 0, 0, 0)


def plain_per_scene(scenes, gravity, macro_dt, device):
    """The plain form on the same scenes: each of the first
    PLAIN_SAMPLE_SCENES scenes alone in its own solver (one macrostep of warm
    up, then one timed macrostep through the same adaptive loop)."""
    from mpm_b200 import calculate_mpm_cfl_microsteps, create_mpm_mls_gpu_solver
    work = device_ms = 0.0
    for particles, config in scenes[:PLAIN_SAMPLE_SCENES]:
        solver = create_mpm_mls_gpu_solver(particles, config, device=device)
        try:
            velocity = solver.cfl_bounds["velocityBound"]
            for timed in (False, True):
                bound = max(_batched_bound(velocity, macro_dt, gravity), solver._last_scheduled_velocity_bound or 0.0)
                plan = calculate_mpm_cfl_microsteps(macro_dt, config["grid"]["cellSize"],
                                                    solver.cfl_bounds["waveSpeedBound"], bound, BATCHED_MAX_MICROSTEPS)
                solver.device_ms_total = 0.0
                solver.committed_microsteps_total = 0
                m = solver.step_cfl_batch_adaptive(1, macro_dt, plan, bound, BATCHED_MAX_MICROSTEPS, gravity)
                velocity = m["recommendedVelocityBound"]
            work += len(particles) * solver.committed_microsteps_total
            device_ms += solver.device_ms_total
        finally:
            solver.dispose()
    return work / (device_ms * 1e-3)


def _init_ranks():
    """(dist or None, rank, local_rank, world): the NCCL process group of a
    multi-rank run (short timeout), the rank's device made current."""
    rank, local_rank, world = _rank_info()
    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local_rank)
    return dist, rank, local_rank, world


def _finish_ranks(dist):
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_b200_batched(args):
    dist, rank, local_rank, world = _init_ranks()
    line = measure_batched(args.steps, args.warmup, args.cfl_recovery_factor, args.cfl_plan_margin, dist, rank,
                           local_rank, world)
    _finish_ranks(dist)
    if rank == 0:
        print(json.dumps(line), flush=True)


def measure_batched(steps, warmup, recovery_factor, plan_margin, dist, rank, local_rank, world):
    """The batched form: 512 independent SI Tait water tanks in one solver, one
    step = one 1/240 s macrostep of every scene through the per-scene
    adaptive CFL loop (MpmBatchedGpuSolver.step_cfl_batch_adaptive).  Returns
    the bench line of the form (`steps` timed after `warmup`)."""
    import torch
    from mpm_b200 import create_mpm_batched_gpu_solver
    from mpm_b200.scenes import BATCHED_TANK_GRAVITY, batched_tank_scene_specs, create_batched_tank_scenes
    from mpm_b200.sharding import scene_cost, shard_by_cost
    # 512 scenes per GPU: the world's 512 x N seeded scenes bin-packed over the
    # ranks by cost (particles + halo nodes), every rank computing the same split
    specs = batched_tank_scene_specs(count=512 * world)
    share = shard_by_cost([scene_cost(n, side, side) for n, side in specs], world)[rank]
    scenes = create_batched_tank_scenes(indices=share)
    gravity = BATCHED_TANK_GRAVITY
    macro_dt = MACRO_DT
    batch = create_mpm_batched_gpu_solver(scenes, device=local_rank)
    n_total = int(batch.particle_counts.sum())
    velocity = [b["velocityBound"] for b in batch.cfl_bounds]

    batch.recovery_bound_factor = recovery_factor

    def one_step():
        nonlocal velocity
        bounds = [_batched_bound(v, macro_dt, gravity) * plan_margin for v in velocity]
        results = batch.step_cfl_batch_adaptive(macro_dt, bounds, BATCHED_MAX_MICROSTEPS, gravity)
        velocity = [r["recommendedVelocityBound"] for r in results]
        return results

    one_step()
    # the project's launch-shape tuner, state restored (skipped for profiling runs)
    shape = batch.autotune(substeps=4) if AUTOTUNE else dict(batch.substep_variant(), **batch.launch_shape())
    for _ in range(warmup - 1):
        one_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    batch.device_ms_total = 0.0
    batch.committed_particle_substeps = 0
    wall = 0.0
    submits = retries = 0
    for _ in range(steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        results = one_step()
        wall += time.perf_counter() - t0
        submits += 1 + max(r["retryCount"] for r in results)
        retries += sum(r["retryCount"] for r in results)
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    (device_s, wall), (work,) = reduce_over_ranks(dist, f"cuda:{local_rank}", [batch.device_ms_total / 1e3, wall],
                                                  [batch.committed_particle_substeps])
    value = work / device_s
    e2e_value = work / wall

    # kernel-by-kernel timing of real substeps of every scene at the smallest
    # microstep dt of the batch, right after the timed region
    from mpm_b200 import calculate_mpm_cfl_microsteps
    dt = min(calculate_mpm_cfl_microsteps(macro_dt, c["grid"]["cellSize"], b["waveSpeedBound"],
                                          _batched_bound(v, macro_dt, gravity), BATCHED_MAX_MICROSTEPS)["microDt"]
             for (_, c), b, v in zip(scenes, batch.cfl_bounds, velocity))
    prof_steps = 8
    prof = batch.profile_substeps(prof_steps, dt, gravity)
    active = batch.count_active_nodes()
    total_ms = sum(ms for ms, _ in prof.values())
    dominant = max(prof, key=lambda k: prof[k][0])
    dom_ms, dom_launches = prof[dominant]
    dom_bytes = kernel_bytes(dominant, n_total, active)
    peak, peak_kind = _peaks()
    achieved = dom_bytes / (dom_ms / dom_launches * 1e-3) / 1e9
    substep_bytes = n_total * 104.0 + float(sum(active)) * 64.0
    substep_ms = total_ms / prof_steps
    launches_per_substep = sum(l for _, l in prof.values()) / prof_steps
    plain = plain_per_scene(scenes, gravity, macro_dt, local_rank) if rank == 0 else None
    counts = batch.particle_counts
    sides = [c["grid"]["cellsX"] for _, c in scenes]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": warmup,
        "ms_per_step": device_s * 1e3 / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scenes, no dataset)",
        "config": {"workload": "batched: 512 independent SI Tait water tanks (0.2 m box, rho 1000, gamma 7, "
                               "c 20 m/s), N log-uniform in 1k-64k, S x S grids with S uniform in 64-512, "
                               "macrostep 1/240 s, per-scene adaptive CFL 0.3",
                   "scenes": len(scenes), "particles": n_total, "particles_range": [int(counts.min()),
                                                                                   int(counts.max())],
                   "grid_sides_range": [min(sides), max(sides)], "macro_dt": macro_dt, "courant": 0.3,
                   "p2g": "gather", "parallelism": f"scene shards x{world} (512 x {world} scenes bin-packed by cost over the GPUs)",
                   "l2": "inputs larger than L2 (every scene's state, about 0.8 GB)",
                   "committed_particle_substeps": work, "submits": submits, "retries": retries,
                   "launch_shape": shape,
                   "cfl_policy": {"recovery_factor": recovery_factor, "plan_margin": plan_margin,
                                  "scene_macrosteps_per_device_s": world * len(scenes) * steps / device_s},
                   "plain_per_scene": {"value": plain, "unit": UNIT,
                                       "sample": f"the first {PLAIN_SAMPLE_SCENES} scenes, each alone in its own "
                                                 "solver, one timed macrostep each"}},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": submits * len(scenes) * 160 // steps,
                "d2h_bytes_per_step": submits * len(scenes) * 256 // steps,
                "path": "Python host MpmBatchedGpuSolver.step_cfl_batch_adaptive -> C ABI"},
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind, "traffic": dram_traffic(dominant + "@batched"),
                     "algorithmic_bytes_per_launch": dom_bytes, "avg_launch_ms": dom_ms / dom_launches,
                     "kernel_share": dom_ms / total_ms,
                     "substep": {"algorithmic_bytes": substep_bytes, "ms": substep_ms,
                                 "achieved_gbs": substep_bytes / (substep_ms * 1e-3) / 1e9,
                                 "frac": substep_bytes / (substep_ms * 1e-3) / 1e9 / peak},
                     "active_channel_nodes": list(active),
                     "kernels_ms_per_substep": {k: v[0] / prof_steps for k, v in prof.items()}},
        "clocks": clock_info,
        "gpu_launches": int(round(launches_per_substep * (work / max(1, n_total)))) if n_total else 0,
    }
    batch.dispose()
    return line


ADJOINT_SUBSTEPS = 200
ADJOINT_CHECKPOINT_EVERY = 20
# algorithmic bytes per particle and backward substep: the segment recompute
# (P2G reads x, v, C, F: 48 B; G2P reads x, F: 24 B, writes x, v, C, F: 48 B),
# the G2P adjoint (reads x, F and the output adjoint: 72 B, writes the G2P
# parts: 24 B) and the fused grid + P2G adjoint (reads x, v, C, F and the G2P
# parts: 72 B, writes the input adjoint: 48 B)
ADJOINT_BYTES_PER_PARTICLE = 48 + 24 + 48 + 72 + 24 + 72 + 48


def run_b200_adjoint(args):
    dist, rank, local_rank, world = _init_ranks()
    line = measure_adjoint(args.steps, args.warmup, dist, rank, local_rank, world)
    _finish_ranks(dist)
    if rank == 0:
        print(json.dumps(line), flush=True)


def measure_adjoint(steps_timed, warmup, dist, rank, local_rank, world, full_tape=True):
    """The differentiable form: 64 scenes of 12,288 Tait water + 4,096
    fixed-corotated particles on 256x256 grids, 200 substeps at each scene's
    fixed CFL dt, checkpoints every 20; one step = one forward pass (loss)
    and one backward pass (gradients wrt initial velocities and the scenes'
    Tait coefficient, lambda, mu).  Returns the bench line of the form."""
    import torch
    from mpm_b200 import create_mpm_batched_gpu_solver
    from mpm_b200.adjoint import create_mpm_adjoint_engine, fixed_cfl_dt
    from mpm_b200.scenes import ADJOINT_GRAVITY, create_adjoint_scenes
    scenes = create_adjoint_scenes(first=rank * 64)  # each rank its own shard of scenes
    gravity = ADJOINT_GRAVITY
    steps = ADJOINT_SUBSTEPS
    dts = []
    for p, c, _ in scenes:
        dt = fixed_cfl_dt(p, c, 90.0, 0.0)
        dts.append(float(np.float32(fixed_cfl_dt(p, c, 90.0, steps * dt))))
    targets = np.concatenate([t for _, _, t in scenes]).astype(np.float32)
    engine = create_mpm_adjoint_engine([(p, c) for p, c, _ in scenes], gravity, device=local_rank)
    n = int(engine.particle_counts.sum())

    def one_step():
        loss = engine.forward(steps, dts, targets, ADJOINT_CHECKPOINT_EVERY)
        gv, gp = engine.backward()
        return loss, gv, gp

    for _ in range(warmup):
        one_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    fwd = bwd = wall = 0.0
    for _ in range(steps_timed):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        loss, gv, gp = one_step()
        wall += time.perf_counter() - t0
        f, b = engine.last_ms()
        fwd += f
        bwd += b
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    # the same passes with the whole trajectory on the tape (one segment of
    # 200 substeps: every substep's state and node sums stay in HBM, the
    # backward pass recomputes nothing); after the timed region
    tape_fwd = tape_bwd = 0.0
    for k in range(2 if full_tape else 0):
        engine.forward(steps, dts, targets, steps)
        engine.backward()
        if k == 1:
            tape_fwd, tape_bwd = engine.last_ms()
    nodes = sum((c["grid"]["cellsX"] + 3) * (c["grid"]["cellsY"] + 3) for _, c, _ in scenes)
    tape_gb = steps * (n * 48 + nodes * 32) / 1e9
    engine.dispose()
    (fwd_s, bwd_s, wall, tape_fwd, tape_bwd), _ = reduce_over_ranks(
        dist, f"cuda:{local_rank}", [fwd / 1e3, bwd / 1e3, wall, tape_fwd, tape_bwd], [])
    # the default solver stepping the same scenes with the same dt
    batch = create_mpm_batched_gpu_solver([(p, c) for p, c, _ in scenes], device=local_rank)
    batch.step_batch([steps] * len(scenes), dts, gravity)
    batch.last_batch_device_ms()
    batch.step_batch([steps] * len(scenes), dts, gravity)
    plain_ms = batch.last_batch_device_ms()
    batch.dispose()
    work = world * n * steps * steps_timed
    value = work / bwd_s
    peak, peak_kind = _peaks()
    achieved = ADJOINT_BYTES_PER_PARTICLE * n * steps * steps_timed / bwd_s / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "particle-substeps/s (adjoint)", "n_gpus": world,
        "steps": steps_timed, "warmup": warmup, "ms_per_step": (fwd_s + bwd_s) * 1e3 / steps_timed,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded scenes, no dataset)",
        "config": {"workload": "differentiable form: 64 scenes of 12,288 Tait water + 4,096 fixed-corotated "
                               "(lambda 20, mu 10) particles on 256x256 grids (cellSize 10, gravity 90), initial "
                               "velocities N(0, 10^2), 200 substeps at each scene's fixed CFL dt, checkpoints every "
                               "20, loss sum |x(T) - target|^2 against a seeded displacement field",
                   "scenes": len(scenes), "particles": n, "substeps": steps,
                   "checkpoint_every": ADJOINT_CHECKPOINT_EVERY,
                   "parallelism": f"scene shards x{world} (64 different scenes per GPU)",
                   "l2": "inputs larger than L2 (1M particles' state and 64 grids of 67,081 nodes)",
                   "adjoint_forward_ratio": bwd_s / fwd_s,
                   "adjoint_over_default_forward": (bwd_s / steps_timed) / (plain_ms * 1e-3),
                   "forward_ms": fwd_s * 1e3 / steps_timed, "backward_ms": bwd_s * 1e3 / steps_timed,
                   "default_solver_forward_ms": plain_ms,
                   "full_tape": None if not full_tape else {
                                 "adjoint_forward_ratio": tape_bwd / tape_fwd, "forward_ms": tape_fwd,
                                 "backward_ms": tape_bwd, "tape_gb": tape_gb,
                                 "note": "every substep's state and node sums kept in HBM (checkpoint_every = "
                                         "substeps): no recompute; measured once after the timed region"}},
        "e2e": {"value": work / wall, "unit": "particle-substeps/s (forward + adjoint)",
                "h2d_bytes_per_step": n * 8 + len(scenes) * 4,
                "d2h_bytes_per_step": n * 8 + len(scenes) * (3 * 8 + 8),
                "path": "Python host MpmAdjointEngine.forward + backward -> C ABI"},
        "roofline": {"bound": "hbm", "kernel": "backward pass (segment recompute + G2P adjoint + grid/P2G adjoint)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "traffic": None,
                     "algorithmic_bytes_per_particle_substep": ADJOINT_BYTES_PER_PARTICLE},
        "clocks": clock_info,
        "gpu_launches": int(steps_timed * (2 * steps + 4 * steps + 1)),
    }
    return line


def run_b200(args):
    dist, rank, local_rank, world = _init_ranks()
    import torch
    from mpm_b200 import create_experimental_mpm_mls_atomic_gpu_solver, create_mpm_mls_gpu_solver

    particles, config, gravity, meta = build_workload(args.workload)
    if args.p2g == "fixed":
        solver = create_experimental_mpm_mls_atomic_gpu_solver(particles, config, device=local_rank,
                                                               fixed_point_shift=args.fixed_shift)
    else:
        solver = create_mpm_mls_gpu_solver(particles, config, device=local_rank)
    n = len(particles)
    macro_dt = meta["macro_dt"]
    max_micro = meta.get("max_microsteps", MAX_MICROSTEPS)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local_rank}")
    velocity = solver.cfl_bounds["velocityBound"]

    def one_step():
        nonlocal velocity
        plan, bound = plan_macrostep(solver, config, velocity, macro_dt, gravity, max_micro)
        m = solver.step_cfl_batch_adaptive(1, macro_dt, plan, bound, max_micro, gravity)
        velocity = m["recommendedVelocityBound"]
        return m

    one_step()
    shape = None
    if args.p2g == "gather":
        shape = solver.autotune(substeps=4) if AUTOTUNE else dict(solver.substep_variant(), **solver.launch_shape())
    for _ in range(args.warmup - 1):
        one_step()
    clocks = ClockSampler(local_rank)
    clocks.start()
    # the timed region (K steps between barriers and synchronizes) is taken
    # args.repeats times back to back; the line reports the repeat with the
    # median device throughput and lists them all
    repeats = []
    for _ in range(args.repeats):
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        solver.device_ms_total = 0.0
        solver.committed_microsteps_total = 0
        wall = 0.0
        retries = 0
        h2d = d2h = 0
        for _ in range(args.steps):
            flush.zero_()  # L2 flush between timed steps (outside the timed batches)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            m = one_step()
            wall += time.perf_counter() - t0
            retries += m["retryCount"]
            batches = 1 + m["retryCount"]
            h2d += batches * 160  # StepParams upload per batch
            d2h += batches * 40   # compact speed / progress / status readback
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        (r_device_s, r_wall), (r_substeps,) = reduce_over_ranks(
            dist, f"cuda:{local_rank}", [solver.device_ms_total / 1e3, wall], [solver.committed_microsteps_total])
        repeats.append({"device_s": r_device_s, "wall_s": r_wall, "substeps": int(r_substeps), "retries": retries,
                        "h2d": h2d, "d2h": d2h,
                        "value": n * r_substeps / r_device_s, "e2e": n * r_substeps / r_wall})
    clock_info = clocks.stop()
    chosen = sorted(repeats, key=lambda r: r["value"])[len(repeats) // 2]
    device_s, wall, retries, h2d, d2h = (chosen["device_s"], chosen["wall_s"], chosen["retries"], chosen["h2d"],
                                         chosen["d2h"])
    substeps = chosen["substeps"]  # summed over ranks
    value = n * substeps / device_s
    e2e_value = n * substeps / wall

    # roofline: kernel-by-kernel timing of real substeps right after the timed region
    plan, bound = plan_macrostep(solver, config, velocity, macro_dt, gravity, max_micro)
    from mpm_b200.cfl import calculate_mpm_cfl_velocity_limit
    limit = calculate_mpm_cfl_velocity_limit(config["grid"]["cellSize"], solver.cfl_bounds["waveSpeedBound"],
                                             plan["microDt"])
    prof = solver.profile_substeps(plan["stepCount"], plan["microDt"], gravity, velocity_limit=limit)
    active = solver.count_active_nodes()
    total_ms = sum(ms for ms, _ in prof.values())
    dominant = max(prof, key=lambda k: prof[k][0])
    dom_ms, dom_launches = prof[dominant]
    dom_bytes = kernel_bytes(dominant, n, active)
    peak, peak_kind = _peaks()
    achieved = dom_bytes / (dom_ms / dom_launches * 1e-3) / 1e9
    substep_bytes = n * 104.0 + float(sum(active)) * 64.0
    substep_ms = total_ms / plan["stepCount"]
    gpu_launches = 0
    launches_per_substep = sum(l for _, l in prof.values()) / plan["stepCount"]
    gpu_launches = int(round(launches_per_substep * substeps / world)) if substeps else 0
    substeps_rank = substeps // world

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": device_s * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene, no dataset)",
        "config": dict(meta, p2g=args.p2g, parallelism=f"replicas x{world}", l2="flushed (512 MiB write) "
                       "between timed steps", committed_substeps=substeps_rank, retries=retries, launch_shape=shape,
                       substeps_per_step=substeps_rank / args.steps,
                       repeats={"count": args.repeats, "reported": "median by value",
                                "values": [r["value"] for r in repeats], "e2e": [r["e2e"] for r in repeats]}),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps,
                "path": "Python host mirror of MpmMlsGpuSolver.stepCflBatchAdaptive -> C ABI"},
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     # the committed capture is of the 1M dam break
                     "traffic": dram_traffic(dominant) if args.workload == "dam-break-1m" else None,
                     "algorithmic_bytes_per_launch": dom_bytes, "avg_launch_ms": dom_ms / dom_launches,
                     "kernel_share": dom_ms / total_ms,
                     "substep": {"algorithmic_bytes": substep_bytes, "ms": substep_ms,
                                 "achieved_gbs": substep_bytes / (substep_ms * 1e-3) / 1e9,
                                 "frac": substep_bytes / (substep_ms * 1e-3) / 1e9 / peak},
                     "active_channel_nodes": list(active),
                     "kernels_ms_per_substep": {k: v[0] / plan["stepCount"] for k, v in prof.items()}},
        "clocks": clock_info,
        "gpu_launches": gpu_launches,
    }
    if args.p2g == "fixed" and "k_prepare_scatter" in prof:
        # the fixed-point scatter's int32 atomics: 9 nodes x 4 words per
        # liquid particle (mass, momentum, volume), 9 x 3 per solid one
        packed, _ = solver.read_particles_packed()
        model = packed[:, 13].view(np.uint32)
        liquid = int(np.count_nonzero((model == 2) | (model == 3)))
        per_substep = 36 * liquid + 27 * (len(model) - liquid)
        ms, launches = prof["k_prepare_scatter"]
        line["atomics"] = {"kernel": "k_prepare_scatter", "per_substep": per_substep,
                           "per_s": per_substep / (ms / launches * 1e-3),
                           "per_particle": {"liquid": 36, "solid": 27}}
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(particles, config, gravity, float(np.float32(plan["microDt"])),
                                            args.cpu_substeps)
    solver.dispose()
    del flush
    torch.cuda.empty_cache()
    if args.workload == "dam-break-1m" and args.p2g == "gather" and not args.no_legs:
        # the metric's other two numbers, after the headline's timed region:
        # the batched form (and the same scenes one solver each) and the
        # differentiable form's adjoint/forward time ratio, each with fewer
        # steps than the headline (stated in the leg)
        b = measure_batched(args.leg_steps, 3, 1.25, 1.0, dist, rank, local_rank, world)
        plain = b["config"]["plain_per_scene"]["value"]
        line["batched"] = {"value": b["value"], "unit": UNIT, "plain_per_scene": plain,
                           "batched_over_plain": None if not plain else b["value"] / plain,
                           "steps": b["steps"], "warmup": b["warmup"], "e2e": b["e2e"]["value"],
                           "workload": b["config"]["workload"], "scenes": b["config"]["scenes"],
                           "particles": b["config"]["particles"], "retries": b["config"]["retries"],
                           "launch_shape": b["config"]["launch_shape"],
                           "roofline": {k: b["roofline"][k] for k in ("kernel", "achieved", "frac", "substep")},
                           "clocks": b["clocks"]}
        a = measure_adjoint(1, 1, dist, rank, local_rank, world, full_tape=False)
        cfg = a["config"]
        line["adjoint"] = {"forward_ms": cfg["forward_ms"], "backward_ms": cfg["backward_ms"],
                           "adjoint_forward_ratio": cfg["adjoint_forward_ratio"],
                           "checkpoint_every": cfg["checkpoint_every"], "substeps": cfg["substeps"],
                           "default_solver_forward_ms": cfg["default_solver_forward_ms"],
                           "adjoint_over_default_forward": cfg["adjoint_over_default_forward"],
                           "value": a["value"], "unit": a["unit"], "steps": 1, "warmup": 1,
                           "workload": cfg["workload"], "clocks": a["clocks"]}
    _finish_ranks(dist)
    if rank == 0:
        print(json.dumps(line), flush=True)


PROFILE_CASES = ("batched", "dense", "adjoint")


def run_profile_case(name: str):
    """Small fixed cases for kernel profiling (ncu launch lists, a few hundred
    launches each); prints the device milliseconds of the last pass.

    batched: the 512 batched tanks, 2 x 4 substeps at the smallest CFL dt;
    dense:   the 64 of those tanks with the most particles per cell, likewise;
    adjoint: the 64 differentiable-form scenes, 2 x (40 forward + 40 backward).
    """
    from mpm_b200 import calculate_mpm_cfl_microsteps, create_mpm_batched_gpu_solver
    from mpm_b200.adjoint import create_mpm_adjoint_engine, fixed_cfl_dt
    from mpm_b200.scenes import (ADJOINT_GRAVITY, BATCHED_TANK_GRAVITY, create_adjoint_scenes,
                                  create_batched_tank_scenes)
    if name in ("batched", "dense"):
        scenes = create_batched_tank_scenes()
        if name == "dense":
            per_cell = np.array([len(p.px) / c["grid"]["cellsX"] ** 2 for p, c in scenes])
            scenes = [scenes[i] for i in np.argsort(per_cell)[-64:]]
        b = create_mpm_batched_gpu_solver(scenes)
        try:
            dt = min(calculate_mpm_cfl_microsteps(1 / 240, c["grid"]["cellSize"], bounds["waveSpeedBound"], 1.0,
                                                  4096)["microDt"] for (_, c), bounds in zip(scenes, b.cfl_bounds))
            for _ in range(2):
                b.step_batch([4] * len(scenes), [dt] * len(scenes), BATCHED_TANK_GRAVITY)
            print(f"{name}: 4 substeps of {len(scenes)} scenes", b.last_batch_device_ms(), "ms")
        finally:
            b.dispose()
        return
    scenes = create_adjoint_scenes()
    dts = [float(np.float32(fixed_cfl_dt(p, c, 90.0, 0.2))) for p, c, _ in scenes]
    targets = np.concatenate([t for _, _, t in scenes]).astype(np.float32)
    e = create_mpm_adjoint_engine([(p, c) for p, c, _ in scenes], ADJOINT_GRAVITY)
    try:
        for _ in range(2):
            e.forward(40, dts, targets, 20)
            e.backward()
        print("adjoint: 40 substeps of 64 scenes, forward / backward", e.last_ms(), "ms")
    finally:
        e.dispose()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", default="dam-break-1m",
                    choices=["dam-break-1m", "si-tank", "batched-512", "adjoint-64"])
    ap.add_argument("--p2g", choices=["gather", "fixed"], default="gather")
    ap.add_argument("--fixed-shift", type=int, default=16)
    ap.add_argument("--cpu-substeps", type=int, default=12)
    ap.add_argument("--reference-substeps", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--repeats", type=int, default=5, help="timed regions of K steps; the median is reported")
    ap.add_argument("--no-legs", action="store_true", help="skip the batched and adjoint legs of the default line")
    ap.add_argument("--leg-steps", type=int, default=3, help="timed macrosteps of the batched leg")
    ap.add_argument("--profile-case", choices=PROFILE_CASES, help="run a small fixed case for kernel profiling")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch variant (profiling runs: the tuner's trials distort under a profiler)")
    # the batched workload's adaptive CFL policy (the reference's: 1.25 and no margin)
    ap.add_argument("--cfl-recovery-factor", type=float, default=1.25)
    ap.add_argument("--cfl-plan-margin", type=float, default=1.0)
    args = ap.parse_args()
    global AUTOTUNE
    AUTOTUNE = not args.no_autotune
    if args.profile_case:
        run_profile_case(args.profile_case)
        return
    if args.warmup < 3:
        raise SystemExit("--warmup must be at least 3")
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched-512":
        run_b200_batched(args)
    elif args.workload == "adjoint-64":
        run_b200_adjoint(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
