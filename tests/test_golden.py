"""The committed golden fixtures (tests/golden/oracle_fp64.npz, written by
tests/golden/make_golden.py).

* CPU: each case's validated input still has the recorded digest, and the
  FP64 oracle still reproduces the recorded end state bit for bit;
* GPU: the CUDA path (gather and fixed-point P2G, through the C ABI) against
  the recorded end state, without running the oracle: every field within
  1e-3 absolute for the two small multi-model cases (the bound of
  src/lib/mpm/experiments/transfer-regression.ts:29); for the scenes,
  positions within 1e-3 cell sizes and velocities within 1e-3 * (1 + |v|).
"""
import importlib.util
import os

import numpy as np
import pytest

from helpers import packed_columns

HERE = os.path.dirname(os.path.abspath(__file__))
_spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
golden = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(golden)

CASES = golden.cases()
FIXTURE = np.load(golden.FIXTURE)


def test_fixture_holds_every_case():
    for name, case in CASES.items():
        assert f"{name}/input_sha256" in FIXTURE.files
        for field in case["fields"]:
            assert FIXTURE[f"{name}/{field}"].shape[0] == len(case["particles"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_the_golden_fixture(name):
    case = CASES[name]
    assert golden.input_digest(case) == str(FIXTURE[f"{name}/input_sha256"]), "the seeded input changed"
    out = golden.run_oracle(case)
    for field in case["fields"]:
        assert np.array_equal(out[field], FIXTURE[f"{name}/{field}"]), field


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["gather", "atomic"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_cuda_path_matches_the_golden_fixture(name, variant):
    from mpm_b200 import create_experimental_mpm_mls_atomic_gpu_solver, create_mpm_mls_gpu_solver
    case = CASES[name]
    factory = create_mpm_mls_gpu_solver if variant == "gather" else create_experimental_mpm_mls_atomic_gpu_solver
    solver = factory(case["particles"], case["config"])
    try:
        solver.step_batch(case["steps"], case["dt"], case["gravity"])
        packed, _ = solver.read_particles_packed()
    finally:
        solver.dispose()
    gpu = packed_columns(packed)
    ref = {field: FIXTURE[f"{name}/{field}"] for field in case["fields"]}
    if case["tolerance"] == "abs":
        for field in case["fields"]:
            err = float(np.max(np.abs(gpu[field] - ref[field])))
            assert err <= 1e-3, f"{name} {variant} {field}: {err}"
    else:
        dx = case["config"]["grid"]["cellSize"]
        pos_err = float(np.max(np.abs(gpu["position"] - ref["position"])))
        vel_err = float(np.max(np.abs(gpu["velocity"] - ref["velocity"]) / (1 + np.abs(ref["velocity"]))))
        assert pos_err <= 1e-3 * dx, f"{name} {variant}: position {pos_err}"
        assert vel_err <= 1e-3, f"{name} {variant}: velocity {vel_err}"
