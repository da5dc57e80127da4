"""The seeded batched-tank scene set (CPU): sizes, placement and seeding."""
import numpy as np

from mpm_b200.layout import validate_mpm_mls_gpu_input
from mpm_b200.scenes import create_batched_tank_scenes


def test_default_set_spans_the_stated_ranges():
    scenes = create_batched_tank_scenes()
    assert len(scenes) == 512
    counts = np.array([len(p.px) for p, _ in scenes])
    sides = np.array([c["grid"]["cellsX"] for _, c in scenes])
    assert counts.min() >= 1_000 and counts.max() <= 64_000
    assert sides.min() >= 64 and sides.max() <= 512
    assert 6e6 < counts.sum() < 10e6  # about 8M particles
    # log-uniform counts: the median sits near the geometric mean of the range
    assert 5_000 < np.median(counts) < 13_000
    for p, c in scenes:
        size = c["grid"]["cellsX"] * c["grid"]["cellSize"]
        assert c["grid"]["cellsX"] == c["grid"]["cellsY"]
        assert p.px.min() > 0 and p.px.max() < size and p.py.min() > 0 and p.py.max() < size


def test_scenes_are_seeded_and_validate():
    a = create_batched_tank_scenes(4, seed=99, particles=(500, 2000), sides=(32, 64))
    b = create_batched_tank_scenes(4, seed=99, particles=(500, 2000), sides=(32, 64))
    c = create_batched_tank_scenes(4, seed=100, particles=(500, 2000), sides=(32, 64))
    for (pa, ca), (pb, cb) in zip(a, b):
        assert ca == cb and np.array_equal(pa.px, pb.px) and np.array_equal(pa.py, pb.py)
        validate_mpm_mls_gpu_input(pa, ca)
    assert any(len(pa.px) != len(pc.px) or not np.array_equal(pa.px, pc.px) for (pa, _), (pc, _) in zip(a, c))
