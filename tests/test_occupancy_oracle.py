"""The FP64 current-area oracle (oracle.current_area_fp64) pinned by the
known answers of src/lib/mpm/reference/occupancy.spec.ts, and the surface
status decoder (decodeSurfaceError, src/lib/mpm/kernels/solver.ts:208-224,
286-294)."""
import numpy as np
import pytest

from mpm_b200 import MpmMlsGpuSurfaceError
from mpm_b200.errors import decode_surface_error
from oracle import OracleError, current_area_fp64

IDENTITY = (1.0, 0.0, 0.0, 1.0)
WATER, OIL, POWDER = 0, 1, 2


def _field(particles, cells=8, cell_size=1.0):
    """particles: (x, y, volume, F, phase) tuples."""
    px = [p[0] for p in particles]
    py = [p[1] for p in particles]
    vol = [p[2] for p in particles]
    F = [p[3] for p in particles]
    phase = [p[4] for p in particles]
    return current_area_fp64(px, py, np.array(F, np.float64).reshape(-1, 4), vol, phase, cells, cells, cell_size)


def test_water_and_oil_are_separate_fields_and_non_liquids_are_ignored():
    # occupancy.spec.ts:63-99 (particleVolume 0.75 for the default-volume particle)
    water = (2.25, 3.75, 0.4, IDENTITY, WATER)
    default_water = (4.25, 2.75, 0.75, IDENTITY, WATER)
    oil = (2.25, 3.75, 0.2, (1.5, 0.0, 0.0, 1.0), OIL)
    powder = (6.25, 5.75, 0.75, IDENTITY, POWDER)
    combined = _field([water, default_water, oil, powder])
    water_only = _field([water, default_water])
    oil_only = _field([oil])
    assert not np.any(_field([powder]))
    assert np.array_equal(combined[..., 0], water_only[..., 0])
    assert np.array_equal(combined[..., 1], oil_only[..., 1])
    assert np.count_nonzero(combined.sum(axis=2)) > 9
    assert combined[..., 0].sum() > 0 and combined[..., 1].sum() > 0


def test_translation_moves_the_stencil_and_halo_nodes_are_kept():
    # occupancy.spec.ts:101-140
    base = _field([(2.25, 3.75, 0.5, IDENTITY, WATER)])
    moved = _field([(4.25, 4.75, 0.5, IDENTITY, WATER)])
    assert np.count_nonzero(base) == np.count_nonzero(moved) == 9
    assert np.array_equal(moved[1:, 2:], base[:-1, :-2])
    low = _field([(0.0, 0.0, 0.5, IDENTITY, WATER)])
    assert low[0, 0, 0] > 0  # node (-1, -1): halo
    assert low[1, 1, 0] > 0  # node (0, 0)
    high = _field([(8.0, 8.0, 0.5, IDENTITY, WATER)])
    assert high[10, 10, 0] > 0  # node (9, 9): halo
    assert high[9, 9, 0] > 0    # node (8, 8)


def test_occupancy_scales_with_the_determinant():
    # occupancy.spec.ts:142-157
    a = _field([(2.25, 3.75, 0.6, IDENTITY, WATER)])
    b = _field([(2.25, 3.75, 0.6, (2.0, 0.0, 0.0, 1.0), WATER)])
    assert np.count_nonzero(a) == np.count_nonzero(b)
    assert np.max(np.abs(b - 2 * a)) <= 1e-12


def test_water_and_oil_area_are_conserved_over_physical_and_halo_nodes():
    # occupancy.spec.ts:159-195: water 1.2 * 1.5 + 0.8 * 1.25 = 2.8, oil 0.75 * 0.5 + 0.4 * 2 = 1.175
    particles = [
        (0.0, 0.0, 1.2, (1.5, 0.0, 0.0, 1.0), WATER),
        (5.0, 7.0, 0.8, (1.0, 0.0, 0.0, 1.25), WATER),
        (12.0, 12.0, 0.75, (1.0, 0.0, 0.0, 0.5), OIL),
        (6.0, 3.0, 0.4, (2.0, 0.0, 0.0, 1.0), OIL),
        (2.25, 3.75, 1.0, IDENTITY, POWDER),
    ]
    f = _field(particles, cells=6, cell_size=2.0)
    assert abs(f[..., 0].sum() * 4 - 2.8) <= 1e-12
    assert abs(f[..., 1].sum() * 4 - 1.175) <= 1e-12
    halo = np.ones(f.shape[:2], bool)
    halo[1:-1, 1:-1] = False  # nodes -1 and cells + 1
    assert f[halo].sum() > 0


def test_invalid_inputs_are_rejected():
    # occupancy.spec.ts:197-232
    with pytest.raises(OracleError, match="grid domain"):
        _field([(-0.01, 2.0, 0.5, IDENTITY, WATER)])
    with pytest.raises(OracleError, match="determinant"):
        _field([(2.0, 2.0, 0.5, (-1.0, 0.0, 0.0, 1.0), WATER)])
    with pytest.raises(OracleError, match="cellSize"):
        _field([], cell_size=0.0)


def test_surface_flags_decode_like_the_reference():
    assert decode_surface_error([0] * 8) is None
    err = decode_surface_error([0] * 7 + [3])
    assert isinstance(err, MpmMlsGpuSurfaceError) and err.flags == 3
    assert str(err) == ("GPU free-surface occupancy generation failed (invalid free-surface bucket state; "
                        "invalid particle area or deformation determinant); particle state was not modified.")
    assert "status 0x8" in str(decode_surface_error([0] * 7 + [8]))
