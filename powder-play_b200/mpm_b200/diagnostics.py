"""Water diagnostics of the reference's SI performance experiment
(summarizeSiWater, src/lib/mpm/experiments/si-performance.ts:19-71), over
packed 20-word particle records as the solvers read them back.

areaRatio = sum(V_p det F_p) / reference area, its drift in percent, the
range of det F, the 95th percentile of the per-particle density error
100 |1 / det F - 1| (the reference's ceil(0.95 n) - 1 order statistic) and
the maximum speed.
"""
from __future__ import annotations

import math

import numpy as np

from .errors import RangeError


def summarize_si_water(packed: np.ndarray, reference_area: float) -> dict:
    if packed.shape[0] == 0 or not math.isfinite(reference_area) or reference_area <= 0:
        raise RangeError("Water diagnostics require particles and a positive reference area.")
    p = packed.astype(np.float64)
    F, C = p[:, 8:12], p[:, 4:8]
    pos, vel, volume = p[:, 0:2], p[:, 2:4], p[:, 17]
    det = F[:, 0] * F[:, 3] - F[:, 1] * F[:, 2]
    values = np.concatenate([F, C, pos, vel, volume[:, None]], axis=1)
    if not np.all(np.isfinite(values)) or not np.all(np.isfinite(det)) or np.any(det <= 0) or np.any(volume <= 0):
        raise RuntimeError("Non-finite or non-positive water state in SI diagnostics.")
    area = float(np.sum(volume * det))
    density_error = np.sort(100.0 * np.abs(1.0 / det - 1.0))
    p95 = float(density_error[math.ceil(0.95 * density_error.size) - 1])
    return {"areaRatio": area / reference_area, "areaDriftPercent": 100.0 * (area / reference_area - 1.0),
            "determinantMin": float(det.min()), "determinantMax": float(det.max()),
            "densityErrorPercentP95": p95, "maximumSpeed": float(np.max(np.hypot(vel[:, 0], vel[:, 1])))}
