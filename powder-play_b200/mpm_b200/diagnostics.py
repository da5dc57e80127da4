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


def summarize_dam_break_phase(packed: np.ndarray) -> dict:
    """Bulk state of one liquid of the two-phase dam break from its packed
    records: centre of mass and spread, mean specific kinetic energy, maximum
    speed, the runout front (99.9th percentile of x), the free surface (0.1st
    percentile of y, gravity +y) and the 5th / 95th percentiles of det F."""
    if packed.shape[0] == 0:
        raise RangeError("Dam-break diagnostics require particles.")
    p = packed.astype(np.float64)
    x, y, vx, vy = p[:, 0], p[:, 1], p[:, 2], p[:, 3]
    F = p[:, 8:12]
    det = F[:, 0] * F[:, 3] - F[:, 1] * F[:, 2]
    if not np.all(np.isfinite(p[:, 0:12])):
        raise RuntimeError("Non-finite state in dam-break diagnostics.")
    speed2 = vx * vx + vy * vy
    return {"cx": float(x.mean()), "cy": float(y.mean()), "sx": float(x.std()), "sy": float(y.std()),
            "ke": float(0.5 * speed2.mean()), "vmax": float(np.sqrt(speed2.max())),
            "front": float(np.quantile(x, 0.999)), "surface": float(np.quantile(y, 0.001)),
            "detP05": float(np.quantile(det, 0.05)), "detP95": float(np.quantile(det, 0.95))}
