"""Crack observables of the reference's crack script (TEST INFRASTRUCTURE ONLY).

Restates run_scripts/w_crack.py in numpy FP64: the projection of a stress
tensor on the normalised box rows (:119-122), the crack-mouth groups
(:125-133) and the crack length from the gap between the lowest atom above
and the highest below the crack plane in bins along the crack axis
(:136-188).
"""
from __future__ import annotations

import numpy as np


def project_to_lattice_axes(tensor, H):
    H = np.asarray(H, np.float64)
    axes = H / np.maximum(np.linalg.norm(H, axis=1, keepdims=True), 1e-12)
    return np.einsum("ai,ij,aj->a", axes, np.asarray(tensor, np.float64), axes)


def mouth_groups(vx, vy, x_center, y_center, half_length):
    mouth_x = x_center + half_length
    for xw in (0.8, 1.2, 1.8, 2.5):
        for yw in (0.8, 1.2, 1.8, 2.5):
            near = np.abs(vx - mouth_x) <= xw
            up = near & (vy > y_center) & ((vy - y_center) <= yw)
            lo = near & (vy < y_center) & ((y_center - vy) <= yw)
            if up.any() and lo.any():
                return up, lo
    raise ValueError("no crack-mouth atoms")


def crack_length(coords, x_unit, y_unit, y_plane, x_min, x_max, x_center, half_length, threshold, bins):
    bins = max(8, int(bins))
    span = max(1.0e-12, float(x_max - x_min))
    vx, vy = coords @ x_unit, coords @ y_unit
    idx = np.clip(np.floor((vx - x_min) / span * bins).astype(np.int64), 0, bins - 1)
    up_min = np.full(bins, np.inf)
    lo_max = np.full(bins, -np.inf)
    np.minimum.at(up_min, idx[vy > y_plane], vy[vy > y_plane])
    np.maximum.at(lo_max, idx[vy < y_plane], vy[vy < y_plane])
    with np.errstate(invalid="ignore"):
        gap = up_min - lo_max
        open_ = (gap >= threshold) & np.isfinite(gap)
    if not open_.any():
        return 0.0, 0.0
    width = span / bins
    centers = x_min + (np.arange(bins) + 0.5) * width
    seeds = np.nonzero(open_ & (centers >= x_center - half_length) & (centers <= x_center + half_length))[0]
    if len(seeds) == 0:
        return 0.0, 0.0
    left, right = int(seeds.min()), int(seeds.max())
    while left > 0 and open_[left - 1]:
        left -= 1
    while right < bins - 1 and open_[right + 1]:
        right += 1
    length = (right - left + 1) * width
    return float(length), float(max(0.0, length - 2.0 * half_length))
