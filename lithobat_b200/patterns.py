"""Synthetic mask generators (pixel transmittances) for tests and benchmarks.

``lines_and_spaces``, ``contact_array`` and ``to_attenuated_psm`` follow
``litho_sim.mask.patterns`` (:22-66, :69-107, :178-208). ``manhattan_clip``
is the seeded random layout clip of the batched workloads: a union of
axis-aligned, pixel-aligned rectangles.
"""

from __future__ import annotations

import numpy as np


def lines_and_spaces(n_pixels, pixel_size, pitch, cd, orientation="vertical"):
    coords = (np.arange(n_pixels) - n_pixels // 2) * pixel_size
    line = (np.mod(coords + pitch / 2, pitch) < cd).astype(np.float64)
    if orientation == "vertical":
        return np.tile(line[np.newaxis, :], (n_pixels, 1))
    if orientation == "horizontal":
        return np.tile(line[:, np.newaxis], (1, n_pixels))
    raise ValueError(f"orientation must be 'vertical' or 'horizontal', got '{orientation}'")


def contact_array(n_pixels, pixel_size, pitch_x, pitch_y, cd_x, cd_y=None):
    cd_y = cd_x if cd_y is None else cd_y
    coords = (np.arange(n_pixels) - n_pixels // 2) * pixel_size
    ox = (np.mod(coords + pitch_x / 2, pitch_x) < cd_x).astype(np.float64)
    oy = (np.mod(coords + pitch_y / 2, pitch_y) < cd_y).astype(np.float64)
    return np.outer(oy, ox)


def to_attenuated_psm(mask, transmission=0.06, phase_shift_deg=180.0):
    """1-regions become amplitude sqrt(T) with the phase shift; 0-regions clear."""
    ph = np.deg2rad(phase_shift_deg)
    return np.where(mask > 0.5, np.sqrt(transmission) * np.exp(1j * ph), 1.0 + 0.0j).astype(np.complex128)


def attenuated_psm_levels(mask, transmission=0.06, phase_shift_deg=180.0):
    """to_attenuated_psm as a level map: (index uint8, levels complex64 [2]),
    index 1 where the pattern is 1 (amplitude sqrt(T) e^{i phase}), 0 clear."""
    ph = np.deg2rad(phase_shift_deg)
    levels = np.array([1.0 + 0.0j, np.sqrt(transmission) * np.exp(1j * ph)], dtype=np.complex128)
    return (np.asarray(mask) > 0.5).astype(np.uint8), levels.astype(np.complex64)


def manhattan_clip(rng, n, pixel_size, n_rect=(20, 60), width_nm=(40.0, 200.0)):
    """Union of rng-drawn axis-aligned rectangles, 0/1 float64, pixel aligned."""
    m = np.zeros((n, n), dtype=np.float64)
    for _ in range(int(rng.integers(n_rect[0], n_rect[1] + 1))):
        w = max(1, int(round(rng.uniform(*width_nm) * 1e-9 / pixel_size)))
        h = max(1, int(round(rng.uniform(*width_nm) * 1e-9 / pixel_size)))
        x0, y0 = int(rng.integers(0, n)), int(rng.integers(0, n))
        m[y0:y0 + h, x0:x0 + w] = 1.0
    return m
