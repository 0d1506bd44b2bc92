"""Host-side FP64 pupil helpers: Jones states and the open-frame throughput.

The device evaluates the pupil at every in-aperture point (csrc/pupil.cuh).
The host needs only what is per source point: the incoherent Jones states of
the vector model (expose/pupil.py:jones_states, :232-289) and the open-frame
("clear") throughput, which the reference accumulates from the DC bin of
every source point's pupil (expose/aerial_image.py:461-486).
"""

from __future__ import annotations

import math

import numpy as np

from .config import POLARISATIONS


def jones_states(polarisation: str, phi_source: float) -> list[tuple[float, float, float]]:
    """(Jx, Jy, weight) of each incoherent polarisation state of one source point."""
    p = polarisation.lower()
    if p == "x":
        return [(1.0, 0.0, 1.0)]
    if p == "y":
        return [(0.0, 1.0, 1.0)]
    if p == "te":
        return [(-math.sin(phi_source), math.cos(phi_source), 1.0)]
    if p == "tm":
        return [(math.cos(phi_source), math.sin(phi_source), 1.0)]
    if p in ("unpolarised", "unpolarized"):
        return [(1.0, 0.0, 0.5), (0.0, 1.0, 0.5)]
    raise ValueError(f"polarisation must be one of {list(POLARISATIONS)}, got '{polarisation}'")


def vector_coefficients(rho, phi, jx, jy, sin_theta_max, obliquity=True):
    """Image-space (Vx, Vy, Vz) of an entrance-pupil Jones vector (pupil.py:292-369)."""
    s2 = np.clip((np.asarray(rho, dtype=np.float64) * sin_theta_max) ** 2, 0.0, 1.0)
    ct, st = np.sqrt(1.0 - s2), np.sqrt(s2)
    cp, sp = np.cos(phi), np.sin(phi)
    es = -jx * sp + jy * cp
    ep = jx * cp + jy * sp
    v = np.stack([-es * sp + ep * ct * cp, es * cp + ep * ct * sp, -ep * st])
    return v * np.sqrt(ct) if obliquity else v


def clear_throughput(src, view, n_image: float, vector: bool, scale=None) -> float:
    """What an unpatterned mask images to, for one plane.

    Scalar: sum of the weights of source points whose pupil passes DC.
    Vector: sum over those points and their states of w * |V(DC)|^2.
    The DC test is the reference's exact one: rho = sqrt((0 - fsx)^2 +
    (0 - fsy)^2) / (NA / lambda) <= 1, in float64. ``scale`` (per source
    point): what the blank returns there, |r|^2 for a mirror (the
    reference's clear_scale, expose/aerial_image.py:431-438); None for a thin
    mask (1).
    """
    k_max = view.NA / view.wavelength
    gx = 0.0 - src.fx
    gy = 0.0 - src.fy
    rho = np.sqrt(gx ** 2 + gy ** 2) / k_max
    inside = rho <= 1.0
    if not vector:
        if scale is None:
            return float(np.sum(src.weight * inside.astype(np.float64)))
        return float(np.sum(src.weight * inside.astype(np.float64) * np.asarray(scale, dtype=np.float64)))
    total = 0.0
    phi = np.arctan2(gy, gx)
    stm = view.NA / n_image
    for s in np.nonzero(inside)[0]:
        for jx, jy, wp in jones_states(view.polarisation, float(src.phi[s])):
            V = vector_coefficients(rho[s], phi[s], jx, jy, stm, view.obliquity)
            cs = 1.0 if scale is None else float(scale[s])
            total += float(src.weight[s]) * wp * float(np.sum(V ** 2)) * cs
    return total
