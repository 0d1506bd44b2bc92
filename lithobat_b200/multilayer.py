"""The EUV mask blank as a Bragg mirror: ``mask_model="multilayer"``.

A reflective EUV mask is a Kirchhoff screen (the pattern) on a Mo/Si
multilayer mirror. Every diffraction order leaves the mask at its own angle,
and the mirror's complex reflection r(theta) varies over those angles, so the
Abbe sum multiplies each source point's spectrum by r evaluated per order
(expose/m3d/provider.py:MultilayerSpectra, :190-295). Here that multiply is
folded into the device pupil table: the table entry of a source point at
spectral bin k becomes P(k - f_s) * r(theta_s(k)), evaluated in FP64 on the
device (``k_pupil_table``), so imaging with the mirror costs exactly what thin
imaging costs.

Host side (this module):

* the stack description — :class:`Multilayer`, :class:`MaskStack`, the
  presets and the optical constants (expose/m3d/multilayer.py:46-152,
  stack.py:45-205, materials.py:58-102), same names, fields and errors;
* the mirror's reflection on an angle table, by the characteristic-matrix
  (Abeles) method for a planar film stack, solved for all table angles at
  once (coat/films.py:88-227 computes the same quantity one angle at a time);
  the scalar path takes the mean of the s and p reflections, tabulated as
  magnitude and unwrapped phase on 501 angles in [0, 25 deg]
  (provider.py:225-250);
* :func:`mask_side_sin_theta` (provider.py:72-126) and the per-source-point
  clear-field factor |r(specular)|^2 (provider.py:283-295).
"""

from __future__ import annotations

import json
import math
from dataclasses import dataclass, field
from typing import Any

import numpy as np

#: Mask-material refractive indices {wavelength [m]: {name: n + ik}}, positive
#: k absorbing; EUV values are 1 - delta + i beta (expose/m3d/materials.py:58-82).
MASK_MATERIALS: dict[float, dict[str, complex]] = {
    13.5e-9: {
        "vacuum": 1.0 + 0.0j,
        "Si": 0.99931 + 0.00182j,
        "Mo": 0.92108 + 0.00644j,
        "Ru": 0.88651 + 0.01710j,
        "TaBN": 0.94900 + 0.03120j,
        "TaBO": 0.97000 + 0.02500j,
        "Ta": 0.94270 + 0.04170j,
        "SiO2": 0.97800 + 0.01070j,
    },
    193e-9: {
        "vacuum": 1.0 + 0.0j,
        "air": 1.0 + 0.0j,
        "quartz": 1.5603 + 0.0j,
        "Cr": 0.84 + 1.65j,
        "CrON": 1.95 + 1.05j,
        "MoSi": 2.343 + 0.586j,
    },
}

REGIMES: tuple[str, ...] = ("euv_reflective", "duv_transmissive")

# Angle table of the reflection (expose/m3d/provider.py:59-64).
THETA_TABLE_MAX_DEG = 25.0
THETA_TABLE_N = 501


def mask_material(name: str, wavelength: float, tol: float = 1e-11) -> complex:
    """n + ik of a mask material at a tabulated wavelength (materials.py:85-102)."""
    for lam, table in MASK_MATERIALS.items():
        if abs(lam - wavelength) <= tol:
            if name not in table:
                raise KeyError(f"Unknown mask material '{name}' at {lam * 1e9:.1f} nm. Known: {sorted(table)}")
            return table[name]
    known = ", ".join(f"{w * 1e9:.1f} nm" for w in sorted(MASK_MATERIALS))
    raise KeyError(f"No mask-material table at {wavelength * 1e9:.3f} nm. Tabulated: {known}")


def _films_reflection(n_stored: np.ndarray, thickness: np.ndarray, wavelength: float, theta: np.ndarray,
                      polarisation: str) -> np.ndarray:
    """Amplitude reflection, seen from the ambient, of a planar stack
    (ambient first, substrate last, layers 1..L-2 finite) at each angle.

    Characteristic-matrix method: per layer j, delta_j = 2 pi n_j cos_j d_j /
    lambda and tilted admittance eta_j = n_j cos_j (s) or n_j / cos_j (p);
    [b, c] = prod_j [[cos d, i sin d / eta], [i eta sin d, cos d]] [1, eta_sub];
    r = (eta_0 - c/b) / (eta_0 + c/b). Indices are stored n + ik (k > 0
    absorbing) and conjugated for propagation (coat/films.py:88-100)."""
    if not wavelength > 0:
        raise ValueError(f"wavelength must be positive, got {wavelength}")
    n = np.conj(np.asarray(n_stored, dtype=np.complex128))
    th = np.asarray(theta, dtype=np.float64)
    sin0 = n[0] * np.sin(th)                                   # (A,)
    cos = np.sqrt(1.0 - (sin0[:, None] / n[None, :]) ** 2)     # (A, L)
    if polarisation == "s":
        eta = n[None, :] * cos
    elif polarisation == "p":
        eta = n[None, :] / cos
    else:
        raise ValueError(f"polarisation must be 's' or 'p', got '{polarisation}'")
    A = th.shape[0]
    m00 = np.ones(A, dtype=np.complex128)
    m01 = np.zeros(A, dtype=np.complex128)
    m10 = np.zeros(A, dtype=np.complex128)
    m11 = np.ones(A, dtype=np.complex128)
    for j in range(1, n.shape[0] - 1):
        delta = 2.0 * np.pi * n[j] * cos[:, j] * thickness[j] / wavelength
        cd, sd = np.cos(delta), np.sin(delta)
        a01 = 1j * sd / eta[:, j]
        a10 = 1j * eta[:, j] * sd
        m00, m01, m10, m11 = (m00 * cd + m01 * a10, m00 * a01 + m01 * cd,
                              m10 * cd + m11 * a10, m10 * a01 + m11 * cd)
    es = eta[:, -1]
    b = m00 + m01 * es
    c = m10 + m11 * es
    Y = c / b
    return (eta[:, 0] - Y) / (eta[:, 0] + Y)


@dataclass(frozen=True)
class Multilayer:
    """A Mo/Si Bragg mirror with a capping layer (expose/m3d/multilayer.py:46-152)."""

    n_bilayers: int = 40
    period: float = 6.94e-9
    gamma: float = 0.4
    cap_material: str = "Ru"
    cap_thickness: float = 2.5e-9
    substrate: str = "Si"

    def __post_init__(self) -> None:
        if self.n_bilayers < 1:
            raise ValueError(f"n_bilayers must be >= 1, got {self.n_bilayers}")
        if not 0.0 < self.gamma < 1.0:
            raise ValueError(f"gamma must be in (0, 1), got {self.gamma}")
        if self.period <= 0.0:
            raise ValueError(f"period must be positive, got {self.period}")

    def layers(self, wavelength: float) -> tuple[np.ndarray, np.ndarray]:
        """(stored indices, thicknesses): vacuum, cap, n x (Si, Mo), substrate."""
        t_mo = self.period * self.gamma
        t_si = self.period - t_mo
        n_si, n_mo = mask_material("Si", wavelength), mask_material("Mo", wavelength)
        idx = [mask_material("vacuum", wavelength), mask_material(self.cap_material, wavelength)]
        d = [0.0, self.cap_thickness]
        for _ in range(self.n_bilayers):
            idx += [n_si, n_mo]
            d += [t_si, t_mo]
        idx.append(mask_material(self.substrate, wavelength))
        d.append(0.0)
        return np.asarray(idx, dtype=np.complex128), np.asarray(d, dtype=np.float64)

    def amplitude_reflection(self, wavelength: float, theta: float = 0.0, polarisation: str = "s") -> complex:
        n, d = self.layers(wavelength)
        return complex(_films_reflection(n, d, wavelength, np.array([float(theta)]), polarisation)[0])

    def to_spec(self) -> dict[str, Any]:
        return {"n_bilayers": self.n_bilayers, "period": self.period, "gamma": self.gamma,
                "cap_material": self.cap_material, "cap_thickness": self.cap_thickness,
                "substrate": self.substrate}

    @classmethod
    def from_spec(cls, spec: dict[str, Any] | None) -> "Multilayer":
        return cls() if not spec else cls(**spec)


@dataclass(frozen=True)
class MaskStack:
    """Absorber on a substrate (expose/m3d/stack.py:45-205). Only the blank
    (the open trench) enters the multilayer model."""

    regime: str = "euv_reflective"
    absorber: str = "TaBN"
    absorber_thickness: float = 60e-9
    sidewall_deg: float = 90.0
    multilayer: Multilayer | None = field(default_factory=Multilayer)
    substrate: str = "SiO2"

    def __post_init__(self) -> None:
        if self.regime not in REGIMES:
            raise ValueError(f"regime must be one of {list(REGIMES)}, got '{self.regime}'")
        if self.absorber_thickness < 0.0:
            raise ValueError(f"absorber_thickness must be >= 0, got {self.absorber_thickness}")
        if not 0.0 < self.sidewall_deg <= 90.0:
            raise ValueError(f"sidewall_deg must be in (0, 90], got {self.sidewall_deg}")
        if self.is_reflective and self.multilayer is None:
            raise ValueError("regime='euv_reflective' needs a multilayer — a reflective mask "
                             "with no mirror reflects nothing.")

    @property
    def is_reflective(self) -> bool:
        return self.regime == "euv_reflective"

    def blank_layers(self, wavelength: float) -> tuple[np.ndarray, np.ndarray]:
        if self.is_reflective:
            return self.multilayer.layers(wavelength)
        q = mask_material(self.substrate, wavelength)
        return (np.asarray([mask_material("vacuum", wavelength), q, q], dtype=np.complex128),
                np.zeros(3, dtype=np.float64))

    def blank_reflection(self, wavelength: float, theta: float = 0.0, polarisation: str = "s") -> complex:
        n, d = self.blank_layers(wavelength)
        return complex(_films_reflection(n, d, wavelength, np.array([float(theta)]), polarisation)[0])

    def to_spec(self) -> dict[str, Any]:
        return {"regime": self.regime, "absorber": self.absorber, "absorber_thickness": self.absorber_thickness,
                "sidewall_deg": self.sidewall_deg, "substrate": self.substrate,
                "multilayer": self.multilayer.to_spec() if self.multilayer else None}

    @classmethod
    def from_spec(cls, spec: dict[str, Any] | None) -> "MaskStack":
        if not spec:
            return cls()
        data = dict(spec)
        ml = data.pop("multilayer", None)
        return cls(multilayer=Multilayer.from_spec(ml) if ml else None, **data)

    @classmethod
    def for_wavelength(cls, wavelength: float) -> "MaskStack":
        if abs(wavelength - 13.5e-9) < 1e-11:
            return cls(**MASK_STACK_PRESETS["EUV TaBN 60nm"])
        return cls(**MASK_STACK_PRESETS["DUV binary Cr"])


MASK_STACK_PRESETS: dict[str, dict[str, Any]] = {
    "EUV TaBN 60nm": {"regime": "euv_reflective", "absorber": "TaBN", "absorber_thickness": 60e-9,
                      "substrate": "SiO2"},
    "EUV TaBN 45nm": {"regime": "euv_reflective", "absorber": "TaBN", "absorber_thickness": 45e-9,
                      "substrate": "SiO2"},
    "DUV binary Cr": {"regime": "duv_transmissive", "absorber": "Cr", "absorber_thickness": 70e-9,
                      "multilayer": None, "substrate": "quartz"},
    "DUV att-PSM 6%": {"regime": "duv_transmissive", "absorber": "MoSi", "absorber_thickness": 71.9e-9,
                       "multilayer": None, "substrate": "quartz"},
}


def stack_for(view) -> MaskStack:
    """The stack an optics view names (its spec, else the wavelength's default),
    refused unless it is a reflective blank (provider.py:527-543)."""
    spec = view.mask_stack_spec() if hasattr(view, "mask_stack_spec") else getattr(view, "mask_stack", None)
    stack = MaskStack.from_spec(spec) if spec is not None else MaskStack.for_wavelength(view.wavelength)
    if not stack.is_reflective:
        raise ValueError(
            "mask_model='multilayer' describes the Bragg mirror under an EUV "
            f"mask, but the stack regime is '{stack.regime}'. Use "
            "mask_model='thin' or 'fdtd' for a transmissive mask.")
    return stack


@dataclass(frozen=True)
class MirrorTable:
    """The blank's scalar reflection on an angle table: theta [rad]
    (ascending from 0), |r| and the unwrapped arg r, all float64."""

    theta: np.ndarray
    mag: np.ndarray
    phase: np.ndarray

    def reflection(self, sin_theta: np.ndarray) -> np.ndarray:
        """r at each direction sine: linear interpolation of |r| and arg r in
        theta, clamped at the table ends; evanescent orders (sin > 1) get 0
        (provider.py:252-264)."""
        s_in = np.asarray(sin_theta, dtype=np.float64)
        prop = s_in <= 1.0
        th = np.arcsin(np.clip(s_in, 0.0, 1.0))
        r = np.interp(th, self.theta, self.mag) * np.exp(1j * np.interp(th, self.theta, self.phase))
        return np.where(prop, r, 0.0).astype(np.complex128)


_TABLES: dict = {}


def mirror_table(stack: MaskStack, wavelength: float) -> MirrorTable:
    """The reflection table of a blank (cached per stack and wavelength)."""
    key = (json.dumps(stack.to_spec(), sort_keys=True, default=str), float(wavelength))
    hit = _TABLES.get(key)
    if hit is not None:
        return hit
    theta = np.linspace(0.0, np.deg2rad(THETA_TABLE_MAX_DEG), THETA_TABLE_N)
    n, d = stack.blank_layers(wavelength)
    r = 0.5 * (_films_reflection(n, d, wavelength, theta, "s") + _films_reflection(n, d, wavelength, theta, "p"))
    t = MirrorTable(theta, np.abs(r), np.unwrap(np.angle(r)))
    if len(_TABLES) > 16:
        _TABLES.clear()
    _TABLES[key] = t
    return t


SOURCE_TILT_SIGN = -1.0


def chief_ray_sines(view) -> tuple[float, float]:
    """(sin_x, sin_y) the chief ray adds at the mask (provider.py:117-126)."""
    cra = math.sin(math.radians(view.chief_ray_deg))
    axis = view.chief_ray_axis.lower()
    if axis == "x":
        return cra, 0.0
    if axis == "y":
        return 0.0, cra
    raise ValueError(f"chief_ray_axis must be 'x' or 'y', got '{view.chief_ray_axis}'")


def mask_side_sin_theta(fs_x, fs_y, optics):
    """Mask-side direction sines of the illumination for source offsets
    (fs_x, fs_y) [1/m] (provider.py:72-126); scalars or arrays."""
    lam, m = optics.wavelength, optics.reduction
    sin_x = SOURCE_TILT_SIGN * lam * np.asarray(fs_x, dtype=np.float64) / m
    sin_y = SOURCE_TILT_SIGN * lam * np.asarray(fs_y, dtype=np.float64) / m
    cx, cy = chief_ray_sines(optics)
    if optics.chief_ray_axis.lower() == "x":
        sin_x = sin_x + cx
    else:
        sin_y = sin_y + cy
    if np.ndim(sin_x) == 0:
        return float(sin_x), float(sin_y)
    return sin_x, sin_y


def clear_scales(view, src) -> np.ndarray:
    """|r|^2 of the specular (DC) order for every source point: what an
    unpatterned blank returns (provider.py:283-295)."""
    t = mirror_table(stack_for(view), view.wavelength)
    sx, sy = mask_side_sin_theta(np.asarray(src.fx), np.asarray(src.fy), view)
    r = t.reflection(np.hypot(sx, sy))
    return np.abs(r) ** 2


__all__ = ["MASK_MATERIALS", "MASK_STACK_PRESETS", "MaskStack", "MirrorTable", "Multilayer", "REGIMES",
           "clear_scales", "mask_material", "mask_side_sin_theta", "mirror_table", "stack_for"]
