"""Illumination sources and their discrete source points (host side, FP64).

The Abbe sum runs over the non-zero pixels of the source map rendered on an
``ns x ns`` normalised pupil grid (rows = eta, columns = xi, both spanning
[-1, 1]). Which pixels are non-zero, and their weights, decide the image at
the O(1) level, so this module reproduces the reference's rasterisation
exactly: the legacy disc shapes of ``expose/illumination.py`` (:26-129,
dispatched by ``build_source`` :132-219), the annular-sector ``Pole`` /
``Source`` of ``expose/source.py`` (:79-219, presets :275-378) and the
point list of ``expose/aerial_image.py:source_points`` (:275-304). It runs
on the host in float64 — a few thousand pixels — and is not part of the
device hot path.
"""

from __future__ import annotations

from dataclasses import asdict, dataclass, field
from typing import Any

import numpy as np

from .config import optics_view


def pupil_grid(n: int):
    """(rho, phi, xi, eta) on the normalised source grid; rows = eta."""
    axis = np.linspace(-1.0, 1.0, n)
    xi, eta = np.meshgrid(axis, axis)
    return np.sqrt(xi ** 2 + eta ** 2), np.arctan2(eta, xi), xi, eta


def _to_unit_sum(src: np.ndarray) -> np.ndarray:
    total = src.sum()
    return src / total if total > 0 else src


# --- legacy disc-pole shapes (the rasterisation older results are pinned to) --

def _discs(n, sigma_outer, sigma_inner, centres) -> np.ndarray:
    radius = (sigma_outer - sigma_inner) / 2.0
    _, _, xi, eta = pupil_grid(n)
    acc = np.zeros((n, n), dtype=np.float64)
    for cx, cy in centres:
        acc += (np.sqrt((xi - cx) ** 2 + (eta - cy) ** 2) <= radius).astype(np.float64)
    return _to_unit_sum(acc)


def conventional(n: int, sigma: float) -> np.ndarray:
    rho = pupil_grid(n)[0]
    return _to_unit_sum((rho <= sigma).astype(np.float64))


def annular(n: int, sigma_outer: float, sigma_inner: float) -> np.ndarray:
    if sigma_inner >= sigma_outer:
        raise ValueError(f"sigma_inner ({sigma_inner:.3f}) must be < sigma_outer ({sigma_outer:.3f})")
    rho = pupil_grid(n)[0]
    return _to_unit_sum(((rho >= sigma_inner) & (rho <= sigma_outer)).astype(np.float64))


def dipole(n: int, sigma_outer: float, sigma_inner: float, axis: str = "x") -> np.ndarray:
    mid = (sigma_outer + sigma_inner) / 2.0
    centres = [(mid, 0.0), (-mid, 0.0)] if axis == "x" else [(0.0, mid), (0.0, -mid)]
    return _discs(n, sigma_outer, sigma_inner, centres)


def quadrupole(n: int, sigma_outer: float, sigma_inner: float, rotation_deg: float = 45.0) -> np.ndarray:
    mid = (sigma_outer + sigma_inner) / 2.0
    angles = np.deg2rad(np.array([0.0, 90.0, 180.0, 270.0]) + rotation_deg)
    return _discs(n, sigma_outer, sigma_inner, [(mid * np.cos(a), mid * np.sin(a)) for a in angles])


# --- composable sources ------------------------------------------------------


@dataclass(frozen=True)
class Pole:
    """One annular sector of the source (expose/source.py:79-136)."""

    sigma_inner: float = 0.0
    sigma_outer: float = 0.9
    angle_deg: float = 0.0
    opening_deg: float = 360.0
    weight: float = 1.0

    def __post_init__(self) -> None:
        if self.sigma_outer <= 0:
            raise ValueError(f"sigma_outer must be > 0, got {self.sigma_outer}")
        if self.sigma_inner < 0:
            raise ValueError(f"sigma_inner must be >= 0, got {self.sigma_inner}")
        if self.sigma_inner >= self.sigma_outer:
            raise ValueError(f"sigma_inner ({self.sigma_inner:.3f}) must be < "
                             f"sigma_outer ({self.sigma_outer:.3f})")
        if not 0.0 < self.opening_deg <= 360.0:
            raise ValueError(f"opening_deg must be in (0, 360], got {self.opening_deg}")
        if self.weight < 0:
            raise ValueError(f"weight must be >= 0, got {self.weight}")

    def render(self, n: int) -> np.ndarray:
        rho, phi, _, _ = pupil_grid(n)
        in_ring = (rho >= self.sigma_inner) & (rho <= self.sigma_outer)
        if self.opening_deg >= 360.0:
            in_sector = np.ones_like(in_ring, dtype=bool)
        else:
            wrapped = np.angle(np.exp(1j * (phi - np.deg2rad(self.angle_deg))))
            in_sector = np.abs(wrapped) <= np.deg2rad(self.opening_deg) / 2.0
        return self.weight * (in_ring & in_sector).astype(np.float64)

    def to_dict(self) -> dict[str, Any]:
        return asdict(self)


@dataclass
class Source:
    """Poles composed additively, optional blur and prune (expose/source.py:143-219)."""

    poles: list[Pole] = field(default_factory=list)
    pixels: np.ndarray | None = None
    blur: float = 0.0
    prune: float = 1e-3
    name: str = "source"

    def render(self, n: int, normalise: bool = True) -> np.ndarray:
        if n < 3:
            raise ValueError(f"source grid must be >= 3, got {n}")
        if self.pixels is not None:
            src = self._resample(n)
        else:
            src = np.zeros((n, n), dtype=np.float64)
            for p in self.poles:
                src += p.render(n)
        if self.blur > 0.0:
            from scipy.ndimage import gaussian_filter
            src = gaussian_filter(src, sigma=self.blur * (n - 1) / 2.0, mode="constant")
        rho = pupil_grid(n)[0]
        src = np.where(rho <= 1.0, src, 0.0)
        if self.prune > 0.0 and src.max() > 0:
            src = np.where(src >= self.prune * src.max(), src, 0.0)
        if normalise:
            total = src.sum()
            if total > 0:
                src = src / total
        return src

    def _resample(self, n: int) -> np.ndarray:
        px = np.asarray(self.pixels, dtype=np.float64)
        if px.ndim != 2:
            raise ValueError(f"pixels must be 2-D, got shape {px.shape}")
        if px.shape == (n, n):
            return px.copy()
        from scipy.ndimage import zoom
        out = zoom(px, (n / px.shape[0], n / px.shape[1]), order=1, mode="nearest")
        if out.shape != (n, n):
            fixed = np.zeros((n, n), dtype=np.float64)
            r, c = min(n, out.shape[0]), min(n, out.shape[1])
            fixed[:r, :c] = out[:r, :c]
            out = fixed
        return np.clip(out, 0.0, None)

    def n_points(self, n: int) -> int:
        return int((self.render(n) > 0).sum())

    # presets (expose/source.py:275-378)
    @classmethod
    def conventional(cls, sigma: float = 0.8, **kw) -> "Source":
        return cls(poles=[Pole(0.0, sigma, 0.0, 360.0)], name="conventional", **kw)

    @classmethod
    def annular(cls, sigma_outer: float = 0.9, sigma_inner: float = 0.6, **kw) -> "Source":
        return cls(poles=[Pole(sigma_inner, sigma_outer, 0.0, 360.0)], name="annular", **kw)

    @classmethod
    def monopole(cls, sigma_outer=0.9, sigma_inner=0.6, angle_deg=0.0, opening_deg=60.0, **kw):
        return cls(poles=[Pole(sigma_inner, sigma_outer, angle_deg, opening_deg)], name="monopole", **kw)

    @classmethod
    def dipole(cls, sigma_outer=0.9, sigma_inner=0.6, opening_deg=60.0, axis="x", **kw):
        if axis not in ("x", "y"):
            raise ValueError(f"axis must be 'x' or 'y', got '{axis}'")
        base = 0.0 if axis == "x" else 90.0
        return cls(poles=[Pole(sigma_inner, sigma_outer, base + a, opening_deg) for a in (0.0, 180.0)],
                   name=f"dipole-{axis}", **kw)

    @classmethod
    def quadrupole(cls, sigma_outer=0.9, sigma_inner=0.6, opening_deg=40.0, rotation_deg=45.0, **kw):
        return cls(poles=[Pole(sigma_inner, sigma_outer, a + rotation_deg, opening_deg)
                          for a in (0.0, 90.0, 180.0, 270.0)], name="quadrupole", **kw)

    @classmethod
    def quasar(cls, sigma_outer=0.9, sigma_inner=0.6, opening_deg=40.0, rotation_deg=45.0, **kw):
        s = cls.quadrupole(sigma_outer, sigma_inner, opening_deg, rotation_deg, **kw)
        s.name = "quasar"
        return s

    @classmethod
    def cquad(cls, sigma_outer=0.9, sigma_inner=0.6, opening_deg=40.0, **kw):
        s = cls.quadrupole(sigma_outer, sigma_inner, opening_deg, 0.0, **kw)
        s.name = "cquad"
        return s

    def to_dict(self) -> dict[str, Any]:
        return {"name": self.name, "blur": self.blur, "prune": self.prune,
                "poles": [p.to_dict() for p in self.poles],
                "pixels": None if self.pixels is None else np.asarray(self.pixels).tolist()}

    @classmethod
    def from_dict(cls, d: dict[str, Any]) -> "Source":
        px = d.get("pixels")
        return cls(poles=[Pole(**p) for p in d.get("poles", [])],
                   pixels=None if px is None else np.asarray(px, dtype=np.float64),
                   blur=float(d.get("blur", 0.0)), prune=float(d.get("prune", 1e-3)),
                   name=str(d.get("name", "source")))


def build_source(n: int, source_type: str, sigma_outer: float, sigma_inner: float = 0.0,
                 spec: dict | None = None, **kwargs) -> np.ndarray:
    """Render a named shape, or a serialised Source when ``spec`` is given."""
    if spec is not None:
        return Source.from_dict(spec).render(n)
    key = source_type.lower()
    if kwargs and key in ("conventional", "annular"):
        raise ValueError(f"Source type '{key}' accepts no extra arguments, got {sorted(kwargs)}. "
                         "Use 'monopole', 'dipole', 'quasar' or 'cquad' for shapes with an angle "
                         "or opening.")
    if key == "conventional":
        return conventional(n, sigma_outer)
    if key == "annular":
        return annular(n, sigma_outer, sigma_inner)
    if key == "dipole":
        return dipole(n, sigma_outer, sigma_inner, **kwargs)
    if key == "quadrupole":
        return quadrupole(n, sigma_outer, sigma_inner, **kwargs)
    if key == "monopole":
        return Source.monopole(sigma_outer, sigma_inner, **kwargs).render(n)
    if key == "quasar":
        return Source.quasar(sigma_outer, sigma_inner, **kwargs).render(n)
    if key == "cquad":
        return Source.cquad(sigma_outer, sigma_inner, **kwargs).render(n)
    raise ValueError(f"Unknown source type '{source_type}'. Available: "
                     "['conventional', 'annular', 'dipole', 'quadrupole', 'monopole', 'quasar', 'cquad']")


@dataclass(frozen=True)
class SourcePoints:
    """The discrete illumination: weights, frequency offsets [1/m], azimuths."""

    weight: np.ndarray
    fx: np.ndarray
    fy: np.ndarray
    phi: np.ndarray
    grid: int

    def __len__(self) -> int:
        return int(self.weight.size)


_CACHE: dict[tuple, SourcePoints] = {}


def source_points(optics) -> SourcePoints:
    """Non-zero source pixels as offsets f_s = xi_s NA / lambda (FP64, exact)."""
    v = optics_view(optics)
    key = v.source_key()
    hit = _CACHE.get(key)
    if hit is not None:
        return hit
    ns = max(int(v.source_grid), 3)
    src = build_source(ns, v.source_type, v.sigma_outer, v.sigma_inner, spec=v.source_spec,
                       **dict(v.source_kwargs))
    rc = np.argwhere(src > 0)
    rows, cols = rc[:, 0].astype(np.float64), rc[:, 1].astype(np.float64)
    half = (ns - 1) / 2.0
    k_max = v.NA / v.wavelength
    sp = SourcePoints(weight=src[rc[:, 0], rc[:, 1]].astype(np.float64),
                      fx=((cols - half) / half) * k_max, fy=((rows - half) / half) * k_max,
                      phi=np.arctan2(rows - half, cols - half), grid=ns)
    if len(_CACHE) > 64:
        _CACHE.clear()
    _CACHE[key] = sp
    return sp
