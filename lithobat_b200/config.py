"""Optics and grid parameters, mirroring the reference's configuration objects.

``OpticsConfig`` and ``GridConfig`` carry the same fields, defaults and
construction-time validation as Lithobat's ``core/config.py`` (OpticsConfig
:383-451, GridConfig :743-759), so code written against the reference runs
unchanged. Every public function of this package also accepts the
reference's own config objects (or anything with the same attributes): they
are read through :func:`optics_view`, never type-checked.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any

IMAGING_MODELS = ("scalar", "vector")
POLARISATIONS = ("unpolarised", "x", "y", "te", "tm")
NORMALISATIONS = ("peak", "clear", "none")
MASK_MODELS = ("thin", "multilayer", "fdtd")
SOURCE_TYPES = ("conventional", "annular", "monopole", "dipole", "quadrupole", "quasar", "cquad")
FOCUS_REFERENCES = ("top", "mid", "bottom")

TECH_NODE_PRESETS: dict[str, dict[str, Any]] = {
    "i-line": {"wavelength": 365e-9, "NA": 0.57},
    "KrF": {"wavelength": 248e-9, "NA": 0.75},
    "ArF": {"wavelength": 193e-9, "NA": 0.93},
    "ArF_immersion": {"wavelength": 193e-9, "NA": 1.35, "n_immersion": 1.44},
    "EUV": {"wavelength": 13.5e-9, "NA": 0.33},
}


def _finite(owner: str, name: str, v: float) -> None:
    if isinstance(v, bool) or not isinstance(v, (int, float)) or not math.isfinite(float(v)):
        raise ValueError(f"{owner}.{name} must be a finite number, got {v!r}")


def _bounded(owner, name, v, lo=None, hi=None, lo_open=False):
    _finite(owner, name, v)
    if lo is not None and (v <= lo if lo_open else v < lo):
        raise ValueError(f"{owner}.{name} must be {'>' if lo_open else '>='} {lo:g}, got {v:g}")
    if hi is not None and v > hi:
        raise ValueError(f"{owner}.{name} must be <= {hi:g}, got {v:g}")


def _choice(owner, name, v, choices):
    if not isinstance(v, str) or v.lower() not in choices:
        raise ValueError(f"{owner}.{name} must be one of {list(choices)}, got {v!r}")


@dataclass
class OpticsConfig:
    """Projection optics (wavelength and lengths in metres)."""

    wavelength: float = 193e-9
    NA: float = 0.93
    n_immersion: float = 1.0
    defocus: float = 0.0
    sigma_outer: float = 0.80
    sigma_inner: float = 0.0
    source_type: str = "conventional"
    source_grid: int = 21
    source_kwargs: dict[str, Any] = field(default_factory=dict)
    source_spec: dict[str, Any] | None = None
    zernike_coeffs: dict[int, float] = field(default_factory=dict)
    exact_defocus: bool = False
    n_image: float | None = None
    imaging_model: str = "scalar"
    polarisation: str = "unpolarised"
    obliquity: bool = True
    normalisation: str = "peak"
    mask_model: str = "thin"
    reduction: float = 4.0
    chief_ray_deg: float = 0.0
    chief_ray_axis: str = "x"
    mask_stack: dict[str, Any] | None = None
    mask_geometry: dict[str, Any] | None = None
    m3d_angles: int = 3

    def __post_init__(self) -> None:
        o = "OpticsConfig"
        _bounded(o, "wavelength", self.wavelength, 0.0, lo_open=True)
        _bounded(o, "NA", self.NA, 0.0, lo_open=True)
        _bounded(o, "n_immersion", self.n_immersion, 0.0, lo_open=True)
        if self.n_image is not None:
            _bounded(o, "n_image", self.n_image, 0.0, lo_open=True)
        if self.NA > self.image_index:
            raise ValueError(
                f"{o}: NA {self.NA:g} exceeds the image-space index {self.image_index:g}, "
                "which would make sin θ > 1. Raise n_immersion (or n_image) or lower NA.")
        _bounded(o, "defocus", self.defocus)
        _bounded(o, "sigma_outer", self.sigma_outer, 0.0, 1.0, lo_open=True)
        _bounded(o, "sigma_inner", self.sigma_inner, 0.0, self.sigma_outer)
        _bounded(o, "source_grid", self.source_grid, 3)
        if self.source_spec is None:
            _choice(o, "source_type", self.source_type, SOURCE_TYPES)
        _choice(o, "imaging_model", self.imaging_model, IMAGING_MODELS)
        _choice(o, "polarisation", self.polarisation, POLARISATIONS)
        _choice(o, "normalisation", self.normalisation, NORMALISATIONS)
        _choice(o, "mask_model", self.mask_model, MASK_MODELS)
        _choice(o, "chief_ray_axis", self.chief_ray_axis, ("x", "y"))
        _bounded(o, "reduction", self.reduction, 0.0, lo_open=True)
        _bounded(o, "chief_ray_deg", self.chief_ray_deg, -90.0, 90.0)
        _bounded(o, "m3d_angles", self.m3d_angles, 1)
        for j, c in (self.zernike_coeffs or {}).items():
            if not isinstance(j, int) or isinstance(j, bool) or j < 1:
                raise ValueError(f"{o}.zernike_coeffs keys are Noll indices (int ≥ 1), got {j!r}")
            _bounded(o, f"zernike_coeffs[{j}]", c)

    @property
    def image_index(self) -> float:
        return self.n_immersion if self.n_image is None else self.n_image

    @property
    def k_max(self) -> float:
        return self.NA / self.wavelength

    @property
    def sin_theta_max(self) -> float:
        return self.NA / self.image_index

    @classmethod
    def from_tech_node(cls, node: str, **kw) -> "OpticsConfig":
        return cls(**{**TECH_NODE_PRESETS[node], **kw})


@dataclass
class GridConfig:
    """Square simulation grid (core/config.py:720-759): n_pixels x n_pixels
    pixels of pixel_size [m]; dz [m] the voxel height and n_z_slices the
    optical planes of a depth-resolved exposure (:func:`exposure_volume`)."""

    n_pixels: int = 128
    pixel_size: float = 4e-9
    dz: float = 2e-9
    n_z_slices: int = 21

    def __post_init__(self) -> None:
        if isinstance(self.n_pixels, bool) or int(self.n_pixels) != self.n_pixels:
            raise TypeError(f"GridConfig.n_pixels must be an integer, got {self.n_pixels!r}")
        _bounded("GridConfig", "n_pixels", self.n_pixels, 1)
        _bounded("GridConfig", "pixel_size", self.pixel_size, 0.0, lo_open=True)
        # dz = 0 is accepted: two-dimensional work never reads it
        _bounded("GridConfig", "dz", self.dz, 0.0)
        _bounded("GridConfig", "n_z_slices", self.n_z_slices, 1)

    @property
    def grid_size(self) -> float:
        return self.n_pixels * self.pixel_size


@dataclass
class ResistConfig:
    """The resist parameters the imaging helpers read, with the names,
    defaults and checks of core/config.py:ResistConfig (:491-718): the
    threshold development (threshold, diffusion_sigma [m]) and the film a
    depth-resolved exposure images through (thickness [m], n_resist, and
    focus_reference, the depth OpticsConfig.defocus refers to). The
    reference's own ResistConfig is accepted wherever this one is."""

    threshold: float = 0.30
    diffusion_sigma: float = 20e-9
    thickness: float = 100e-9
    n_resist: float = 1.70
    focus_reference: str = "mid"

    def __post_init__(self) -> None:
        r = "ResistConfig"
        _finite(r, "threshold", self.threshold)
        if not 0.0 < self.threshold < 1.0:
            raise ValueError(f"{r}.threshold must be in (0, 1), got {self.threshold:g}")
        _bounded(r, "diffusion_sigma", self.diffusion_sigma, 0.0)
        _bounded(r, "thickness", self.thickness, 0.0)
        _bounded(r, "n_resist", self.n_resist, 0.0, lo_open=True)
        _choice(r, "focus_reference", self.focus_reference, FOCUS_REFERENCES)


@dataclass(frozen=True)
class OpticsView:
    """The fields the imaging path reads, taken from any optics-like object."""

    wavelength: float
    NA: float
    n_immersion: float
    defocus: float
    sigma_outer: float
    sigma_inner: float
    source_type: str
    source_grid: int
    source_kwargs: tuple
    source_spec: Any
    zernike: tuple          # ((j, c), ...) sorted
    exact_defocus: bool
    image_index: float
    imaging_model: str
    polarisation: str
    obliquity: bool
    normalisation: str
    mask_model: str
    reduction: float = 4.0
    chief_ray_deg: float = 0.0
    chief_ray_axis: str = "x"
    mask_stack: str | None = None   # the stack spec as sorted JSON (hashable)

    def mask_stack_spec(self) -> dict | None:
        import json
        return None if self.mask_stack is None else json.loads(self.mask_stack)

    @property
    def zernike_coeffs(self) -> dict[int, float]:
        return dict(self.zernike)

    def source_key(self) -> tuple:
        import json
        spec = None if self.source_spec is None else json.dumps(self.source_spec, sort_keys=True,
                                                                  default=str)
        return (self.wavelength, self.NA, self.source_type, self.source_grid, self.sigma_outer,
                self.sigma_inner, self.source_kwargs, spec)


def optics_view(optics) -> OpticsView:
    if isinstance(optics, OpticsView):
        return optics
    g = lambda n, d: getattr(optics, n, d)  # noqa: E731
    n_img = g("n_image", None)
    n_imm = float(g("n_immersion", 1.0))
    zc = g("zernike_coeffs", None) or {}
    return OpticsView(
        wavelength=float(optics.wavelength), NA=float(optics.NA), n_immersion=n_imm,
        defocus=float(g("defocus", 0.0)), sigma_outer=float(g("sigma_outer", 0.8)),
        sigma_inner=float(g("sigma_inner", 0.0)), source_type=str(g("source_type", "conventional")),
        source_grid=int(g("source_grid", 21)),
        source_kwargs=tuple(sorted((g("source_kwargs", None) or {}).items())),
        source_spec=g("source_spec", None),
        zernike=tuple(sorted((int(j), float(c)) for j, c in zc.items())),
        exact_defocus=bool(g("exact_defocus", False)),
        image_index=float(n_imm if n_img is None else n_img),
        imaging_model=str(g("imaging_model", "scalar")), polarisation=str(g("polarisation", "unpolarised")),
        obliquity=bool(g("obliquity", True)), normalisation=str(g("normalisation", "peak")),
        mask_model=str(g("mask_model", "thin")),
        reduction=float(g("reduction", 4.0)), chief_ray_deg=float(g("chief_ray_deg", 0.0)),
        chief_ray_axis=str(g("chief_ray_axis", "x")), mask_stack=_stack_json(g("mask_stack", None)),
    )


def _stack_json(spec) -> str | None:
    if spec is None:
        return None
    import json
    if hasattr(spec, "to_spec"):
        spec = spec.to_spec()
    return json.dumps(spec, sort_keys=True, default=str)
