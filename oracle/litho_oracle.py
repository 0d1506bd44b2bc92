"""FP64 numpy restatement of Lithobat's partially coherent imaging path.

TEST INFRASTRUCTURE. This module is the oracle the CUDA path is checked
against. It is imported only by ``tests/``, by ``__graft_entry__.smoke()`` and
by ``bench.py``'s CPU baseline / ``--impl reference`` arm, never by the
product package ``lithobat_b200``.

Every function restates one function of the reference (``bat723/Lithobat``,
package ``litho_sim``) and cites the file:line it follows. The arithmetic is
kept in the same order wherever an operation decides a discrete outcome
(aperture inclusion ``rho <= 1``, the SOCS band test, the source prune), so
those decisions are bit-identical to the reference's. The reference is pure
numpy/scipy; the FFTs here are the same library calls it makes
(``numpy.fft`` / ``scipy.fft``, pocketfft) and the eigendecomposition is the
same ``numpy.linalg.eigh``.

Parity of this restatement is pinned by ``tests/golden/*.npz``: outputs of the
reference itself, generated by ``tests/golden/make_golden.py`` and checked in
``tests/test_oracle_golden.py``.

Configuration objects are duck-typed: any object with the attributes of the
reference's ``OpticsConfig`` / ``GridConfig`` (``core/config.py:383-406``,
``:743-746``) works, including the reference's own classes and the product's.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
from scipy import fft as sfft
from scipy.ndimage import gaussian_filter

# core/config.py:173-176
IMAGING_MODELS = ("scalar", "vector")
POLARISATIONS = ("unpolarised", "x", "y", "te", "tm")
NORMALISATIONS = ("peak", "clear", "none")

# expose/aerial_image.py:73 and :78
SOURCE_TILT_SIGN = -1.0
FFT_BATCH_BYTES = 64 * 2 ** 20


def _opt(optics, name, default):
    return getattr(optics, name, default)


def image_index(optics) -> float:
    """core/config.py:470-477 — n_image, defaulting to n_immersion."""
    n_img = _opt(optics, "n_image", None)
    return float(_opt(optics, "n_immersion", 1.0) if n_img is None else n_img)


# ---------------------------------------------------------------------------
# Grids
# ---------------------------------------------------------------------------


def make_freq_grid(n: int, pixel_size: float):
    """core/utils.py:45-66 — fftfreq meshgrid, FFT ordering, DC at [0, 0]."""
    f = np.fft.fftfreq(n, d=pixel_size)
    fx, fy = np.meshgrid(f, f)
    return fx.astype(np.float64), fy.astype(np.float64)


def pupil_grid(n: int):
    """expose/pupil.py:35-48 — normalised [-1, 1] grid, rows = eta, cols = xi."""
    c = np.linspace(-1.0, 1.0, n)
    xi, eta = np.meshgrid(c, c)
    return np.sqrt(xi ** 2 + eta ** 2), np.arctan2(eta, xi), xi, eta


# ---------------------------------------------------------------------------
# Source rendering (expose/illumination.py, expose/source.py)
# ---------------------------------------------------------------------------


def _unit_sum(a):
    """illumination.py:21-23."""
    s = a.sum()
    return a / s if s > 0 else a


def _legacy_disc_poles(n, sigma_outer, sigma_inner, centres):
    r_pole = (sigma_outer - sigma_inner) / 2.0
    _, _, xi, eta = pupil_grid(n)
    out = np.zeros((n, n), dtype=np.float64)
    for cx, cy in centres:
        d = np.sqrt((xi - cx) ** 2 + (eta - cy) ** 2)
        out += (d <= r_pole).astype(np.float64)
    return _unit_sum(out)


def render_legacy(n, kind, sigma_outer, sigma_inner, **kw):
    """illumination.py:26-129 — the disc-based named shapes."""
    rho, *_ = pupil_grid(n)
    if kind == "conventional":
        return _unit_sum((rho <= sigma_outer).astype(np.float64))
    if kind == "annular":
        if sigma_inner >= sigma_outer:
            raise ValueError(
                f"sigma_inner ({sigma_inner:.3f}) must be < sigma_outer ({sigma_outer:.3f})")
        return _unit_sum(((rho >= sigma_inner) & (rho <= sigma_outer)).astype(np.float64))
    c_mid = (sigma_outer + sigma_inner) / 2.0
    if kind == "dipole":
        axis = kw.get("axis", "x")
        centres = [(c_mid, 0.0), (-c_mid, 0.0)] if axis == "x" else [(0.0, c_mid), (0.0, -c_mid)]
        return _legacy_disc_poles(n, sigma_outer, sigma_inner, centres)
    if kind == "quadrupole":
        rot = kw.get("rotation_deg", 45.0)
        ang = np.deg2rad(np.array([0.0, 90.0, 180.0, 270.0]) + rot)
        centres = [(c_mid * np.cos(a), c_mid * np.sin(a)) for a in ang]
        return _legacy_disc_poles(n, sigma_outer, sigma_inner, centres)
    raise ValueError(kind)


def render_pole(n, sigma_inner, sigma_outer, angle_deg, opening_deg, weight):
    """source.py:122-132 — one annular sector."""
    rho, phi, _, _ = pupil_grid(n)
    radial = (rho >= sigma_inner) & (rho <= sigma_outer)
    if opening_deg >= 360.0:
        angular = np.ones_like(radial, dtype=bool)
    else:
        d = np.angle(np.exp(1j * (phi - np.deg2rad(angle_deg))))
        angular = np.abs(d) <= np.deg2rad(opening_deg) / 2.0
    return weight * (radial & angular).astype(np.float64)


def render_spec(spec: dict, n: int):
    """source.py:174-219 — Source.render from its dict form (source.py:425-434)."""
    if n < 3:
        raise ValueError(f"source grid must be >= 3, got {n}")
    pixels = spec.get("pixels")
    if pixels is not None:
        px = np.asarray(pixels, dtype=np.float64)
        if px.shape != (n, n):
            raise NotImplementedError("oracle: free-form resampling is not restated")
        src = px.copy()
    else:
        src = np.zeros((n, n), dtype=np.float64)
        for p in spec.get("poles", []):
            src += render_pole(
                n, float(p.get("sigma_inner", 0.0)), float(p.get("sigma_outer", 0.9)),
                float(p.get("angle_deg", 0.0)), float(p.get("opening_deg", 360.0)),
                float(p.get("weight", 1.0)),
            )
    blur = float(spec.get("blur", 0.0))
    if blur > 0.0:
        src = gaussian_filter(src, sigma=blur * (n - 1) / 2.0, mode="constant")
    rho, _, _, _ = pupil_grid(n)
    src = np.where(rho <= 1.0, src, 0.0)
    prune = float(spec.get("prune", 1e-3))
    if prune > 0.0 and src.max() > 0:
        src = np.where(src >= prune * src.max(), src, 0.0)
    total = src.sum()
    if total > 0:
        src = src / total
    return src


def _spec_of_preset(kind, sigma_outer, sigma_inner, **kw):
    """source.py:275-378 — the pole sets of the Source presets."""
    def pole(si, so, a, op):
        return {"sigma_inner": si, "sigma_outer": so, "angle_deg": a,
                "opening_deg": op, "weight": 1.0}
    if kind == "monopole":
        return {"poles": [pole(sigma_inner, sigma_outer, kw.get("angle_deg", 0.0),
                               kw.get("opening_deg", 60.0))]}
    if kind in ("quasar", "cquad"):
        rot = kw.get("rotation_deg", 45.0) if kind == "quasar" else 0.0
        op = kw.get("opening_deg", 40.0)
        return {"poles": [pole(sigma_inner, sigma_outer, a + rot, op)
                          for a in (0.0, 90.0, 180.0, 270.0)]}
    raise ValueError(kind)


def build_source(n, source_type, sigma_outer, sigma_inner=0.0, spec=None, **kw):
    """illumination.py:132-219."""
    if spec is not None:
        return render_spec(spec, n)
    key = source_type.lower()
    if key in ("conventional", "annular", "dipole", "quadrupole"):
        if kw and key in ("conventional", "annular"):
            raise ValueError(f"Source type '{key}' accepts no extra arguments")
        return render_legacy(n, key, sigma_outer, sigma_inner, **kw)
    if key in ("monopole", "quasar", "cquad"):
        return render_spec(_spec_of_preset(key, sigma_outer, sigma_inner, **kw), n)
    raise ValueError(f"Unknown source type '{source_type}'")


@dataclass(frozen=True)
class SourcePoints:
    """aerial_image.py:249-272."""
    weight: np.ndarray
    fx: np.ndarray
    fy: np.ndarray
    phi: np.ndarray
    grid: int

    def __len__(self):
        return int(self.weight.size)


def source_points(optics) -> SourcePoints:
    """aerial_image.py:275-304 — non-zero source pixels as frequency offsets."""
    ns = max(int(_opt(optics, "source_grid", 21)), 3)
    src = build_source(
        ns, _opt(optics, "source_type", "conventional"), _opt(optics, "sigma_outer", 0.8),
        _opt(optics, "sigma_inner", 0.0), spec=_opt(optics, "source_spec", None),
        **(_opt(optics, "source_kwargs", None) or {}),
    )
    idx = np.argwhere(src > 0)
    rows = idx[:, 0].astype(np.float64)
    cols = idx[:, 1].astype(np.float64)
    half = (ns - 1) / 2.0
    k_max = optics.NA / optics.wavelength
    return SourcePoints(
        weight=src[idx[:, 0], idx[:, 1]].astype(np.float64),
        fx=((cols - half) / half) * k_max,
        fy=((rows - half) / half) * k_max,
        phi=np.arctan2(rows - half, cols - half),
        grid=ns,
    )


# ---------------------------------------------------------------------------
# Pupil (expose/pupil.py)
# ---------------------------------------------------------------------------

# pupil.py:56-78 — Noll j -> (n, m)
NOLL = {
    1: (0, 0), 2: (1, 1), 3: (1, -1), 4: (2, 0), 5: (2, -2), 6: (2, 2),
    7: (3, -1), 8: (3, 1), 9: (3, -3), 10: (3, 3), 11: (4, 0), 12: (4, 2),
    13: (4, -2), 14: (4, 4), 15: (4, -4), 16: (5, 1), 17: (5, -1), 18: (5, 3),
    19: (5, -3), 20: (5, 5), 21: (5, -5),
}


def radial_poly(n, m, rho):
    """pupil.py:81-100 — R_n^|m| by the explicit sum, rho clipped to [0, 1]."""
    ma = abs(m)
    r = np.clip(rho, 0.0, 1.0)
    out = np.zeros_like(r, dtype=np.float64)
    for s in range((n - ma) // 2 + 1):
        c = ((-1) ** s * math.factorial(n - s)
             / (math.factorial(s) * math.factorial((n + ma) // 2 - s)
                * math.factorial((n - ma) // 2 - s)))
        out += c * r ** (n - 2 * s)
    return out


def zernike_noll(j, rho, phi):
    """pupil.py:103-141 — unknown j gives zeros."""
    if j not in NOLL:
        return np.zeros_like(rho, dtype=np.float64)
    n, m = NOLL[j]
    norm = math.sqrt(n + 1) if m == 0 else math.sqrt(2.0 * (n + 1))
    R = radial_poly(n, m, rho)
    if m > 0:
        return norm * R * np.cos(m * phi)
    if m < 0:
        return norm * R * np.sin(abs(m) * phi)
    return norm * R


def defocus_opd(rho, wavelength, NA, defocus, n_image=1.0, exact=False):
    """pupil.py:155-221 — paraxial or exact defocus phase [rad]."""
    if defocus == 0.0:
        return np.zeros_like(rho, dtype=np.float64)
    r = np.asarray(rho, dtype=np.float64)
    if not exact:
        return np.pi * NA ** 2 * r ** 2 * defocus / (wavelength * n_image)
    s2 = np.clip((r * NA / n_image) ** 2, 0.0, 1.0)
    return (2.0 * np.pi / wavelength) * (n_image * defocus * (1.0 - np.sqrt(1.0 - s2)))


def jones_states(polarisation: str, phi_source: float):
    """pupil.py:232-289 — list of (Jx, Jy, weight) incoherent states."""
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
    """pupil.py:292-369 — (Vx, Vy, Vz) with the sqrt(cos theta) obliquity."""
    s2 = np.clip((np.asarray(rho, dtype=np.float64) * sin_theta_max) ** 2, 0.0, 1.0)
    ct, st = np.sqrt(1.0 - s2), np.sqrt(s2)
    cp, sp = np.cos(phi), np.sin(phi)
    e_s = -jx * sp + jy * cp
    e_p = jx * cp + jy * sp
    vx = -e_s * sp + e_p * ct * cp
    vy = e_s * cp + e_p * ct * sp
    vz = -e_p * st
    if obliquity:
        a = np.sqrt(ct)
        vx, vy, vz = vx * a, vy * a, vz * a
    return vx.astype(np.complex128), vy.astype(np.complex128), vz.astype(np.complex128)


def pupil_phase(rho, phi, wavelength, NA, defocus, n_image, zernike, exact):
    """aerial_image.py:142-166 — defocus plus 2*pi*sum c_j Z_j."""
    W = defocus_opd(rho, wavelength, NA, defocus, n_image, exact=exact)
    if zernike:
        W = np.array(W, dtype=np.float64, copy=True)
        for j, c in zernike.items():
            W += 2.0 * np.pi * c * zernike_noll(j, rho, phi)
    return W


# ---------------------------------------------------------------------------
# Abbe sum (expose/aerial_image.py)
# ---------------------------------------------------------------------------


def normalisation_scale(mode, peak, clear, dose=1.0):
    """aerial_image.py:217-241."""
    m = mode.lower()
    if m == "peak":
        return dose / peak if peak > 0 else dose
    if m == "clear":
        return dose / clear if clear > 0 else dose
    if m == "none":
        return dose
    raise ValueError(f"normalisation must be 'peak', 'clear' or 'none', got '{mode}'")


# ---------------------------------------------------------------------------
# The EUV blank as a Bragg mirror (mask_model="multilayer")
# ---------------------------------------------------------------------------

# expose/m3d/materials.py:58-82 (n + ik, k > 0 absorbing)
_MASK_N = {
    13.5e-9: {"vacuum": 1.0 + 0.0j, "Si": 0.99931 + 0.00182j, "Mo": 0.92108 + 0.00644j,
              "Ru": 0.88651 + 0.01710j, "TaBN": 0.94900 + 0.03120j, "TaBO": 0.97000 + 0.02500j,
              "Ta": 0.94270 + 0.04170j, "SiO2": 0.97800 + 0.01070j},
    193e-9: {"vacuum": 1.0 + 0.0j, "air": 1.0 + 0.0j, "quartz": 1.5603 + 0.0j, "Cr": 0.84 + 1.65j,
             "CrON": 1.95 + 1.05j, "MoSi": 2.343 + 0.586j},
}
# expose/m3d/multilayer.py:72-77 defaults; stack.py:178-187 presets (the parts the blank uses)
_ML_DEFAULT = {"n_bilayers": 40, "period": 6.94e-9, "gamma": 0.4, "cap_material": "Ru",
               "cap_thickness": 2.5e-9, "substrate": "Si"}


def _mask_n(name, lam):
    """materials.py:85-102."""
    for w, table in _MASK_N.items():
        if abs(w - lam) <= 1e-11:
            return table[name]
    raise KeyError(f"No mask-material table at {lam * 1e9:.3f} nm")


def blank_films(optics):
    """The blank's (indices, thicknesses): stack.py:106-132 + multilayer.py:86-110;
    raises for a transmissive stack as provider.py:536-542."""
    lam = optics.wavelength
    spec = _opt(optics, "mask_stack", None)
    if spec is None:                                   # stack.py:160-169: preset by wavelength
        reflective = abs(lam - 13.5e-9) < 1e-11
        ml = dict(_ML_DEFAULT) if reflective else None
    elif not spec:                                     # stack.py:147-149: empty spec = defaults
        reflective, ml = True, dict(_ML_DEFAULT)
    else:                                              # stack.py:150-152
        reflective = spec.get("regime", "euv_reflective") == "euv_reflective"
        ml_spec = spec.get("multilayer", None)
        ml = {**_ML_DEFAULT, **ml_spec} if ml_spec else None
        if reflective and ml is None:
            raise ValueError("regime='euv_reflective' needs a multilayer")
    if not reflective:
        raise ValueError("mask_model='multilayer' describes the Bragg mirror under an EUV mask, "
                         "but the stack regime is 'duv_transmissive'.")
    t_mo = ml["period"] * ml["gamma"]
    t_si = ml["period"] - t_mo
    n = [_mask_n("vacuum", lam), _mask_n(ml["cap_material"], lam)]
    d = [0.0, ml["cap_thickness"]]
    for _ in range(ml["n_bilayers"]):
        n += [_mask_n("Si", lam), _mask_n("Mo", lam)]
        d += [t_si, t_mo]
    n.append(_mask_n(ml["substrate"], lam))
    d.append(0.0)
    return np.asarray(n, dtype=complex), np.asarray(d, dtype=np.float64)


def films_reflection(n_stored, d, lam, theta0, pol):
    """coat/films.py:168-227 — one angle, characteristic matrices multiplied
    top-down, r = (eta_0 - C/B) / (eta_0 + C/B)."""
    n = np.conj(np.asarray(n_stored, dtype=complex))
    sin0 = n[0] * np.sin(theta0)
    cos_t = np.sqrt(1.0 - (sin0 / n) ** 2)
    eta = n * cos_t if pol == "s" else n / cos_t
    M = np.eye(2, dtype=complex)
    for j in range(1, len(n) - 1):
        delta = 2.0 * np.pi * n[j] * cos_t[j] * d[j] / lam
        M = M @ np.array([[np.cos(delta), 1j * np.sin(delta) / eta[j]],
                          [1j * eta[j] * np.sin(delta), np.cos(delta)]], dtype=complex)
    b, c = M @ np.array([1.0, eta[-1]], dtype=complex)
    Y = c / b
    return complex((eta[0] - Y) / (eta[0] + Y))


def mirror_table(optics):
    """provider.py:237-250 — (theta, |r|, unwrapped arg r) of the mean s/p reflection."""
    n, d = blank_films(optics)
    lam = optics.wavelength
    theta = np.linspace(0.0, np.deg2rad(25.0), 501)
    rs = np.array([films_reflection(n, d, lam, float(t), "s") for t in theta])
    rp = np.array([films_reflection(n, d, lam, float(t), "p") for t in theta])
    r = 0.5 * (rs + rp)
    return theta, np.abs(r), np.unwrap(np.angle(r))


def mirror_reflection(table, sin_theta):
    """provider.py:252-264."""
    theta_t, mag_t, ph_t = table
    prop = sin_theta <= 1.0
    th = np.arcsin(np.clip(sin_theta, 0.0, 1.0))
    r = np.interp(th, theta_t, mag_t) * np.exp(1j * np.interp(th, theta_t, ph_t))
    return np.where(prop, r, 0.0).astype(np.complex128)


def mask_side_sines(fsx, fsy, optics):
    """provider.py:72-126."""
    lam, m = optics.wavelength, _opt(optics, "reduction", 4.0)
    sx = SOURCE_TILT_SIGN * lam * fsx / m
    sy = SOURCE_TILT_SIGN * lam * fsy / m
    cra = math.sin(math.radians(_opt(optics, "chief_ray_deg", 0.0)))
    if _opt(optics, "chief_ray_axis", "x").lower() == "x":
        sx += cra
    else:
        sy += cra
    return sx, sy


def abbe_sum(mask, optics, grid, planes, source_subset=None):
    """aerial_image.py:351-494 (thin mask) — raw (P,n,n), peak (P,), clear (P,).

    The per-source-point transforms are stacked and sent to
    ``scipy.fft.ifft2(workers=-1)`` in batches of at most ``FFT_BATCH_BYTES``,
    as the reference's ``_Batch`` does (aerial_image.py:312-348).
    ``source_subset`` (oracle-only) restricts the loop to the given source
    indices; the CPU baseline uses it to time a bounded sample.
    """
    n = int(grid.n_pixels)
    lam, NA = optics.wavelength, optics.NA
    model = _opt(optics, "imaging_model", "scalar").lower()
    if model not in IMAGING_MODELS:
        raise ValueError(
            f"imaging_model must be 'scalar' or 'vector', got '{optics.imaging_model}'")
    vector = model == "vector"
    exact = bool(_opt(optics, "exact_defocus", False)) or vector
    zern = _opt(optics, "zernike_coeffs", None) or None
    need_phi = vector or bool(zern)

    src = source_points(optics)
    M = np.fft.fft2(np.asarray(mask).astype(np.complex128))     # m3d/provider.py:177-178
    FX, FY = make_freq_grid(n, grid.pixel_size)
    mmodel = _opt(optics, "mask_model", "thin").lower()
    if mmodel not in ("thin", "multilayer"):
        raise ValueError(f"oracle images thin and multilayer masks, got mask_model={mmodel!r}")
    mirror = mirror_table(optics) if mmodel == "multilayer" else None
    if mirror is not None:                                     # provider.py:222-225
        doff_x = lam * FX / _opt(optics, "reduction", 4.0)
        doff_y = lam * FY / _opt(optics, "reduction", 4.0)
    k_max = NA / lam

    P = len(planes)
    aerial = np.zeros((P, n, n), dtype=np.float64)
    clear = np.zeros(P, dtype=np.float64)
    limit = max(1, FFT_BATCH_BYTES // (n * n * 16))
    stack, where, wts = [], [], []

    def flush():
        if not stack:
            return
        fields = sfft.ifft2(np.stack(stack), axes=(-2, -1), workers=-1)
        inten = fields.real ** 2 + fields.imag ** 2
        pl = np.asarray(where)
        w = np.asarray(wts, dtype=np.float64)
        for p in np.unique(pl):
            sel = pl == p
            aerial[p] += np.tensordot(w[sel], inten[sel], axes=1)
        stack.clear(); where.clear(); wts.clear()

    def push(spec, p, w):
        stack.append(spec); where.append(p); wts.append(w)
        if len(stack) >= limit:
            flush()

    order = range(len(src)) if source_subset is None else source_subset
    for s in order:
        w_s = float(src.weight[s])
        fsx, fsy = float(src.fx[s]), float(src.fy[s])
        M_s, clear_scale = M, 1.0
        if mirror is not None:                                 # provider.py:266-295
            sx0, sy0 = mask_side_sines(fsx, fsy, optics)
            sx, sy = sx0 + doff_x, sy0 + doff_y
            M_s = M * mirror_reflection(mirror, np.sqrt(sx * sx + sy * sy))
            clear_scale = float(abs(mirror_reflection(mirror, np.array([math.hypot(sx0, sy0)]))[0]) ** 2)
        gx, gy = FX - fsx, FY - fsy
        RHO = np.sqrt(gx ** 2 + gy ** 2) / k_max                 # aerial_image.py:136
        PHI = np.arctan2(gy, gx) if need_phi else None
        inside = RHO <= 1.0
        idx = np.nonzero(inside)
        rho_in = RHO[idx]
        phi_in = None if PHI is None else PHI[idx]
        M_in = M_s[idx]
        dc_in = float(inside[0, 0])
        states = jones_states(optics.polarisation, float(src.phi[s])) if vector else None
        for p, (dz, n_img) in enumerate(planes):
            W = pupil_phase(rho_in, phi_in, lam, NA, dz, n_img, zern, exact)
            coh = M_in * np.exp(1j * W)
            if not vector:
                spec = np.zeros((n, n), dtype=np.complex128)
                spec[idx] = coh
                push(spec, p, w_s)
                clear[p] += w_s * dc_in * clear_scale
                continue
            for jx, jy, wp in states:
                V = vector_coefficients(rho_in, phi_in, jx, jy, NA / n_img,
                                        obliquity=bool(_opt(optics, "obliquity", True)))
                for comp in V:
                    spec = np.zeros((n, n), dtype=np.complex128)
                    spec[idx] = coh * comp
                    push(spec, p, w_s * wp)
                if dc_in:
                    at = np.nonzero((idx[0] == 0) & (idx[1] == 0))[0][0]
                    clear[p] += (w_s * wp) * sum(abs(c[at]) ** 2 for c in V) * clear_scale
    flush()
    peak = aerial.reshape(P, -1).max(axis=1)
    return aerial, peak, clear


def compute_aerial_image(mask, optics, grid, dose=1.0, return_raw=False):
    """aerial_image.py:502-548."""
    raw, peak, clear = abbe_sum(mask, optics, grid,
                                [(float(_opt(optics, "defocus", 0.0)), image_index(optics))])
    a, pk, cl = raw[0], float(peak[0]), float(clear[0])
    if return_raw:
        return a, pk, cl
    return a * normalisation_scale(_opt(optics, "normalisation", "peak"), pk, cl, dose)


def compute_aerial_planes(mask, optics, grid, planes, dose=1.0):
    """aerial_image.py:551-587 — each plane normalised on its own."""
    raw, peak, clear = abbe_sum(mask, optics, grid, planes)
    for p in range(raw.shape[0]):
        raw[p] *= normalisation_scale(_opt(optics, "normalisation", "peak"),
                                      float(peak[p]), float(clear[p]), dose)
    return raw


# ---------------------------------------------------------------------------
# SOCS (expose/hopkins.py)
# ---------------------------------------------------------------------------


@dataclass
class SOCS:
    """hopkins.py:58-94 — kernels on the full grid plus their bookkeeping."""
    kernels: np.ndarray
    weights: np.ndarray
    clear: float
    energy_kept: float
    n_band: int
    n_source: int
    band: tuple
    n: int
    normalisation: str = "peak"

    def __len__(self):
        return int(self.weights.size)


def socs_band(n, pixel_size, k_max):
    """hopkins.py:144-145 — FFT-grid indices with hypot(f) <= 2 k_max (1 + 1e-9)."""
    FX, FY = make_freq_grid(n, pixel_size)
    return np.nonzero(np.hypot(FX, FY) <= 2.0 * k_max + 1e-9 * k_max), FX, FY


def socs_pupil_matrix(optics, grid):
    """hopkins.py:139-167 — A[s, band] = sqrt(w_s) exp(iW) in-aperture."""
    lam, NA = optics.wavelength, optics.NA
    k_max = NA / lam
    src = source_points(optics)
    band, FX, FY = socs_band(int(grid.n_pixels), grid.pixel_size, k_max)
    fxb, fyb = FX[band], FY[band]
    zern = _opt(optics, "zernike_coeffs", None) or None
    A = np.zeros((len(src), fxb.size), dtype=np.complex128)
    for s in range(len(src)):
        dx, dy = fxb - src.fx[s], fyb - src.fy[s]
        rho = np.hypot(dx, dy) / k_max
        inside = rho <= 1.0
        if not inside.any():
            continue
        phi = np.arctan2(dy[inside], dx[inside]) if zern else None
        W = pupil_phase(rho[inside], phi, lam, NA, float(_opt(optics, "defocus", 0.0)),
                        image_index(optics), zern, bool(_opt(optics, "exact_defocus", False)))
        A[s, inside] = np.sqrt(src.weight[s]) * np.exp(1j * W)
    return A, band, src


def socs_build(optics, grid, tol=1e-8, max_kernels=None):
    """hopkins.py:103-198 — TCC over the band, eigh, keep/trim, scatter."""
    if not (_opt(optics, "imaging_model", "scalar").lower() == "scalar"
            and _opt(optics, "mask_model", "thin") == "thin"):
        raise ValueError("SOCS kernels apply to the scalar thin-mask process only")
    n = int(grid.n_pixels)
    A, band, src = socs_pupil_matrix(optics, grid)
    tcc = A.T @ A.conj()
    ev, vec = np.linalg.eigh(tcc)
    o = np.argsort(ev)[::-1]
    ev, vec = ev[o], vec[:, o]
    trace = float(np.sum(np.clip(ev, 0.0, None)))
    keep = ev > (tol * ev[0] if ev.size else 0.0)
    keep &= ev > 0.0
    if max_kernels is not None:
        keep[max_kernels:] = False
    lam_k, vec_k = ev[keep], vec[:, keep]
    K = int(lam_k.size)
    kern = np.zeros((K, n, n), dtype=np.complex128)
    for k in range(K):
        kern[k][band] = vec_k[:, k]
    dc = np.nonzero((band[0] == 0) & (band[1] == 0))[0]
    clear = float(np.sum(lam_k * np.abs(vec_k[dc[0], :]) ** 2)) if dc.size else 0.0
    kept = float(lam_k.sum() / trace) if trace > 0 else 1.0
    return SOCS(kern, lam_k, clear, kept, int(band[0].size), len(src), band, n,
                _opt(optics, "normalisation", "peak"))


def socs_raw(k: SOCS, mask):
    """hopkins.py:205-218."""
    if mask.shape != (k.n, k.n):
        raise ValueError(f"mask must be {(k.n, k.n)} for these kernels, got {mask.shape}")
    M = np.fft.fft2(np.asarray(mask, dtype=np.complex128))
    f = sfft.ifft2(k.kernels * M[None], axes=(-2, -1), workers=-1)
    inten = np.tensordot(k.weights, f.real ** 2 + f.imag ** 2, axes=1)
    return inten, float(inten.max()), k.clear


def socs_image(k: SOCS, mask, dose=1.0):
    """hopkins.py:220-223."""
    raw, peak, clear = socs_raw(k, mask)
    return raw * normalisation_scale(k.normalisation, peak, clear, dose)


# ---------------------------------------------------------------------------
# ILT (opc/ilt.py)
# ---------------------------------------------------------------------------


def socs_fields(k: SOCS, mask):
    """opc/ilt.py:208-232 — fields kept, numpy FFT as the reference."""
    if mask.shape != (k.n, k.n):
        raise ValueError(f"mask must be {(k.n, k.n)} for these kernels, got {mask.shape}")
    spec = np.fft.fft2(np.asarray(mask, dtype=np.complex128))
    fields = np.fft.ifft2(k.kernels * spec[None], axes=(-2, -1))
    inten = np.tensordot(k.weights, fields.real ** 2 + fields.imag ** 2, axes=1)
    return fields, inten


def socs_gradient(k: SOCS, fields, sensitivity):
    """opc/ilt.py:235-266 — 2 Re sum_k lam_k F^-1(conj(phi_k) F(G E_k))."""
    g = np.asarray(sensitivity, dtype=np.float64)
    back = np.fft.fft2(g[None] * fields)
    adj = np.fft.ifft2(np.conj(k.kernels) * back, axes=(-2, -1))
    return 2.0 * np.real(np.tensordot(k.weights, adj, axes=1))


def blur(a, sigma_px):
    """opc/ilt.py:274-289 — scipy gaussian_filter, mode 'reflect', truncate 4."""
    if sigma_px < 1e-3:
        return a
    return gaussian_filter(a, sigma=sigma_px)


def apply_peb(pac_map, diffusion_sigma, pixel_size):
    """bake/peb.py:24-70 — Gaussian PEB diffusion (scipy, reflect), clipped to [0, 1]."""
    a = np.asarray(pac_map)
    if a.ndim != 2:
        raise ValueError(f"apply_peb expects a 2-D (ny, nx) map, got ndim={a.ndim}")
    if diffusion_sigma < 0:
        raise ValueError(f"diffusion_sigma must be >= 0, got {diffusion_sigma!r}")
    if pixel_size <= 0:
        raise ValueError(f"pixel_size must be > 0, got {pixel_size!r}")
    sigma_px = diffusion_sigma / pixel_size
    if sigma_px < 1e-3:
        return a.copy()
    return np.clip(gaussian_filter(a.astype(np.float64), sigma=sigma_px), 0.0, 1.0)


def dose_focus_images(mask, optics, grid, doses, defoci_nm, normalisation="clear"):
    """analysis/process_window.py:215-300 (the imaging part of sweep_dose_focus):
    one Abbe sum per defocus, each dose a rescale of the raw sum. (F, D, N, N)."""
    import copy

    def _with(o, **kw):
        c = copy.copy(o)
        for k, v in kw.items():
            setattr(c, k, v)
        return c
    base = optics
    if normalisation is not None and normalisation != getattr(optics, "normalisation", "peak"):
        base = _with(optics, normalisation=normalisation)
    out = []
    for d_nm in defoci_nm:
        local = _with(base, defocus=d_nm * 1e-9)
        raw, peak, clear = compute_aerial_image(mask, local, grid, return_raw=True)
        out.append([raw * normalisation_scale(base.normalisation, peak, clear, dose) for dose in doses])
    return np.array(out)


def focus_reference_depth(resist):
    """develop/resist3d.py:66-81 — the depth the optics' defocus refers to."""
    ref = resist.focus_reference
    if ref == "top":
        return 0.0
    if ref == "mid":
        return resist.thickness / 2.0
    if ref == "bottom":
        return resist.thickness
    raise ValueError(f"focus_reference must be 'top', 'mid', or 'bottom', got '{ref}'")


def effective_defocus(depth, optics, resist):
    """develop/resist3d.py:84-110."""
    return optics.defocus - (depth - focus_reference_depth(resist)) * (optics.n_immersion / resist.n_resist)


def exposure_volume(mask, optics, grid, resist, dose=1.0):
    """develop/resist3d.py:113-193 — n_slices optical planes through the film
    (resist as the image medium, defocus in resist units), then np.interp per
    pixel onto the voxel planes, iz = 0 at the bottom. (intensity, z)."""
    nz = max(int(round(resist.thickness / grid.dz)), 1)
    n_slices = int(np.clip(grid.n_z_slices, 2, nz))
    depths = np.linspace(0.0, resist.thickness, n_slices)
    ratio = resist.n_resist / optics.n_immersion
    planes = compute_aerial_planes(mask, optics, grid,
                                   [(effective_defocus(float(d), optics, resist) * ratio, resist.n_resist)
                                    for d in depths], dose=dose)
    zq = ((np.arange(nz) + 0.5) * grid.dz)[::-1]
    flat = planes.reshape(n_slices, -1)
    out = np.empty((nz, flat.shape[1]), dtype=np.float64)
    for k in range(flat.shape[1]):
        out[:, k] = np.interp(zq, depths, flat[:, k])
    return out.reshape(nz, grid.n_pixels, grid.n_pixels), (np.arange(nz) + 0.5) * grid.dz


def objective(k: SOCS, target, mask, scale, level, sigma_px, sign, steepness,
              weight_tv=0.0, weight_discrete=0.0):
    """opc/ilt.py:311-360 — (cost, grad, signed, pattern_error)."""
    fields, raw = socs_fields(k, mask)
    fld = blur(raw * scale, sigma_px)
    signed = sign * (fld - level)
    a = steepness / max(abs(level), 1e-12)
    z = 1.0 / (1.0 + np.exp(-np.clip(a * signed, -60.0, 60.0)))
    resid = z - target
    npix = float(resid.size)
    cost = float(np.sum(resid ** 2) / npix)
    dz = (2.0 / npix) * resid * (a * z * (1.0 - z))
    d_int = blur(sign * dz, sigma_px) * scale
    grad = socs_gradient(k, fields, d_int)
    if weight_tv > 0.0:
        lap = (np.roll(mask, 1, 0) + np.roll(mask, -1, 0) + np.roll(mask, 1, 1)
               + np.roll(mask, -1, 1) - 4.0 * mask)
        gx = mask - np.roll(mask, 1, 1)
        gy = mask - np.roll(mask, 1, 0)
        cost += weight_tv * float(np.sum(gx ** 2 + gy ** 2) / npix)
        grad += weight_tv * (-2.0 / npix) * lap
    if weight_discrete > 0.0:
        cost += weight_discrete * float(np.sum(mask * (1.0 - mask)) / npix)
        grad += weight_discrete * (1.0 - 2.0 * mask) / npix
    perr = int(np.count_nonzero((signed > 0.0) != (target > 0.5)))
    return cost, grad, signed, perr


def mask_of(theta, beta, smooth_px):
    """opc/ilt.py:368-378 — sigma(beta * G(theta)), clip +-60."""
    f = blur(theta, smooth_px)
    return 1.0 / (1.0 + np.exp(-np.clip(beta * f, -60.0, 60.0)))


def grad_theta(grad_mask, mask, beta, smooth_px):
    """opc/ilt.py:381-389."""
    return blur(grad_mask * (beta * mask * (1.0 - mask)), smooth_px)


def adam_step(theta, mom1, mom2, grad_t, it, step, b1=0.9, b2=0.999, eps=1e-8):
    """opc/ilt.py:582-591 — one Adam update at iteration ``it`` (1-based)."""
    mom1 = b1 * mom1 + (1.0 - b1) * grad_t
    mom2 = b2 * mom2 + (1.0 - b2) * grad_t ** 2
    m_hat = mom1 / (1.0 - b1 ** it)
    v_hat = mom2 / (1.0 - b2 ** it)
    return theta - step * m_hat / (np.sqrt(v_hat) + eps), mom1, mom2


# ---------------------------------------------------------------------------
# Masks (mask/patterns.py) — synthetic inputs
# ---------------------------------------------------------------------------


def lines_and_spaces(n, pixel_size, pitch, cd, orientation="vertical"):
    """mask/patterns.py:22-66."""
    coords = (np.arange(n) - n // 2) * pixel_size
    line = (np.mod(coords + pitch / 2, pitch) < cd).astype(np.float64)
    if orientation == "vertical":
        return np.tile(line[np.newaxis, :], (n, 1))
    return np.tile(line[:, np.newaxis], (1, n))


def contact_array(n, pixel_size, pitch_x, pitch_y, cd_x, cd_y=None):
    """mask/patterns.py:69-107."""
    cd_y = cd_x if cd_y is None else cd_y
    coords = (np.arange(n) - n // 2) * pixel_size
    ox = (np.mod(coords + pitch_x / 2, pitch_x) < cd_x).astype(np.float64)
    oy = (np.mod(coords + pitch_y / 2, pitch_y) < cd_y).astype(np.float64)
    return np.outer(oy, ox)


def to_attenuated_psm(mask, transmission=0.06, phase_shift_deg=180.0):
    """mask/patterns.py:178-208 — amplitude sqrt(T) e^{i phi} on 1-regions."""
    ph = np.deg2rad(phase_shift_deg)
    return np.where(mask > 0.5, np.sqrt(transmission) * np.exp(1j * ph),
                    1.0 + 0.0j).astype(np.complex128)
