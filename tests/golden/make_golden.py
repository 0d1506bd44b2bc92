"""Generate the golden fixtures in this folder from the reference itself.

Run in a container that has the reference checked out, with
``LITHO_REFERENCE`` naming its root (the folder that holds ``src/litho_sim``)::

    LITHO_REFERENCE=<path to the reference checkout> python tests/golden/make_golden.py

It imports the reference package ``litho_sim`` from ``<ref>/src`` unmodified.
``litho_sim.opc`` imports matplotlib for layout rasterisation (mask/geometry.py),
which is off the imaging path and not installed here, so a throw-away stub
package is put on ``sys.path`` for the import only.

Each case is one ``.npz`` with the inputs (or the parameters that rebuild
them), the optics/grid as JSON, and the reference's outputs in float64. The
fixtures pin ``oracle/litho_oracle.py`` (CPU tests) and the CUDA path
(GPU tests). Nothing at test time reads the reference.
"""

from __future__ import annotations

import dataclasses
import json
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _reference_root() -> Path:
    root = os.environ.get("LITHO_REFERENCE")
    if not root:
        raise SystemExit("set LITHO_REFERENCE to the reference checkout (the folder holding src/litho_sim)")
    path = Path(root)
    if not (path / "src" / "litho_sim").is_dir():
        raise SystemExit(f"LITHO_REFERENCE={root!r} does not hold src/litho_sim")
    return path


def _import_reference():
    REF = _reference_root()
    stub = Path(tempfile.mkdtemp()) / "matplotlib"
    stub.mkdir()
    (stub / "__init__.py").write_text("")
    (stub / "path.py").write_text(
        "class Path:\n    def __init__(self, *a, **k):\n"
        "        raise RuntimeError('matplotlib stub: layout rasterisation unavailable')\n")
    sys.path[:0] = [str(REF / "src"), str(stub.parent)]
    import litho_sim  # noqa: F401
    return litho_sim


def optics_dict(o) -> dict:
    d = dataclasses.asdict(o)
    d["zernike_coeffs"] = {str(k): v for k, v in (o.zernike_coeffs or {}).items()}
    return d


def grid_dict(g) -> dict:
    return {"n_pixels": g.n_pixels, "pixel_size": g.pixel_size}


def save(name: str, optics=None, grid=None, **arrays):
    meta = {}
    if optics is not None:
        meta["optics"] = optics_dict(optics)
    if grid is not None:
        meta["grid"] = grid_dict(grid)
    np.savez_compressed(HERE / f"{name}.npz", meta=np.array(json.dumps(meta)), **arrays)
    print(f"  {name}: {sorted(arrays)}")


def manhattan_clip(rng, n, px, n_rect=(20, 60), width_nm=(40, 200)):
    """Union of axis-aligned rectangles, pixel aligned (the batched-clip inputs)."""
    m = np.zeros((n, n), dtype=np.float64)
    for _ in range(int(rng.integers(n_rect[0], n_rect[1] + 1))):
        w = max(1, int(round(rng.uniform(*width_nm) * 1e-9 / px)))
        h = max(1, int(round(rng.uniform(*width_nm) * 1e-9 / px)))
        x0, y0 = int(rng.integers(0, n)), int(rng.integers(0, n))
        m[y0:y0 + h, x0:x0 + w] = 1.0
    return m


def main():
    _import_reference()
    from litho_sim.core.config import GridConfig, OpticsConfig
    from litho_sim.expose import (SOCSKernels, compute_aerial_image, compute_aerial_planes,
                                  source_points)
    from litho_sim.expose.pupil import (defocus_opd, jones_states, vector_coefficients,
                                        zernike_noll)
    from litho_sim.expose.source import Source
    from litho_sim.mask.patterns import (contact_array, lines_and_spaces,
                                         to_attenuated_psm)
    from litho_sim.opc.ilt import (_grad_theta, _mask_of, _Objective, socs_fields,
                                   socs_gradient)

    print("golden fixtures ->", HERE)

    # --- pupil functions on scattered points --------------------------------
    rng = np.random.default_rng(11)
    rho = np.concatenate([rng.random(200) * 1.05, [0.0, 1.0, 0.5]])
    phi = np.concatenate([rng.uniform(-np.pi, np.pi, 200), [0.0, np.pi, -np.pi / 2]])
    Z = np.stack([zernike_noll(j, rho, phi) for j in range(1, 23)])
    dpar = defocus_opd(rho, 193e-9, 1.35, 80e-9, 1.44, exact=False)
    dexa = defocus_opd(rho, 193e-9, 1.35, 80e-9, 1.44, exact=True)
    V = []
    for pol in ("x", "y", "te", "tm", "unpolarised"):
        for jx, jy, _w in jones_states(pol, 0.7):
            V.append(np.stack(vector_coefficients(rho, phi, jx, jy, 1.35 / 1.7, True)))
            V.append(np.stack(vector_coefficients(rho, phi, jx, jy, 1.35 / 1.7, False)))
    save("pupil_functions", rho=rho, phi=phi, zernike=Z, defocus_paraxial=dpar,
         defocus_exact=dexa, vector=np.stack(V))

    # --- source point lists ---------------------------------------------------
    src_cases = {
        "annular31": OpticsConfig(source_type="annular", sigma_inner=0.5, sigma_outer=0.8,
                                  source_grid=31),
        "annular31_imm": OpticsConfig(NA=1.35, n_immersion=1.44, source_type="annular",
                                      sigma_inner=0.5, sigma_outer=0.9, source_grid=31),
        "conventional21": OpticsConfig(),
        "dipole_legacy": OpticsConfig(source_type="dipole", sigma_outer=0.9, sigma_inner=0.6,
                                      source_grid=11, source_kwargs={"axis": "y"}),
        "quadrupole_legacy": OpticsConfig(source_type="quadrupole", sigma_outer=0.9,
                                          sigma_inner=0.6, source_grid=15),
        "cquad_spec": OpticsConfig(NA=1.35, n_immersion=1.44, source_spec=Source.quadrupole(
            sigma_outer=0.9, sigma_inner=0.7, opening_deg=30, rotation_deg=0).to_dict()),
        "euv_dipole43": OpticsConfig(wavelength=13.5e-9, NA=0.33, source_grid=43,
                                     source_spec=Source.dipole(0.9, 0.6, opening_deg=60).to_dict()),
        "quasar_blur": OpticsConfig(source_grid=25, source_spec=Source.quasar(
            0.9, 0.6, blur=0.03).to_dict()),
        "monopole": OpticsConfig(source_type="monopole", sigma_outer=0.9, sigma_inner=0.5,
                                 source_grid=17, source_kwargs={"angle_deg": 30.0}),
    }
    for name, o in src_cases.items():
        sp = source_points(o)
        save(f"source_{name}", optics=o, grid=None, weight=sp.weight, fx=sp.fx, fy=sp.fy,
             phi=sp.phi)

    # --- Abbe: the reference's own small test optics ---------------------------
    g64 = GridConfig(n_pixels=64, pixel_size=4e-9)
    ls64 = lines_and_spaces(64, 4e-9, pitch=128e-9, cd=64e-9)
    abbe_cases = {
        "conventional": dict(NA=0.93, sigma_outer=0.8, source_grid=9),
        "annular_aberrated": dict(NA=0.93, source_type="annular", sigma_outer=0.85,
                                  sigma_inner=0.5, source_grid=11, defocus=120e-9,
                                  zernike_coeffs={7: 0.03, 11: -0.02}),
        "dipole_exact_clear": dict(NA=1.35, n_immersion=1.44, n_image=1.7, source_type="dipole",
                                   source_kwargs={"axis": "x"}, sigma_outer=0.9,
                                   sigma_inner=0.6, source_grid=11, defocus=-60e-9,
                                   exact_defocus=True, normalisation="clear"),
    }
    for name, kw in abbe_cases.items():
        o = OpticsConfig(**kw)
        raw, peak, clear = compute_aerial_image(ls64, o, g64, return_raw=True)
        img = compute_aerial_image(ls64, o, g64, dose=1.3)
        save(f"abbe_{name}", optics=o, grid=g64, mask=ls64, raw=raw, peak=peak, clear=clear,
             image_dose13=img)

    # vector model, every polarisation (test_vector_imaging.py style optics)
    rng = np.random.default_rng(5)
    cmask = contact_array(64, 4e-9, 96e-9, 96e-9, 48e-9)
    psm = to_attenuated_psm(1.0 - cmask, transmission=0.06, phase_shift_deg=180.0)
    for pol in ("te", "tm", "x", "y", "unpolarised"):
        o = OpticsConfig(NA=1.35, n_immersion=1.44, imaging_model="vector", polarisation=pol,
                         source_type="annular", sigma_outer=0.9, sigma_inner=0.5,
                         source_grid=9, defocus=30e-9, zernike_coeffs={5: 0.02, 9: -0.01})
        raw, peak, clear = compute_aerial_image(psm, o, g64, return_raw=True)
        save(f"abbe_vector_{pol}", optics=o, grid=g64, mask=psm, raw=raw, peak=peak,
             clear=clear)

    # planes (test_hopkins.py:61-72 optics, four planes)
    o = OpticsConfig(**abbe_cases["annular_aberrated"])
    planes = np.array([(-100e-9, 1.7), (0.0, 1.7), (45e-9, 1.7), (150e-9, 1.44)])
    stack = compute_aerial_planes(ls64, o, g64, [tuple(p) for p in planes], dose=1.3)
    save("planes_scalar", optics=o, grid=g64, mask=ls64, planes=planes, stack=stack)
    ov = OpticsConfig(NA=1.35, n_immersion=1.44, imaging_model="vector", polarisation="te",
                      source_type="dipole", source_kwargs={"axis": "x"}, sigma_outer=0.9,
                      sigma_inner=0.6, source_grid=9, normalisation="clear")
    planes_v = np.array([(0.0, 1.7), (80e-9, 1.7)])
    stack_v = compute_aerial_planes(ls64, ov, g64, [tuple(p) for p in planes_v])
    save("planes_vector", optics=ov, grid=g64, mask=ls64, planes=planes_v, stack=stack_v)

    # --- the first workload at full size: scalar Abbe, ArF dry, 256^2 ------------
    o1 = OpticsConfig(wavelength=193e-9, NA=0.93, source_type="annular", sigma_inner=0.5,
                      sigma_outer=0.8, source_grid=31)
    g1 = GridConfig(n_pixels=256, pixel_size=4e-9)
    m1 = lines_and_spaces(256, 4e-9, 200e-9, 100e-9)
    raw, peak, clear = compute_aerial_image(m1, o1, g1, return_raw=True)
    save("c1_scalar_256", optics=o1, grid=g1, raw=raw, peak=peak, clear=clear,
         image=compute_aerial_image(m1, o1, g1))

    # --- a batched-clip style case: immersion cquad, defocus + Z4..Z21 ----------
    rng = np.random.default_rng(2024)
    g2 = GridConfig(n_pixels=128, pixel_size=2e-9)
    m2 = manhattan_clip(rng, 128, 2e-9, n_rect=(8, 16))
    zern = {j: float(rng.uniform(-0.02, 0.02)) for j in range(4, 22)}
    o2 = OpticsConfig(NA=1.35, n_immersion=1.44, defocus=float(rng.uniform(-60e-9, 60e-9)),
                      zernike_coeffs=zern, source_spec=Source.quadrupole(
                          sigma_outer=0.9, sigma_inner=0.7, opening_deg=30,
                          rotation_deg=0).to_dict())
    raw, peak, clear = compute_aerial_image(m2.astype(np.complex64), o2, g2, return_raw=True)
    save("c2_clip_128", optics=o2, grid=g2, mask=m2.astype(np.uint8), raw=raw, peak=peak,
         clear=clear)

    # --- vector TE att-PSM contacts (scaled-down third workload) ----------------
    g3 = GridConfig(n_pixels=128, pixel_size=2e-9)
    c3 = contact_array(128, 2e-9, 100e-9, 100e-9, 55e-9)
    m3 = to_attenuated_psm(1.0 - c3, transmission=0.06, phase_shift_deg=180.0)
    o3 = OpticsConfig(NA=1.35, n_immersion=1.44, imaging_model="vector", polarisation="te",
                      source_type="annular", sigma_inner=0.5, sigma_outer=0.9, source_grid=15)
    raw, peak, clear = compute_aerial_image(m3, o3, g3, return_raw=True)
    save("c3_vector_128", optics=o3, grid=g3, mask=m3, raw=raw, peak=peak, clear=clear)

    # --- SOCS ------------------------------------------------------------------
    for name, kw in abbe_cases.items():
        o = OpticsConfig(**kw)
        full = SOCSKernels.build(o, g64, tol=0.0)
        trimmed = SOCSKernels.build(o, g64)
        capped = SOCSKernels.build(o, g64, max_kernels=3)
        rf, pf, cf = full.raw(ls64)
        rt, pt, ct = trimmed.raw(ls64)
        save(f"socs_{name}", optics=o, grid=g64, mask=ls64,
             weights_full=full.weights, weights_tol=trimmed.weights,
             weights_cap3=capped.weights, clear_full=full.clear, clear_tol=trimmed.clear,
             energy_tol=trimmed.energy_kept, energy_cap3=capped.energy_kept,
             n_band=full.n_band, n_source=full.n_source, raw_full=rf, raw_tol=rt,
             raw_cap3=capped.raw(ls64)[0], peak_full=pf, image_tol=trimmed.image(ls64, 0.8))

    # SOCS ILT-style optics (ArF immersion annular, clear normalisation), mid size
    o4 = OpticsConfig(wavelength=193e-9, NA=1.35, n_immersion=1.44, source_type="annular",
                      sigma_inner=0.5, sigma_outer=0.8, normalisation="clear")
    g4 = GridConfig(n_pixels=128, pixel_size=4e-9)
    k4 = SOCSKernels.build(o4, g4, tol=0.0, max_kernels=24)
    kall = SOCSKernels.build(o4, g4, tol=0.0)
    m4 = manhattan_clip(np.random.default_rng(7), 128, 4e-9, n_rect=(6, 12))
    r4 = k4.raw(m4)
    save("socs_imm_128_k24", optics=o4, grid=g4, mask=m4.astype(np.uint8),
         weights=k4.weights, weights_all=kall.weights, clear=k4.clear,
         energy=k4.energy_kept, n_band=k4.n_band, n_source=k4.n_source, raw=r4[0],
         peak=r4[1])

    # the fourth workload's decomposition at full size (weights only: small)
    g4f = GridConfig(n_pixels=1024, pixel_size=1e-9)
    k4f = SOCSKernels.build(o4, g4f, tol=0.0, max_kernels=26)
    save("socs_imm_1024_weights", optics=o4, grid=g4f, weights=k4f.weights,
         clear24=float(np.sum(k4f.weights[:24] * np.abs(
             k4f.kernels[:24, 0, 0]) ** 2)),
         energy24=float(k4f.weights[:24].sum() / k4f.weights.sum() * k4f.energy_kept),
         n_band=k4f.n_band, n_source=k4f.n_source)

    # --- ILT adjoint and objective (test_ilt.py 'small' fixture) ----------------
    gs = GridConfig(n_pixels=32, pixel_size=8e-9)
    ks = SOCSKernels.build(OpticsConfig(), gs, tol=1e-6)
    rng = np.random.default_rng(2)
    mask = rng.random((32, 32))
    sens = rng.standard_normal((32, 32))
    fields, inten = socs_fields(ks, mask)
    grad = socs_gradient(ks, fields, sens)
    rng = np.random.default_rng(3)
    mask3 = rng.random((32, 32))
    target3 = (rng.random((32, 32)) > 0.5).astype(float)
    obj = _Objective(kernels=ks, target=target3, scale=1.7, level=0.3, sigma_px=1.5,
                     sign=1.0, steepness=12.0, weight_tv=1e-3, weight_discrete=1e-3)
    cost, g_obj, signed, perr = obj(mask3)
    obj0 = _Objective(kernels=ks, target=target3, scale=2.0, level=0.3, sigma_px=0.0,
                      sign=-1.0, steepness=20.0, weight_tv=0.0, weight_discrete=0.0)
    cost0, g_obj0, signed0, perr0 = obj0(mask3)
    rng = np.random.default_rng(5)
    theta = 0.5 * rng.standard_normal((32, 32))
    m_of = _mask_of(theta, 6.0, 2.0)
    g_th = _grad_theta(g_obj, m_of, 6.0, 2.0)
    save("ilt_small", optics=OpticsConfig(), grid=gs, weights=ks.weights, clear=ks.clear,
         mask=mask, sens=sens, intensity=inten, grad=grad, mask3=mask3, target3=target3,
         cost=cost, grad_obj=g_obj, signed=signed, perr=perr, cost0=cost0,
         grad_obj0=g_obj0, signed0=signed0, perr0=perr0, theta=theta, mask_of=m_of,
         grad_theta=g_th)

    # ILT at the fourth workload's optics, scaled down: 128^2, K=24, no blur
    rng = np.random.default_rng(9)
    theta = 0.5 * rng.standard_normal((128, 128))
    target = manhattan_clip(np.random.default_rng(10), 128, 4e-9, n_rect=(6, 12))
    m = 1.0 / (1.0 + np.exp(-np.clip(4.0 * theta, -60, 60)))
    objk = _Objective(kernels=k4, target=target, scale=1.0 / k4.clear, level=0.3,
                      sigma_px=0.0, sign=1.0, steepness=50.0 * 0.3, weight_tv=0.0,
                      weight_discrete=0.0)
    cost, gk, signed, perr = objk(m)
    save("ilt_imm_128_k24", optics=o4, grid=g4, theta=theta, target=target.astype(np.uint8),
         beta=4.0, cost=cost, grad=gk, signed=signed, perr=perr)
    wide()
    next_rows()
    print("done")


def wide():
    """EUV cases whose pupil is wider than 15 bins (coarse grids above 64)."""
    _import_reference()
    from litho_sim.core.config import GridConfig, OpticsConfig
    from litho_sim.expose import SOCSKernels, compute_aerial_image
    from litho_sim.expose.source import Source

    # 256^2 at 2.5 nm: pupil radius 15.6 bins (h = 16)
    g = GridConfig(n_pixels=256, pixel_size=2.5e-9)
    o = OpticsConfig(wavelength=13.5e-9, NA=0.33, source_grid=21, defocus=20e-9,
                     zernike_coeffs={5: 0.01, 8: -0.008},
                     source_spec=Source.dipole(0.9, 0.6, opening_deg=60).to_dict())
    m = manhattan_clip(np.random.default_rng(31), 256, 2.5e-9, n_rect=(10, 20), width_nm=(20, 80))
    raw, peak, clear = compute_aerial_image(m, o, g, return_raw=True)
    save("euv_wide_256", optics=o, grid=g, mask=m.astype(np.uint8), raw=raw, peak=peak, clear=clear)

    # SOCS with a 31-bin kernel band (128^2 at 5 nm), 24 kernels
    g = GridConfig(n_pixels=128, pixel_size=5e-9)
    o = OpticsConfig(wavelength=13.5e-9, NA=0.33, source_grid=15, normalisation="clear",
                     source_spec=Source.dipole(0.9, 0.6, opening_deg=60).to_dict())
    k = SOCSKernels.build(o, g, tol=0.0, max_kernels=24)
    m = manhattan_clip(np.random.default_rng(32), 128, 5e-9, n_rect=(6, 12), width_nm=(20, 80))
    r = k.raw(m)
    save("socs_euv_wide_128_k24", optics=o, grid=g, mask=m.astype(np.uint8), weights=k.weights,
         clear=k.clear, n_band=k.n_band, raw=r[0], peak=r[1])

    # the SOCS adjoint with those kernels (opc/ilt.py:235-266), the wide-band ILT gradient
    from litho_sim.opc.ilt import socs_fields, socs_gradient
    rng = np.random.default_rng(33)
    mask = rng.random((128, 128))
    sens = rng.standard_normal((128, 128))
    fields, inten = socs_fields(k, mask)
    save("ilt_euv_wide_128_k24", optics=o, grid=g, mask=mask, sens=sens, intensity=inten,
         grad=socs_gradient(k, fields, sens))


def next_rows():
    """Rows beyond the imaging core: PEB diffusion (bake/peb.py) and the
    imaging part of the dose-focus sweep (analysis/process_window.py)."""
    _import_reference()
    import dataclasses

    from litho_sim.bake.peb import apply_peb
    from litho_sim.core.config import GridConfig, OpticsConfig
    from litho_sim.expose import compute_aerial_image, normalisation_scale
    rng = np.random.default_rng(41)
    pac = rng.random((96, 96))
    save("peb_small", pac=pac, sigma=np.array([7e-9, 0.0]), px=np.array(4e-9),
         out=apply_peb(pac, 7e-9, 4e-9), out0=apply_peb(pac, 0.0, 4e-9))
    g = GridConfig(n_pixels=64, pixel_size=4e-9)
    o = OpticsConfig(NA=0.93, source_type="annular", sigma_inner=0.5, sigma_outer=0.85, source_grid=11,
                     normalisation="clear")
    m = manhattan_clip(np.random.default_rng(42), 64, 4e-9, n_rect=(4, 8), width_nm=(40, 120))
    defoci, doses = [-60.0, 0.0, 45.0], [0.8, 1.0, 1.25]
    stack = []
    for d_nm in defoci:
        local = dataclasses.replace(o, defocus=d_nm * 1e-9)
        raw, peak, clear = compute_aerial_image(m, local, g, return_raw=True)
        stack.append([raw * normalisation_scale(o.normalisation, peak, clear, dose) for dose in doses])
    save("dose_focus_64", optics=o, grid=g, mask=m.astype(np.uint8), defoci=np.array(defoci),
         doses=np.array(doses), stack=np.array(stack))


def volume():
    """The depth-resolved aerial image through a resist film
    (develop/resist3d.py:exposure_volume): a scalar and a vector case."""
    _import_reference()
    from litho_sim.core.config import GridConfig, OpticsConfig, ResistConfig
    from litho_sim.develop.resist3d import exposure_volume
    cases = [
        ("volume_scalar_64",
         OpticsConfig(NA=0.93, source_type="annular", sigma_inner=0.5, sigma_outer=0.85, source_grid=11,
                      defocus=20e-9),
         GridConfig(n_pixels=64, pixel_size=4e-9, dz=6e-9, n_z_slices=5),
         ResistConfig(thickness=60e-9, focus_reference="bottom"), 43, 1.0),
        ("volume_vector_64",
         OpticsConfig(wavelength=193e-9, NA=1.35, n_immersion=1.44, imaging_model="vector", polarisation="te",
                      source_type="annular", sigma_inner=0.5, sigma_outer=0.9, source_grid=11,
                      normalisation="clear", defocus=-15e-9),
         GridConfig(n_pixels=64, pixel_size=4e-9, dz=4e-9, n_z_slices=7),
         ResistConfig(thickness=50e-9, n_resist=1.72, focus_reference="mid"), 44, 1.3),
    ]
    for name, o, g, r, seed, dose in cases:
        m = manhattan_clip(np.random.default_rng(seed), g.n_pixels, g.pixel_size, n_rect=(4, 10),
                           width_nm=(40, 160))
        vol, z = exposure_volume(m, o, g, r, dose=dose)
        save(name, optics=o, grid=g, mask=m.astype(np.uint8), dz=np.array(g.dz), n_z_slices=np.array(g.n_z_slices),
             thickness=np.array(r.thickness), n_resist=np.array(r.n_resist),
             focus_reference=np.array(r.focus_reference), dose=np.array(dose), volume=vol, z=z)


def multilayer():
    """The EUV blank as a Bragg mirror (mask_model="multilayer",
    expose/m3d/provider.py:190-295): images, the reflection table, the
    clear-field factors and the reflection at chosen direction sines."""
    _import_reference()
    import dataclasses

    from litho_sim.core.config import GridConfig, OpticsConfig
    from litho_sim.expose import compute_aerial_image, compute_aerial_planes
    from litho_sim.expose.m3d import MaskStack
    from litho_sim.expose.m3d.provider import MultilayerSpectra
    from litho_sim.expose.source import Source
    from litho_sim.mask.patterns import lines_and_spaces

    # the reference test's grating (tests/test_m3d.py:211-231): 32 nm half pitch at 2 nm
    g = GridConfig(n_pixels=128, pixel_size=2e-9)
    m = lines_and_spaces(128, 2e-9, pitch=64e-9, cd=32e-9)
    base = OpticsConfig(wavelength=13.5e-9, NA=0.33, sigma_outer=0.6, source_grid=11, chief_ray_deg=6.0,
                        reduction=4.0, normalisation="clear", mask_model="multilayer")
    for name, o in (("ml_ls_128_cra6", base),
                    ("ml_ls_128_cram6", dataclasses.replace(base, chief_ray_deg=-6.0)),
                    ("ml_ls_128_thin", dataclasses.replace(base, mask_model="thin"))):
        raw, peak, clear = compute_aerial_image(m, o, g, return_raw=True)
        save(name, optics=o, grid=g, mask=m.astype(np.uint8), raw=raw, peak=peak, clear=clear)

    # through focus (the best-focus shift, tests/test_m3d.py:258-278), one planes call
    foci = np.linspace(-40e-9, 40e-9, 9)
    planes = [(float(d), 1.0) for d in foci]
    stack = compute_aerial_planes(m, base, g, planes)
    save("ml_ls_128_focus", optics=base, grid=g, mask=m.astype(np.uint8), foci=foci, images=np.asarray(stack))

    # a Manhattan clip: dipole, y chief ray, Zernikes, a custom stack, peak normalisation
    g2 = GridConfig(n_pixels=256, pixel_size=2e-9)
    o2 = OpticsConfig(wavelength=13.5e-9, NA=0.33, source_grid=17, chief_ray_deg=5.0, chief_ray_axis="y",
                      defocus=15e-9, zernike_coeffs={7: 0.02, 9: -0.01}, mask_model="multilayer",
                      mask_stack={"regime": "euv_reflective", "absorber": "TaBN", "absorber_thickness": 60e-9,
                                  "substrate": "SiO2",
                                  "multilayer": {"n_bilayers": 30, "period": 7.0e-9, "gamma": 0.42}},
                      source_spec=Source.dipole(0.9, 0.6, opening_deg=60).to_dict())
    m2 = manhattan_clip(np.random.default_rng(51), 256, 2e-9, n_rect=(10, 20), width_nm=(20, 80))
    raw, peak, clear = compute_aerial_image(m2, o2, g2, return_raw=True)
    save("ml_dipole_256", optics=o2, grid=g2, mask=m2.astype(np.uint8), raw=raw, peak=peak, clear=clear)

    # wide pupil (512^2 at 2 nm: coarse grid 128), vector TE model
    g3 = GridConfig(n_pixels=512, pixel_size=2e-9)
    o3 = OpticsConfig(wavelength=13.5e-9, NA=0.33, source_type="annular", sigma_inner=0.5, sigma_outer=0.8,
                      source_grid=9, chief_ray_deg=6.0, mask_model="multilayer", imaging_model="vector",
                      polarisation="te", normalisation="clear")
    m3 = manhattan_clip(np.random.default_rng(52), 512, 2e-9, n_rect=(20, 40), width_nm=(20, 80))
    raw, peak, clear = compute_aerial_image(m3, o3, g3, return_raw=True)
    save("ml_vector_512", optics=o3, grid=g3, mask=m3.astype(np.uint8), raw=raw.astype(np.float32), peak=peak,
         clear=clear)

    # the reflection itself: table, clear factors, values at chosen sines
    stack = MaskStack.for_wavelength(13.5e-9)
    sp = MultilayerSpectra(np.ones((128, 128)), base, g, stack)
    sines = np.array([0.0, 0.02, 0.05, 0.1045, 0.15, 0.2, 0.3, 0.5, 1.0, 1.4, 12.0])
    fs = np.array([[0.0, 0.0], [1.2e6, -0.7e6], [-2.0e6, 1.5e6], [4.0e6, 0.0]])
    save("ml_reflection", theta=sp._theta, mag=sp._mag, phase=sp._phase, sines=sines,
         r=sp._reflection(sines), fs=fs, clear_intensity=np.array([sp.clear_intensity(a, b) for a, b in fs]),
         blank_s_6deg=np.array(stack.blank_reflection(13.5e-9, np.radians(6.0), "s")),
         blank_p_9deg=np.array(stack.blank_reflection(13.5e-9, np.radians(9.0), "p")))


if __name__ == "__main__":
    if sys.argv[1:] == ["multilayer"]:
        multilayer()
    elif sys.argv[1:] == ["wide"]:
        wide()
    elif sys.argv[1:] == ["next"]:
        next_rows()
    elif sys.argv[1:] == ["volume"]:
        volume()
    else:
        main()
