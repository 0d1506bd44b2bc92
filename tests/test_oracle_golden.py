"""Pin the CPU oracle against the reference's own outputs (tests/golden).

The oracle restates the reference in numpy; these tests show the restatement
reproduces the reference to FP64 rounding on every fixture, so that GPU
parity against the oracle is parity against the reference.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden, ns_grid, ns_optics
from oracle import litho_oracle as O

SOURCE_CASES = ["annular31", "annular31_imm", "conventional21", "dipole_legacy",
                "quadrupole_legacy", "cquad_spec", "euv_dipole43", "quasar_blur", "monopole"]


@pytest.mark.parametrize("name", SOURCE_CASES)
def test_source_points_bit_exact(name):
    a, od, _ = load_golden(f"source_{name}")
    sp = O.source_points(ns_optics(od))
    for k in ("weight", "fx", "fy", "phi"):
        np.testing.assert_array_equal(getattr(sp, k), a[k])


def test_pupil_functions():
    a, _, _ = load_golden("pupil_functions")
    rho, phi = a["rho"], a["phi"]
    Z = np.stack([O.zernike_noll(j, rho, phi) for j in range(1, 23)])
    np.testing.assert_allclose(Z, a["zernike"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(O.defocus_opd(rho, 193e-9, 1.35, 80e-9, 1.44, False),
                               a["defocus_paraxial"], rtol=1e-14, atol=0)
    np.testing.assert_allclose(O.defocus_opd(rho, 193e-9, 1.35, 80e-9, 1.44, True),
                               a["defocus_exact"], rtol=1e-14, atol=0)
    V = []
    for pol in ("x", "y", "te", "tm", "unpolarised"):
        for jx, jy, _w in O.jones_states(pol, 0.7):
            V.append(np.stack(O.vector_coefficients(rho, phi, jx, jy, 1.35 / 1.7, True)))
            V.append(np.stack(O.vector_coefficients(rho, phi, jx, jy, 1.35 / 1.7, False)))
    np.testing.assert_allclose(np.stack(V), a["vector"], rtol=0, atol=1e-14)


ABBE = ["abbe_conventional", "abbe_annular_aberrated", "abbe_dipole_exact_clear",
        "abbe_vector_te", "abbe_vector_tm", "abbe_vector_x", "abbe_vector_y",
        "abbe_vector_unpolarised", "c2_clip_128", "c3_vector_128", "euv_wide_256"]


@pytest.mark.parametrize("name", ABBE)
def test_abbe_raw_matches_reference(name):
    a, od, gd = load_golden(name)
    o, g = ns_optics(od), ns_grid(gd)
    mask = a["mask"].astype(np.complex64) if name == "c2_clip_128" else a["mask"]
    if mask.dtype == np.uint8:
        mask = mask.astype(np.float64)
    raw, peak, clear = O.compute_aerial_image(mask, o, g, return_raw=True)
    np.testing.assert_allclose(raw, a["raw"], rtol=0, atol=1e-12 * float(a["peak"]))
    assert peak == pytest.approx(float(a["peak"]), rel=1e-12)
    assert clear == pytest.approx(float(a["clear"]), rel=1e-12, abs=1e-300)
    if "image_dose13" in a:
        np.testing.assert_allclose(O.compute_aerial_image(mask, o, g, dose=1.3),
                                   a["image_dose13"], rtol=0, atol=1e-12)


def test_c1_full_size():
    a, od, gd = load_golden("c1_scalar_256")
    o, g = ns_optics(od), ns_grid(gd)
    mask = O.lines_and_spaces(256, 4e-9, 200e-9, 100e-9)
    raw, peak, clear = O.compute_aerial_image(mask, o, g, return_raw=True)
    np.testing.assert_allclose(raw, a["raw"], rtol=0, atol=1e-12 * peak)
    np.testing.assert_allclose(O.compute_aerial_image(mask, o, g), a["image"], atol=1e-12)


@pytest.mark.parametrize("name", ["planes_scalar", "planes_vector"])
def test_planes(name):
    a, od, gd = load_golden(name)
    o, g = ns_optics(od), ns_grid(gd)
    planes = [tuple(p) for p in a["planes"]]
    dose = 1.3 if name == "planes_scalar" else 1.0
    st = O.compute_aerial_planes(a["mask"], o, g, planes, dose=dose)
    np.testing.assert_allclose(st, a["stack"], rtol=0, atol=1e-12 * a["stack"].max())


@pytest.mark.parametrize("name", ["conventional", "annular_aberrated", "dipole_exact_clear"])
def test_socs_build_and_raw(name):
    a, od, gd = load_golden(f"socs_{name}")
    o, g = ns_optics(od), ns_grid(gd)
    full = O.socs_build(o, g, tol=0.0)
    tr = O.socs_build(o, g)
    cap = O.socs_build(o, g, max_kernels=3)
    np.testing.assert_allclose(full.weights, a["weights_full"], rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(tr.weights, a["weights_tol"], rtol=1e-10)
    np.testing.assert_allclose(cap.weights, a["weights_cap3"], rtol=1e-12)
    assert full.n_band == int(a["n_band"]) and full.n_source == int(a["n_source"])
    rf = O.socs_raw(full, a["mask"])[0]
    np.testing.assert_allclose(rf, a["raw_full"], rtol=0, atol=1e-12 * rf.max())
    np.testing.assert_allclose(O.socs_raw(tr, a["mask"])[0], a["raw_tol"], atol=1e-12 * rf.max())
    np.testing.assert_allclose(O.socs_image(tr, a["mask"], 0.8), a["image_tol"], atol=1e-12)


def test_socs_mid_size_k24():
    a, od, gd = load_golden("socs_imm_128_k24")
    k = O.socs_build(ns_optics(od), ns_grid(gd), tol=0.0, max_kernels=24)
    np.testing.assert_allclose(k.weights, a["weights"], rtol=1e-10)
    assert k.clear == pytest.approx(float(a["clear"]), rel=1e-10)
    raw = O.socs_raw(k, a["mask"].astype(np.float64))[0]
    np.testing.assert_allclose(raw, a["raw"], rtol=0, atol=1e-11 * raw.max())


def test_ilt_small():
    a, od, gd = load_golden("ilt_small")
    k = O.socs_build(ns_optics(od), ns_grid(gd), tol=1e-6)
    np.testing.assert_allclose(k.weights, a["weights"], rtol=1e-10)
    fields, inten = O.socs_fields(k, a["mask"])
    np.testing.assert_allclose(inten, a["intensity"], atol=1e-12)
    g = O.socs_gradient(k, fields, a["sens"])
    np.testing.assert_allclose(g, a["grad"], rtol=0, atol=1e-11 * np.abs(a["grad"]).max())
    cost, gr, signed, perr = O.objective(k, a["target3"], a["mask3"], 1.7, 0.3, 1.5, 1.0,
                                         12.0, 1e-3, 1e-3)
    assert cost == pytest.approx(float(a["cost"]), rel=1e-12)
    np.testing.assert_allclose(gr, a["grad_obj"], atol=1e-11 * np.abs(gr).max())
    np.testing.assert_allclose(signed, a["signed"], atol=1e-12)
    assert perr == int(a["perr"])
    cost0, gr0, signed0, perr0 = O.objective(k, a["target3"], a["mask3"], 2.0, 0.3, 0.0, -1.0,
                                             20.0)
    assert cost0 == pytest.approx(float(a["cost0"]), rel=1e-12)
    np.testing.assert_allclose(gr0, a["grad_obj0"], atol=1e-11 * np.abs(gr0).max())
    assert perr0 == int(a["perr0"])
    m = O.mask_of(a["theta"], 6.0, 2.0)
    np.testing.assert_allclose(m, a["mask_of"], atol=1e-15)
    np.testing.assert_allclose(O.grad_theta(a["grad_obj"], m, 6.0, 2.0), a["grad_theta"],
                               atol=1e-12 * np.abs(a["grad_theta"]).max())


def test_ilt_mid_size_objective():
    a, od, gd = load_golden("ilt_imm_128_k24")
    s, _, _ = load_golden("socs_imm_128_k24")
    k = O.socs_build(ns_optics(od), ns_grid(gd), tol=0.0, max_kernels=24)
    m = O.mask_of(a["theta"], float(a["beta"]), 0.0)
    cost, g, signed, perr = O.objective(k, a["target"].astype(np.float64), m, 1.0 / k.clear,
                                        0.3, 0.0, 1.0, 15.0)
    assert cost == pytest.approx(float(a["cost"]), rel=1e-10)
    np.testing.assert_allclose(g, a["grad"], rtol=0, atol=1e-9 * np.abs(a["grad"]).max())
    assert perr == int(a["perr"])


def test_peb_matches_reference():
    a = load_golden("peb_small")[0]
    np.testing.assert_allclose(O.apply_peb(a["pac"], 7e-9, 4e-9), a["out"], rtol=0, atol=1e-14)
    np.testing.assert_array_equal(O.apply_peb(a["pac"], 0.0, 4e-9), a["out0"])
    with pytest.raises(ValueError):
        O.apply_peb(a["pac"][None], 7e-9, 4e-9)
    with pytest.raises(ValueError):
        O.apply_peb(a["pac"], -1e-9, 4e-9)


def test_dose_focus_images_match_reference():
    a, od, gd = load_golden("dose_focus_64")
    o, g = ns_optics(od), ns_grid(gd)
    st = O.dose_focus_images(a["mask"].astype(np.float64), o, g, list(a["doses"]), list(a["defoci"]),
                             normalisation=None)
    np.testing.assert_allclose(st, a["stack"], rtol=0, atol=1e-12 * float(np.abs(a["stack"]).max()))


def _volume_case(name):
    from types import SimpleNamespace
    a, od, gd = load_golden(name)
    o = ns_optics(od)
    g = SimpleNamespace(**gd, dz=float(a["dz"]), n_z_slices=int(a["n_z_slices"]))
    r = SimpleNamespace(thickness=float(a["thickness"]), n_resist=float(a["n_resist"]),
                        focus_reference=str(a["focus_reference"]))
    return a, o, g, r


@pytest.mark.parametrize("name", ["volume_scalar_64", "volume_vector_64"])
def test_exposure_volume_matches_reference(name):
    a, o, g, r = _volume_case(name)
    vol, z = O.exposure_volume(a["mask"].astype(np.float64), o, g, r, dose=float(a["dose"]))
    np.testing.assert_array_equal(z, a["z"])
    np.testing.assert_allclose(vol, a["volume"], rtol=0, atol=1e-12 * float(np.abs(a["volume"]).max()))
