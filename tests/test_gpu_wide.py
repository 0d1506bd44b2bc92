"""Wide pupils (coarse grids of 128 points and more): EUV clips at 256^2-512^2.

The band-limited engine moves the two passes of each coherent transform to
thread blocks once 4h + 1 > 64 (csrc/wide.cu). Same bar as everywhere:
max |I_gpu - I_ref| / max I_ref <= 1e-5 against the reference's fixtures and
the FP64 oracle.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden
from oracle import litho_oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.fixture(scope="module")
def lb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lithobat_b200
    return lithobat_b200


def _optics(lb, od):
    od = dict(od)
    od["zernike_coeffs"] = {int(k): v for k, v in (od.get("zernike_coeffs") or {}).items()}
    keep = {k: od[k] for k in lb.OpticsConfig.__dataclass_fields__ if k in od}
    return lb.OpticsConfig(**keep)


def rel_err(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / np.abs(b).max())


def _plan_L(lb, o, g):
    from lithobat_b200 import aerial
    v = lb.config.optics_view(o)
    pd = aerial.plan_abbe([v], g.n_pixels, g.pixel_size, [[(v.defocus, v.image_index)]], 1.0, True, False)
    return int(pd.plan.L)


def test_wide_euv_matches_reference(lb):
    a, od, gd = load_golden("euv_wide_256")
    o, g = _optics(lb, od), lb.GridConfig(**gd)
    assert _plan_L(lb, o, g) == 128
    raw, peak, clear = lb.compute_aerial_image(a["mask"].astype(np.float64), o, g, return_raw=True)
    assert rel_err(raw, a["raw"]) <= TOL
    assert peak == pytest.approx(float(a["peak"]), rel=TOL)
    assert clear == pytest.approx(float(a["clear"]), rel=1e-12)
    img = lb.compute_aerial_image(a["mask"].astype(np.float64), o, g, dose=0.9)
    assert rel_err(img, a["raw"] * (0.9 / float(a["peak"]))) <= TOL


def test_wide_vector_high_na_against_oracle(lb):
    """High-NA EUV, vector TE, att-PSM contacts: pupil radius 20.9 bins."""
    g = lb.GridConfig(n_pixels=256, pixel_size=2e-9)
    c = lb.patterns.contact_array(256, 2e-9, 40e-9, 40e-9, 18e-9)
    mask = lb.patterns.to_attenuated_psm(1.0 - c, 0.06, 180.0)
    o = lb.OpticsConfig(wavelength=13.5e-9, NA=0.55, imaging_model="vector", polarisation="te",
                        source_type="annular", sigma_inner=0.3, sigma_outer=0.8, source_grid=9,
                        zernike_coeffs={7: 0.01}, normalisation="clear")
    assert _plan_L(lb, o, g) == 128
    raw, peak, clear = lb.compute_aerial_image(mask, o, g, return_raw=True)
    ref = O.compute_aerial_image(mask, o, g, return_raw=True)
    assert rel_err(raw, ref[0]) <= TOL
    assert clear == pytest.approx(ref[2], rel=1e-12)
    img = lb.compute_aerial_image(mask, o, g, dose=1.1)
    assert rel_err(img, O.compute_aerial_image(mask, o, g, dose=1.1)) <= TOL


def test_wide_planes_512_against_oracle(lb):
    """512^2 at 2 nm, EUV dipole: radius 25 bins, two focus planes."""
    from lithobat_b200.patterns import lines_and_spaces
    g = lb.GridConfig(n_pixels=512, pixel_size=2e-9)
    mask = lines_and_spaces(512, 2e-9, 64e-9, 32e-9)
    o = lb.OpticsConfig(wavelength=13.5e-9, NA=0.33, source_type="dipole", sigma_outer=0.9, sigma_inner=0.6,
                        source_grid=11, source_kwargs={"axis": "x"})
    assert _plan_L(lb, o, g) == 128
    planes = [(0.0, 1.0), (40e-9, 1.0)]
    st = lb.compute_aerial_planes(mask, o, g, planes, dose=1.2)
    ref = O.compute_aerial_planes(mask, o, g, planes, dose=1.2)
    for p in range(len(planes)):
        assert rel_err(st[p], ref[p]) <= TOL


def test_wide_fused_and_plain_agree(lb):
    import torch
    from lithobat_b200 import aerial
    g = lb.GridConfig(n_pixels=512, pixel_size=2e-9)
    rng = np.random.default_rng(4)
    masks = torch.from_numpy((rng.random((3, 512, 512)) > 0.6).astype(np.float32)).cuda()
    o = lb.OpticsConfig(wavelength=13.5e-9, NA=0.33, source_type="annular", sigma_inner=0.4,
                        sigma_outer=0.8, source_grid=9)
    v = lb.config.optics_view(o)
    pd = aerial.plan_abbe([v] * 3, 512, 2e-9, [[(v.defocus, v.image_index)]] * 3, 1.0, True, False)
    a, pa = aerial.run_abbe(pd, masks)
    a = a.clone()
    b, pb = aerial.run_abbe(pd, masks, engine="plain")
    d = (a.double() - b.double()).abs().amax(dim=(1, 2)) / b.double().abs().amax(dim=(1, 2))
    assert float(d.max()) <= TOL
    assert torch.allclose(pa, pb, rtol=1e-5)


def test_wide_socs_matches_reference(lb):
    """SOCS kernels with a 31-bin band (128-point coarse grid), 24 kernels."""
    a, od, gd = load_golden("socs_euv_wide_128_k24")
    o, g = _optics(lb, od), lb.GridConfig(**gd)
    k = lb.SOCSKernels.build(o, g, tol=0.0, max_kernels=24)
    assert k.halfwidth > 15 and k.n_band == int(a["n_band"])
    # the source has fewer points than 24: the Gram route returns its rank,
    # the reference's eigh also returns round-off eigenvalues past it
    K = len(k)
    assert K == min(24, k.n_source)
    np.testing.assert_allclose(k.weights, a["weights"][:K], rtol=1e-6, atol=1e-9 * float(a["weights"][0]))
    assert np.all(np.abs(a["weights"][K:]) < 1e-10 * float(a["weights"][0]))
    raw, peak, clear = k.raw(a["mask"].astype(np.float64))
    assert rel_err(raw, a["raw"]) <= TOL
    assert clear == pytest.approx(float(a["clear"]), rel=1e-6)


def test_wide_socs_all_kernels_equal_abbe(lb):
    """Every kernel kept: SOCS is the Abbe sum (test_hopkins.py:104-118)."""
    g = lb.GridConfig(n_pixels=128, pixel_size=5e-9)
    o = lb.OpticsConfig(wavelength=13.5e-9, NA=0.33, source_type="annular", sigma_inner=0.5, sigma_outer=0.8,
                        source_grid=9)
    mask = (np.random.default_rng(8).random((128, 128)) > 0.5).astype(np.float64)
    k = lb.SOCSKernels.build(o, g, tol=0.0)
    raw_s = k.raw(mask)[0]
    raw_a = lb.compute_aerial_image(mask, o, g, return_raw=True)[0]
    assert rel_err(raw_s, raw_a) <= TOL
