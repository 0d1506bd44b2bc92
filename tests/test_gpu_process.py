"""Process-window helpers on the GPU: dose-focus images and the threshold
print model, against the reference's fixtures and the oracle (1e-5 bar;
PEB to 1e-6 absolute on maps in [0, 1])."""

from __future__ import annotations

from types import SimpleNamespace

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


def test_dose_focus_images_match_reference(lb):
    from lithobat_b200.process import dose_focus_images
    a, od, gd = load_golden("dose_focus_64")
    st = dose_focus_images(a["mask"].astype(np.float64), _optics(lb, od), lb.GridConfig(**gd),
                           list(a["doses"]), list(a["defoci"]), normalisation=None)
    assert st.shape == a["stack"].shape
    assert float(np.abs(st - a["stack"]).max() / np.abs(a["stack"]).max()) <= TOL


def test_dose_focus_peak_mode_against_oracle(lb):
    from lithobat_b200.process import dose_focus_images
    g = lb.GridConfig(n_pixels=256, pixel_size=2e-9)
    o = lb.OpticsConfig(NA=1.35, n_immersion=1.44, source_type="annular", sigma_inner=0.5, sigma_outer=0.9,
                        source_grid=9)
    mask = lb.patterns.lines_and_spaces(256, 2e-9, 80e-9, 40e-9)
    st = dose_focus_images(mask, o, g, [0.9, 1.1], [-40.0, 0.0, 40.0], normalisation="peak")
    ref = O.dose_focus_images(mask, o, g, [0.9, 1.1], [-40.0, 0.0, 40.0], normalisation="peak")
    assert float(np.abs(st - ref).max() / np.abs(ref).max()) <= TOL


def test_peb_matches_reference(lb):
    from lithobat_b200.process import apply_peb
    a = load_golden("peb_small")[0]
    np.testing.assert_allclose(apply_peb(a["pac"], 7e-9, 4e-9), a["out"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(apply_peb(a["pac"], 0.0, 4e-9), a["out0"], rtol=0, atol=1e-7)
    with pytest.raises(ValueError):
        apply_peb(a["pac"], -1e-9, 4e-9)


def test_print_image_threshold_model(lb):
    """SOCS ("auto") and Abbe prints of one clip agree, and the developed field
    is the oracle's PEB of the oracle's aerial image."""
    from lithobat_b200.process import print_image
    g = lb.GridConfig(n_pixels=128, pixel_size=4e-9)
    o = lb.OpticsConfig(NA=0.93, source_type="annular", sigma_inner=0.5, sigma_outer=0.8, source_grid=11)
    rng = np.random.default_rng(5)
    from lithobat_b200.patterns import manhattan_clip
    mask = manhattan_clip(rng, 128, 4e-9, n_rect=(6, 12), width_nm=(40, 160))
    resist = SimpleNamespace(diffusion_sigma=10e-9, threshold=0.3)
    a_abbe, f_abbe, lvl = print_image(mask, o, g, resist, dose=1.1, imaging="abbe")
    a_socs, f_socs, _ = print_image(mask, o, g, resist, dose=1.1, imaging="auto", socs_tol=0.0)
    assert lvl == 0.3
    import dataclasses
    ref_aerial = O.compute_aerial_image(mask, dataclasses.replace(o, normalisation="clear"), g, dose=1.1)
    assert float(np.abs(a_abbe - ref_aerial).max() / np.abs(ref_aerial).max()) <= TOL
    assert float(np.abs(a_socs - a_abbe).max() / np.abs(a_abbe).max()) <= TOL
    np.testing.assert_allclose(f_abbe, O.apply_peb(ref_aerial, 10e-9, 4e-9), rtol=0, atol=1e-5)


def _volume_inputs(lb, name):
    a, od, gd = load_golden(name)
    g = lb.GridConfig(**gd, dz=float(a["dz"]), n_z_slices=int(a["n_z_slices"]))
    r = lb.config.ResistConfig(thickness=float(a["thickness"]), n_resist=float(a["n_resist"]),
                               focus_reference=str(a["focus_reference"]))
    return a, _optics(lb, od), g, r


@pytest.mark.parametrize("name", ["volume_scalar_64", "volume_vector_64"])
def test_exposure_volume_matches_reference(lb, name):
    from lithobat_b200.process import exposure_volume
    a, o, g, r = _volume_inputs(lb, name)
    vol, z = exposure_volume(a["mask"].astype(np.float64), o, g, r, dose=float(a["dose"]))
    assert vol.shape == a["volume"].shape and vol.dtype == np.float64
    np.testing.assert_array_equal(z, a["z"])
    assert float(np.abs(vol - a["volume"]).max() / np.abs(a["volume"]).max()) <= TOL


def test_exposure_volume_512_against_oracle(lb):
    """A 512² clip through a 100 nm film at 2 nm voxels (50 voxel planes from
    21 optical planes, the reference's defaults), on a device mask: float32
    CUDA result against the oracle's FP64 volume."""
    import torch
    from lithobat_b200.process import exposure_volume
    g = lb.GridConfig(n_pixels=512, pixel_size=2e-9)
    o = lb.OpticsConfig(NA=1.35, n_immersion=1.44, source_type="annular", sigma_inner=0.5, sigma_outer=0.9,
                        source_grid=9, defocus=25e-9)
    r = lb.config.ResistConfig()
    mask = lb.patterns.lines_and_spaces(512, 2e-9, 90e-9, 45e-9)
    vol, z = exposure_volume(torch.from_numpy(mask).cuda(), o, g, r, check=True)
    assert vol.is_cuda and vol.dtype == torch.float32 and tuple(vol.shape) == (50, 512, 512)
    ref, zr = O.exposure_volume(mask, o, g, r)
    np.testing.assert_array_equal(z, zr)
    got = vol.cpu().numpy().astype(np.float64)
    assert float(np.abs(got - ref).max() / np.abs(ref).max()) <= TOL
