"""Host-side logic of the product package, checked without a GPU."""

from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import load_golden
from lithobat_b200 import GridConfig, OpticsConfig, normalisation_scale, source_points
from lithobat_b200.aerial import disc_halfwidth, plan_abbe
from lithobat_b200.config import optics_view
from lithobat_b200.pupil import clear_throughput
from lithobat_b200.source import Source

SOURCE_CASES = ["annular31", "annular31_imm", "conventional21", "dipole_legacy",
                "quadrupole_legacy", "cquad_spec", "euv_dipole43", "quasar_blur", "monopole"]


def _optics(od):
    od = dict(od)
    od["zernike_coeffs"] = {int(k): v for k, v in (od.get("zernike_coeffs") or {}).items()}
    keep = {k: od[k] for k in OpticsConfig.__dataclass_fields__ if k in od}
    return OpticsConfig(**keep)


@pytest.mark.parametrize("name", SOURCE_CASES)
def test_source_points_are_bit_identical_to_the_reference(name):
    a, od, _ = load_golden(f"source_{name}")
    sp = source_points(_optics(od))
    for k in ("weight", "fx", "fy", "phi"):
        np.testing.assert_array_equal(getattr(sp, k), a[k])


ABBE = ["abbe_conventional", "abbe_annular_aberrated", "abbe_dipole_exact_clear",
        "abbe_vector_te", "abbe_vector_tm", "abbe_vector_x", "abbe_vector_y",
        "abbe_vector_unpolarised", "c2_clip_128", "c3_vector_128", "c1_scalar_256"]


@pytest.mark.parametrize("name", ABBE)
def test_clear_throughput_matches_the_reference(name):
    a, od, gd = load_golden(name)
    o = _optics(od)
    v = optics_view(o)
    got = clear_throughput(source_points(o), v, v.image_index, v.imaging_model == "vector")
    assert got == pytest.approx(float(a["clear"]), rel=1e-12, abs=1e-300)


def test_normalisation_scale_modes():
    assert normalisation_scale("peak", 2.0, 5.0, 1.5) == 0.75
    assert normalisation_scale("clear", 2.0, 5.0, 1.5) == 0.3
    assert normalisation_scale("none", 2.0, 5.0, 1.5) == 1.5
    assert normalisation_scale("PEAK", 0.0, 5.0, 1.5) == 1.5
    with pytest.raises(ValueError, match="normalisation must be"):
        normalisation_scale("max", 1, 1)


@pytest.mark.parametrize("NA,lam,n,px", [(0.93, 193e-9, 256, 4e-9), (1.35, 193e-9, 1024, 1e-9),
                                         (1.35, 193e-9, 512, 2e-9), (0.33, 13.5e-9, 256, 2e-9),
                                         (1.35, 193e-9, 64, 4e-9)])
def test_every_in_aperture_bin_lies_in_the_coarse_box(NA, lam, n, px):
    """The box [c - h, c + h]^2 around a source point's nearest bin must hold
    every bin the reference's exact aperture test admits."""
    R, h = disc_halfwidth(NA, lam, n, px)
    val = 1.0 / (n * px)
    k_max = NA / lam
    rng = np.random.default_rng(0)
    fs = rng.uniform(-1, 1, size=(400, 2)) * k_max
    k = np.arange(-(n // 2), (n - 1) // 2 + 1)
    for fsx, fsy in fs:
        cx, cy = int(np.rint(fsx / val)), int(np.rint(fsy / val))
        sel = np.abs(k * val - fsx) <= 1.01 * k_max
        kx = k[sel]
        sel = np.abs(k * val - fsy) <= 1.01 * k_max
        ky = k[sel]
        KX, KY = np.meshgrid(kx, ky)
        rho = np.sqrt((KX * val - fsx) ** 2 + (KY * val - fsy) ** 2) / k_max
        inside = rho <= 1.0
        assert np.all(np.abs(KX[inside] - cx) <= h) and np.all(np.abs(KY[inside] - cy) <= h)


def test_plan_groups_jobs_by_output_and_counts_transforms():
    o = OpticsConfig(NA=1.35, n_immersion=1.44, imaging_model="vector", polarisation="unpolarised",
                     source_type="annular", sigma_outer=0.9, sigma_inner=0.5, source_grid=9)
    v = optics_view(o)
    pd = plan_abbe([v, v], 64, 4e-9, [[(0.0, 1.44), (50e-9, 1.7)]] * 2, 1.0, False, False)
    S = len(source_points(o))
    assert pd.n_out == 4 and pd.jobs == 4 * S * 2 and pd.transforms == 3 * pd.jobs
    assert pd.plan.ncomp_max == 3 and 4 * pd.plan.h + 1 <= pd.plan.L
    assert pd.plan.bm >= pd.plan.h
    # two clips with the same optics share the pupil-table slots of each plane
    assert pd.plan.n_tab == 2 * S * 2


def test_thick_masks_and_bad_models_are_refused():
    with pytest.raises(ValueError, match="thin"):
        plan_abbe([optics_view(OpticsConfig(mask_model="fdtd"))], 64, 4e-9, [[(0.0, 1.0)]], 1.0, False, False)
    with pytest.raises(ValueError, match="imaging_model"):
        OpticsConfig(imaging_model="quantum")


def test_source_presets_round_trip_through_dicts():
    s = Source.quadrupole(0.9, 0.7, opening_deg=30, rotation_deg=0)
    d = s.to_dict()
    assert Source.from_dict(d).render(21).tolist() == s.render(21).tolist()
    assert s.n_points(21) == 34


def test_level_masks_factor_and_expand():
    """LevelMasks.from_masks: per-clip distinct values and a uint8 index
    that spell out the masks exactly; too many levels or bad shapes refused."""
    import numpy as np
    import pytest
    import lithobat_b200 as lb
    rng = np.random.default_rng(3)
    pats = (rng.random((3, 32, 32)) > 0.5).astype(np.float64)
    m = lb.patterns.to_attenuated_psm(pats)
    f = lb.LevelMasks.from_masks(m)
    assert f.index.dtype == np.uint8 and f.levels.shape == (3, 2)
    assert np.array_equal(f.expand(), m.astype(np.complex64))
    idx, lv = lb.patterns.attenuated_psm_levels(pats)
    assert np.array_equal(lv[idx], m.astype(np.complex64))
    with pytest.raises(ValueError):
        lb.LevelMasks.from_masks(rng.random((1, 32, 32)), max_levels=16)
    with pytest.raises(ValueError):
        lb.LevelMasks(idx[0], lv[None])


def test_depth_intervals_follow_np_interp():
    """The host-side interval and weight of every voxel plane reproduce
    np.interp (develop/resist3d.py:176-183), ends and interior nodes included."""
    from lithobat_b200.process import depth_intervals
    rng = np.random.default_rng(3)
    for n_slices in (1, 2, 5, 21):
        depths = np.linspace(0.0, 80e-9, n_slices)
        z = np.concatenate([rng.uniform(-10e-9, 90e-9, 40), depths, [0.0, 80e-9]])
        k, w = depth_intervals(z, depths)
        f = rng.standard_normal((n_slices, 7))
        got = f[k[:, 0]] + w[:, None] * (f[k[:, 1]] - f[k[:, 0]])
        want = np.stack([np.interp(z, depths, f[:, j]) for j in range(7)], axis=1)
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)
        assert k.min() >= 0 and k.max() <= n_slices - 1


def test_focus_reference_and_effective_defocus():
    from types import SimpleNamespace

    from lithobat_b200.config import ResistConfig
    from lithobat_b200.process import effective_defocus, focus_reference_depth
    o = SimpleNamespace(defocus=10e-9, n_immersion=1.44)
    for ref, d_ref in (("top", 0.0), ("mid", 50e-9), ("bottom", 100e-9)):
        r = ResistConfig(thickness=100e-9, n_resist=1.7, focus_reference=ref)
        assert focus_reference_depth(r) == d_ref
        assert effective_defocus(30e-9, o, r) == 10e-9 - (30e-9 - d_ref) * (1.44 / 1.7)
    with pytest.raises(ValueError, match="focus_reference must be 'top', 'mid', or 'bottom'"):
        focus_reference_depth(SimpleNamespace(focus_reference="centre", thickness=1e-7))
    with pytest.raises(ValueError, match="ResistConfig.focus_reference"):
        ResistConfig(focus_reference="centre")
    with pytest.raises(ValueError, match="ResistConfig.threshold"):
        ResistConfig(threshold=1.0)
    with pytest.raises(ValueError, match="GridConfig.n_z_slices"):
        GridConfig(n_z_slices=0)
