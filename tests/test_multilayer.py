"""The EUV blank as a Bragg mirror (mask_model="multilayer"), on the CPU.

Pins the oracle's restatement of expose/m3d/provider.py:MultilayerSpectra and
the product's host side (the stack description, the reflection table, the
clear-field factors) against fixtures made by the reference itself.
"""

from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from conftest import load_golden, ns_grid, ns_optics
from oracle import litho_oracle as O


def _rel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / np.abs(b).max())


@pytest.mark.parametrize("name", ["ml_ls_128_cra6", "ml_ls_128_cram6", "ml_ls_128_thin", "ml_dipole_256"])
def test_oracle_images_match_reference(name):
    a, od, gd = load_golden(name)
    o, g = ns_optics(od), ns_grid(gd)
    raw, peak, clear = O.abbe_sum(a["mask"].astype(np.float64), o, g, [(o.defocus, o.image_index)])
    assert _rel(raw[0], a["raw"]) < 1e-12
    assert abs(clear[0] - float(a["clear"])) < 1e-12 * abs(float(a["clear"]))
    assert abs(peak[0] - float(a["peak"])) < 1e-12 * float(a["peak"])


def test_oracle_vector_wide_matches_reference():
    a, od, gd = load_golden("ml_vector_512")
    o, g = ns_optics(od), ns_grid(gd)
    raw, peak, clear = O.abbe_sum(a["mask"].astype(np.float64), o, g, [(o.defocus, o.image_index)])
    assert _rel(raw[0], a["raw"]) < 1e-6          # the fixture stores the image in float32
    assert abs(clear[0] - float(a["clear"])) < 1e-12 * abs(float(a["clear"]))


def test_the_mirror_changes_the_image_and_the_clear_field():
    """The blank is not a thin mask: the image moves and the clear field is ~0.75."""
    ml, _, _ = load_golden("ml_ls_128_cra6")
    thin, _, _ = load_golden("ml_ls_128_thin")
    assert _rel(ml["raw"], thin["raw"]) > 0.05
    assert 0.70 < float(ml["clear"]) / float(thin["clear"]) < 0.80


def test_reflection_table_matches_reference():
    from lithobat_b200 import multilayer as ML
    a, _, _ = load_golden("ml_reflection")
    t = ML.mirror_table(ML.MaskStack.for_wavelength(13.5e-9), 13.5e-9)
    assert np.array_equal(t.theta, a["theta"])
    assert np.abs(t.mag - a["mag"]).max() < 1e-12
    assert np.abs(t.phase - a["phase"]).max() < 1e-10
    r = t.reflection(a["sines"])
    assert np.abs(r - a["r"]).max() < 1e-12
    assert r[-1] == 0 and r[-2] == 0                 # evanescent orders carry nothing
    ot = O.mirror_table(ns_optics({"wavelength": 13.5e-9, "n_immersion": 1.0, "n_image": None}))
    assert np.abs(ot[1] - a["mag"]).max() < 1e-12 and np.abs(ot[2] - a["phase"]).max() < 1e-10


def test_blank_reflection_and_clear_factors_match_reference():
    from lithobat_b200 import multilayer as ML
    from lithobat_b200.config import optics_view
    from lithobat_b200 import OpticsConfig
    a, _, _ = load_golden("ml_reflection")
    st = ML.MaskStack.for_wavelength(13.5e-9)
    assert abs(st.blank_reflection(13.5e-9, np.radians(6.0), "s") - complex(a["blank_s_6deg"])) < 1e-13
    assert abs(st.blank_reflection(13.5e-9, np.radians(9.0), "p") - complex(a["blank_p_9deg"])) < 1e-13
    v = optics_view(OpticsConfig(wavelength=13.5e-9, NA=0.33, sigma_outer=0.6, source_grid=11,
                                 chief_ray_deg=6.0, normalisation="clear", mask_model="multilayer"))
    src = dataclasses.make_dataclass("S", ["fx", "fy"])(a["fs"][:, 0], a["fs"][:, 1])
    got = ML.clear_scales(v, src)
    assert np.abs(got - a["clear_intensity"]).max() < 1e-13
    assert 0.70 < got[0] < 0.80                      # an EUV blank reflects about 75 %


def test_stack_refusals_follow_the_reference():
    from lithobat_b200 import OpticsConfig
    from lithobat_b200 import multilayer as ML
    from lithobat_b200.config import optics_view
    duv = optics_view(OpticsConfig(wavelength=13.5e-9, NA=0.33, mask_model="multilayer",
                                   mask_stack={"regime": "duv_transmissive", "absorber": "Cr",
                                               "absorber_thickness": 70e-9, "multilayer": None,
                                               "substrate": "quartz"}))
    with pytest.raises(ValueError, match="describes the Bragg mirror"):
        ML.stack_for(duv)
    with pytest.raises(ValueError, match="needs a multilayer"):
        ML.MaskStack.from_spec({"regime": "euv_reflective", "absorber": "TaBN"})
    with pytest.raises(ValueError, match="gamma"):
        ML.Multilayer(gamma=1.2)
    with pytest.raises(KeyError, match="No mask-material table"):
        ML.mask_material("Si", 193.5e-9)
    with pytest.raises(ValueError, match="chief_ray_axis"):
        OpticsConfig(chief_ray_axis="z")
    # a DUV wavelength without a stack gets the transmissive default, which the mirror refuses
    from lithobat_b200.aerial import plan_abbe
    with pytest.raises(ValueError, match="describes the Bragg mirror"):
        plan_abbe([optics_view(OpticsConfig(mask_model="multilayer"))], 64, 4e-9, [[(0.0, 1.0)]], 1.0, True,
                  False)


def test_plan_carries_one_mirror_per_pupil():
    """The device plan holds LithoMirror[n_pupils] and the shared table."""
    from lithobat_b200 import OpticsConfig
    from lithobat_b200 import _native as nat
    from lithobat_b200.aerial import plan_abbe
    from lithobat_b200.config import optics_view
    thin = optics_view(OpticsConfig(wavelength=13.5e-9, NA=0.33, sigma_outer=0.6, source_grid=7))
    ml = optics_view(OpticsConfig(wavelength=13.5e-9, NA=0.33, sigma_outer=0.6, source_grid=7,
                                  chief_ray_deg=6.0, mask_model="multilayer"))
    pd = plan_abbe([thin, ml, ml], 128, 2e-9, [[(0.0, 1.0)]] * 3, 1.0, True, False)
    assert pd.plan.mirrored == 1
    seg = pd.blob[pd.plan.off_mirrors:]
    rows = np.frombuffer(seg[:3 * nat.MIRROR_DTYPE.itemsize].tobytes(), dtype=nat.MIRROR_DTYPE)
    assert rows["n_theta"].tolist() == [0, 501, 501]
    assert rows["off_table"][1] == rows["off_table"][2] > 0
    o = int(rows["off_table"][1])
    tab = np.frombuffer(seg[o:o + 3 * 501 * 8].tobytes(), dtype="<f8").reshape(3, 501)
    assert tab[0, -1] == pytest.approx(np.deg2rad(25.0))
    assert abs(rows["sin_cx"][1] - np.sin(np.radians(6.0))) < 1e-16 and rows["sin_cy"][1] == 0.0
    assert pd.clears[1] < pd.clears[0]              # the mirror returns less than a thin mask
    pd_thin = plan_abbe([thin], 128, 2e-9, [[(0.0, 1.0)]], 1.0, True, False)
    assert pd_thin.plan.mirrored == 0
