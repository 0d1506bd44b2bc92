"""mask_model="multilayer" on the GPU: the blank's reflection folded into the
pupil table, through every engine (coarse 32/64, wide, plain).

Bar: max |I_gpu - I_ref| / max I_ref <= 1e-5 against the reference's own
images (tests/golden/ml_*.npz), plus the physical properties the reference's
tests pin (tests/test_m3d.py:258-346): best focus moves, the placement shift
follows the chief ray, an unpatterned blank images flat at ~75 %.
"""

from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from conftest import load_golden

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


def _grid(lb, gd):
    return lb.GridConfig(n_pixels=gd["n_pixels"], pixel_size=gd["pixel_size"])


def rel_err(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / np.abs(b).max())


@pytest.mark.parametrize("name", ["ml_ls_128_cra6", "ml_ls_128_cram6", "ml_dipole_256", "ml_vector_512"])
def test_multilayer_images_match_reference(lb, name):
    a, od, gd = load_golden(name)
    o, g = _optics(lb, od), _grid(lb, gd)
    raw, peak, clear = lb.compute_aerial_image(a["mask"].astype(np.float64), o, g, return_raw=True)
    assert rel_err(raw, a["raw"]) <= TOL
    assert abs(clear - float(a["clear"])) <= 1e-9 * abs(float(a["clear"]))
    assert abs(peak - float(a["peak"])) <= TOL * float(a["peak"])


@pytest.mark.parametrize("name", ["ml_ls_128_cra6", "ml_dipole_256"])
def test_plain_engine_carries_the_mirror(lb, name):
    a, od, gd = load_golden(name)
    o, g = _optics(lb, od), _grid(lb, gd)
    img, peak, clear = lb.compute_aerial_batch(a["mask"], o, g, return_raw=True, engine="plain")
    assert rel_err(img[0, 0].cpu().numpy(), a["raw"]) <= TOL
    assert abs(float(clear[0, 0]) - float(a["clear"])) <= 1e-9 * abs(float(a["clear"]))


def test_thin_fixture_unchanged(lb):
    a, od, gd = load_golden("ml_ls_128_thin")
    raw, _, clear = lb.compute_aerial_image(a["mask"].astype(np.float64), _optics(lb, od), _grid(lb, gd),
                                            return_raw=True)
    assert rel_err(raw, a["raw"]) <= TOL
    assert abs(clear - float(a["clear"])) <= 1e-12 * float(a["clear"])


def test_focus_stack_and_best_focus_shift(lb):
    """Planes of one launch match the reference's images; the mirror moves
    best focus by about -7 nm and the thin mask does not (test_m3d.py:258-278)."""
    a, od, gd = load_golden("ml_ls_128_focus")
    o, g = _optics(lb, od), _grid(lb, gd)
    m = a["mask"].astype(np.float64)
    got = lb.compute_aerial_planes(m, o, g, [(float(d), 1.0) for d in a["foci"]])
    assert rel_err(np.asarray(got), a["images"]) <= TOL

    def best_focus(model):
        foci = np.linspace(-40e-9, 40e-9, 41)
        oo = dataclasses.replace(o, mask_model=model)
        imgs = np.asarray(lb.compute_aerial_planes(m, oo, g, [(float(d), 1.0) for d in foci]), np.float64)
        c = (imgs.max(axis=(1, 2)) - imgs.min(axis=(1, 2))) / (imgs.max(axis=(1, 2)) + imgs.min(axis=(1, 2)))
        k = int(np.clip(c.argmax(), 1, 39))
        den = c[k - 1] - 2 * c[k] + c[k + 1]
        sh = 0.0 if den == 0 else (c[k - 1] - c[k + 1]) / (2 * den)
        return float((foci[k] + sh * (foci[1] - foci[0])) * 1e9)

    assert abs(best_focus("thin")) < 1.0
    bf = best_focus("multilayer")
    assert bf < -3.0 and abs(bf + 7.0) < 4.0


def test_placement_shift_follows_the_chief_ray(lb):
    a, od, gd = load_golden("ml_ls_128_cra6")
    o, g = _optics(lb, od), _grid(lb, gd)
    m = a["mask"].astype(np.float64)

    def centre(img):
        row = np.asarray(img, np.float64)[img.shape[0] // 2]
        k = int(np.argmax(row))
        idx = np.arange(k - 6, k + 7)
        v = row[idx % len(row)]
        x = idx * g.pixel_size * 1e9
        return float((x * v).sum() / v.sum())

    ref = centre(lb.compute_aerial_image(m, dataclasses.replace(o, mask_model="thin"), g))
    plus = centre(lb.compute_aerial_image(m, o, g)) - ref
    minus = centre(lb.compute_aerial_image(m, dataclasses.replace(o, chief_ray_deg=-6.0), g)) - ref
    assert abs(plus) > 1.0 and plus * minus < 0.0 and abs(plus + minus) < 0.4 * abs(plus)


def test_unpatterned_blank_images_flat(lb):
    a, od, gd = load_golden("ml_reflection")
    _, od2, gd2 = load_golden("ml_ls_128_cra6")
    o, g = _optics(lb, od2), _grid(lb, gd2)
    raw, _, clear = lb.compute_aerial_image(np.ones((128, 128)), o, g, return_raw=True)
    raw = np.asarray(raw, np.float64)
    assert raw.std() <= 1e-6 * raw.mean()
    # the on-axis DC of a clear mask, normalised by the clear field, is 1
    assert abs(raw.mean() / clear - 1.0) < 1e-5
    thin = lb.compute_aerial_image(np.ones((128, 128)), dataclasses.replace(o, mask_model="thin"), g,
                                   return_raw=True)[2]
    assert 0.70 < clear / thin < 0.80


def test_uneven_batch_with_the_mirror(lb):
    """Mixed sizes of mirrored clips through the grouped, graph-captured path."""
    import torch
    from lithobat_b200.uneven import compute_aerial_uneven
    _, od, _ = load_golden("ml_dipole_256")
    o = _optics(lb, od)
    rng = np.random.default_rng(5)
    masks = [torch.from_numpy((rng.random((n, n)) > 0.6).astype(np.float32)).cuda() for n in (256, 128, 256)]
    got = compute_aerial_uneven(masks, o, 2e-9)
    for mk, img in zip(masks, got):
        n = mk.shape[-1]
        one = lb.compute_aerial_image(mk, o, lb.GridConfig(n_pixels=n, pixel_size=2e-9))
        assert rel_err(img.cpu().numpy(), one.cpu().numpy().astype(np.float64)) <= 1e-6
