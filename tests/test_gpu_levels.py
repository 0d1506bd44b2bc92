"""Level-map masks (litho_abbe_levels: one byte per pixel indexing each
clip's complex levels) give the images of the complex masks they spell out.
Maps of more than two levels read the same complex values as the complex
path (bit-identical images); two-level maps transform the binary map as real
rows, two per complex transform, and add the constant level at DC, so they
agree with them to FP32 rounding (bound 5e-6 of the image maximum) and with
the FP64 oracle to the usual 1e-5."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 5e-6
TOL_FP64 = 1e-5


def rel(a, b):
    return float((a.double() - b.double()).abs().max() / b.double().abs().max())


@pytest.fixture(scope="module")
def lb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lithobat_b200
    return lithobat_b200


def _psm(lb, n, px, seed, count):
    rng = np.random.default_rng(seed)
    pats = []
    for _ in range(count):
        p = rng.uniform(80e-9, 140e-9)
        pats.append(1.0 - lb.patterns.contact_array(n, px, p, p, rng.uniform(40e-9, 70e-9)))
    return np.stack(pats)


@pytest.mark.parametrize("n,px,vector", [(256, 2e-9, False), (1024, 1e-9, True)])
def test_level_maps_equal_complex_masks(lb, n, px, vector):
    import torch
    from lithobat_b200 import aerial
    o = lb.OpticsConfig(NA=1.35, n_immersion=1.44, imaging_model="vector" if vector else "scalar", polarisation="te",
                        source_type="annular", sigma_inner=0.5, sigma_outer=0.9, source_grid=9)
    g = lb.GridConfig(n_pixels=n, pixel_size=px)
    pats = _psm(lb, n, px, 5, 6)
    idx, lv = lb.patterns.attenuated_psm_levels(pats)
    masks = lb.patterns.to_attenuated_psm(pats).astype(np.complex64)
    ref, rpk, _ = lb.compute_aerial_batch(torch.from_numpy(masks).cuda(), o, g)
    levels = lb.LevelMasks(idx, np.tile(lv, (len(pats), 1)))
    img, pk, _ = lb.compute_aerial_batch(levels, o, g)
    torch.cuda.synchronize()
    err = rel(img, ref)
    assert err <= TOL and rel(pk, rpk) <= TOL
    from oracle import litho_oracle as O
    r64, _pk64, _c = O.compute_aerial_image(masks[0].astype(np.complex128), o, g, return_raw=True)
    e64 = float(np.abs(img[0, 0].double().cpu().numpy() - r64 / r64.max()).max())
    print(f"PARITY level_map_{n} vs_complex {err:.3e} vs_fp64 {e64:.3e}")
    assert e64 <= TOL_FP64
    # the factoring helper gives the same levels (in another order) and images
    f = lb.LevelMasks.from_masks(masks)
    assert np.array_equal(f.expand(), masks)
    img2, _, _ = lb.compute_aerial_batch(f, o, g)
    assert rel(img2, ref) <= TOL
    # three levels (a third, unused value): the complex-valued path, bit-identical
    three = lb.LevelMasks(idx, np.concatenate([np.tile(lv, (len(pats), 1)), np.zeros((len(pats), 1), np.complex64)],
                                              axis=1))
    img3, _, _ = lb.compute_aerial_batch(three, o, g)
    assert torch.equal(img3, ref)
    # an index past the table takes the last level (no read outside it)
    v = lb.config.optics_view(o)
    pd = aerial.plan_abbe([v] * 6, n, px, [[(v.defocus, v.image_index)]] * 6, 1.0, False, True)
    bad = torch.from_numpy(idx).cuda().clone()
    bad[bad == 1] = 200
    im3, _ = aerial.run_abbe_levels(pd, bad, torch.from_numpy(np.tile(lv, (6, 1))).cuda())
    aerial.check_status(pd, bad.device)
    assert torch.equal(im3.view_as(img), img)


def test_pipeline_with_level_maps(lb):
    import torch
    from lithobat_b200.pipeline import AbbePipeline
    g = lb.GridConfig(n_pixels=128, pixel_size=2e-9)
    o = lb.OpticsConfig(NA=1.35, n_immersion=1.44, source_type="annular", sigma_inner=0.5, sigma_outer=0.9,
                        source_grid=9)
    batches, cbatches = [], []
    for b in range(4):
        pats = _psm(lb, 128, 2e-9, 10 + b, 3)
        idx, lv = lb.patterns.attenuated_psm_levels(pats)
        batches.append(torch.from_numpy(idx).pin_memory())
        cbatches.append(torch.from_numpy(lb.patterns.to_attenuated_psm(pats).astype(np.complex64)).pin_memory())
    levels = torch.from_numpy(np.tile(lv, (3, 1)))
    outs = [torch.empty((3, 128, 128), dtype=torch.float32).pin_memory() for _ in range(4)]
    couts = [torch.empty((3, 128, 128), dtype=torch.float32).pin_memory() for _ in range(4)]
    AbbePipeline(o, g, 3, mask_complex=True, level_masks=True).run(batches, outs, levels=levels)
    AbbePipeline(o, g, 3, mask_complex=True).run(cbatches, couts)
    for a, b in zip(outs, couts):
        assert rel(a, b) <= TOL
    with pytest.raises(ValueError):
        AbbePipeline(o, g, 3, mask_complex=True, level_masks=True).run(batches, outs)
