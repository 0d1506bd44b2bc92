"""Uneven batches (clips of mixed sizes in one CUDA-graph replay) against
one-clip-at-a-time imaging; same 1e-5 bar."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.fixture(scope="module")
def lb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lithobat_b200
    return lithobat_b200


def _euv(lb):
    from lithobat_b200.source import Source
    return lb.OpticsConfig(wavelength=13.5e-9, NA=0.33, source_grid=21,
                           source_spec=Source.dipole(0.9, 0.6, opening_deg=60).to_dict())


def _clips(seed, sizes):
    from lithobat_b200.patterns import manhattan_clip
    rng = np.random.default_rng(seed)
    return [manhattan_clip(rng, n, 2e-9, n_rect=(6, 16), width_nm=(20, 80)).astype(np.float32) for n in sizes]


def test_uneven_batch_matches_one_clip_at_a_time(lb):
    """128^2 (32-point coarse grid), 256^2 (64), 512^2 (wide, 128) in one
    replay; two batches in a row through the same graph."""
    import torch
    from lithobat_b200.uneven import UnevenAbbe
    o = _euv(lb)
    sizes = [256, 128, 512, 256, 128]
    run = UnevenAbbe(sizes, o, 2e-9, tune=True, graph=True)
    assert run.graph is not None and set(run.tuned) == {128, 256, 512}
    for seed in (1, 2):
        clips = _clips(seed, sizes)
        imgs = run([torch.from_numpy(c).cuda() for c in clips])
        torch.cuda.synchronize()
        for c, im in zip(clips, imgs):
            g = lb.GridConfig(n_pixels=c.shape[0], pixel_size=2e-9)
            ref = lb.compute_aerial_image(c.astype(np.float64), o, g)
            got = im.double().cpu().numpy()
            assert float(np.abs(got - ref).max() / np.abs(ref).max()) <= TOL


def test_uneven_function_numpy_in_numpy_out(lb):
    from lithobat_b200.uneven import compute_aerial_uneven
    o = _euv(lb)
    clips = _clips(3, [128, 256])
    out = compute_aerial_uneven(clips, o, 2e-9, return_raw=True)
    for c, im in zip(clips, out):
        assert isinstance(im, np.ndarray) and im.dtype == np.float64 and im.shape == c.shape
        g = lb.GridConfig(n_pixels=c.shape[0], pixel_size=2e-9)
        ref = lb.compute_aerial_image(c.astype(np.float64), o, g, return_raw=True)[0]
        assert float(np.abs(im - ref).max() / np.abs(ref).max()) <= TOL


def test_uneven_ilt_groups_and_steps(lb):
    """Mixed sizes: 128^2 (kernel band on chip) and 256^2 (wide band) at 2 nm
    EUV; each group's step equals its own IltBatch step, costs fall."""
    import torch
    from lithobat_b200 import ilt
    from lithobat_b200.uneven import UnevenIlt
    o = lb.OpticsConfig(wavelength=13.5e-9, NA=0.33, source_grid=15, normalisation="clear",
                        source_spec=__import__("lithobat_b200.source", fromlist=["Source"]).Source.dipole(
                            0.9, 0.6, opening_deg=60).to_dict())
    sizes = [256, 128, 128]
    tg = _clips(7, sizes)
    rng = np.random.default_rng(8)
    th = [0.5 * rng.standard_normal((n, n)).astype(np.float32) for n in sizes]

    def params(k):
        return ilt.IltParams(scale=1.0 / k.clear, level=0.3, steepness=15.0, step=0.1, beta=4.0)
    u = UnevenIlt(tg, th, o, 2e-9, params, max_kernels=12)
    assert [g[0] for g in u.groups] == [128, 256]
    assert u.groups[0][2].halfwidth <= 15 < u.groups[1][2].halfwidth
    c0 = [float(c) for c in u.step()]
    for _ in range(4):
        c = [float(x) for x in u.step()]
    assert all(b < a for a, b in zip(c0, c))
    # the 256^2 group against its own batch
    k = u.groups[1][2]
    b = ilt.IltBatch(k, torch.from_numpy(tg[0][None]).cuda(), torch.from_numpy(th[0][None]).cuda(), params(k))
    for _ in range(5):
        b.step(want_signed=False)
    assert float((b.theta[0] - u.theta()[0]).abs().max()) < 1e-5
