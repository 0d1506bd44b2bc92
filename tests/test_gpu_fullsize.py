"""The benchmark workloads at their full sizes, against the FP64 oracle.

Each test runs the engine exactly as the benchmark does (same batch sizes, so
the same kernels: the 1024^2 headline batch takes the tcgen05 synthesis) and
compares outputs with the oracle's FP64 numpy restatement of the reference
(dense FFTs in complex128, the reference's own algorithm) on a few clips of
the batch. Bounds (stated per result):

* images: max |I_gpu - I_fp64| / max I_fp64 <= 1e-5;
* ILT objective: cost relative error <= 1e-5; gradient max |dg| / max |g|
  <= 1e-5 (FP32 band-limited adjoint against the FP64 dense adjoint of 48
  full FFTs; about 2.5e-6 measured on a B200).

Measured errors are printed as ``PARITY <case> <error>`` lines (run with -s).
The oracle takes about 30-40 s per 1024^2 / 400-point image on 8-16 cores.
"""

from __future__ import annotations

import time

import numpy as np
import pytest

from oracle import litho_oracle as O

pytestmark = pytest.mark.gpu
TOL_I = 1e-5
TOL_G = 1e-5


@pytest.fixture(scope="module")
def lb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lithobat_b200
    return lithobat_b200


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    return float(np.abs(a - b).max() / np.abs(b).max())


def report(case: str, err: float, t0: float) -> None:
    print(f"PARITY {case} {err:.3e} (oracle {time.perf_counter() - t0:.1f} s)", flush=True)


def c3_masks(seed: int, count: int, n: int = 1024, px: float = 1e-9):
    """6 % att-PSM (phase pi) contact-hole arrays, pitch 80-140 nm, hole 40-70 nm."""
    from lithobat_b200 import patterns
    rng = np.random.default_rng(seed)
    out = np.empty((count, n, n), dtype=np.complex64)
    for i in range(count):
        p = rng.uniform(80e-9, 140e-9)
        hole = rng.uniform(40e-9, 70e-9)
        out[i] = patterns.to_attenuated_psm(1.0 - patterns.contact_array(n, px, p, p, hole), 0.06, 180.0)
    return out


def test_c3_vector_te_1024_in_a_tensor_core_batch(lb):
    """Vector TE, NA 1.35/1.44, annular 0.5-0.9 at source grid 31 (400 points,
    1200 transforms), 1024^2 at 1 nm, 80 att-PSM clips in one call (>= 74:
    the tcgen05 FP16 hi/lo synthesis), peak normalisation as benchmarked."""
    import torch
    from lithobat_b200 import aerial
    B = 80
    o = lb.OpticsConfig(NA=1.35, n_immersion=1.44, imaging_model="vector", polarisation="te",
                        source_type="annular", sigma_inner=0.5, sigma_outer=0.9, source_grid=31)
    v = lb.config.optics_view(o)
    masks = c3_masks(3, B)
    pd = aerial.plan_abbe([v] * B, 1024, 1e-9, [[(v.defocus, v.image_index)]] * B, 1.0, False, True)
    assert pd.jobs // B == 400 and pd.transforms // B == 1200
    assert aerial.engine_info(pd) == {"engine": "coarse", "synthesis": "tensor_cores"}
    md = torch.from_numpy(masks).cuda()
    img, peak = aerial.run_abbe(pd, md)
    aerial.check_status(pd, md.device)
    img, peak = img.cpu().numpy(), peak.cpu().numpy()

    class G:
        n_pixels, pixel_size = 1024, 1e-9
    for c in (0, B - 1):
        t0 = time.perf_counter()
        raw, rpk, _ = O.abbe_sum(masks[c].astype(np.complex128), o, G, [(v.defocus, v.image_index)])
        e_img = rel(img[c], raw[0] / rpk[0])
        e_pk = abs(float(peak[c]) - rpk[0]) / rpk[0]
        report(f"c3_vector_te_1024_clip{c}_image", e_img, t0)
        report(f"c3_vector_te_1024_clip{c}_peak", e_pk, t0)
        assert e_img <= TOL_I and e_pk <= TOL_I


def test_c2_batch_512_per_clip_defocus_and_zernikes(lb):
    """64 Manhattan clips, 512^2 at 2 nm, quadrupole 0.7-0.9 30 deg, per-clip
    defocus U(-60, 60) nm and Z4-Z21 U(-0.02, 0.02) waves, complex64 masks,
    one batched call."""
    rng = np.random.default_rng(20)
    n, px, B = 512, 2e-9, 64
    masks = np.stack([lb.patterns.manhattan_clip(rng, n, px) for _ in range(B)]).astype(np.complex64)
    src = lb.Source.quadrupole(0.9, 0.7, 30, 0).to_dict()
    optics = [lb.OpticsConfig(NA=1.35, n_immersion=1.44, source_spec=src,
                              defocus=float(rng.uniform(-60e-9, 60e-9)),
                              zernike_coeffs={j: float(rng.uniform(-0.02, 0.02)) for j in range(4, 22)})
              for _ in range(B)]
    g = lb.GridConfig(n_pixels=n, pixel_size=px)
    img, peak, clear = lb.compute_aerial_batch(masks, optics, g, return_raw=True)
    img = img.cpu().numpy()
    for c in (0, 21, 42, 63):
        t0 = time.perf_counter()
        raw, rpk, rcl = O.compute_aerial_image(masks[c], optics[c], g, return_raw=True)
        e = rel(img[c, 0], raw)
        report(f"c2_quadrupole_512_clip{c}_raw", e, t0)
        assert e <= TOL_I
        assert float(peak[c, 0]) == pytest.approx(rpk, rel=TOL_I)
        assert float(clear[c, 0]) == pytest.approx(rcl, rel=1e-12)


def test_c4_ilt_objective_and_gradient_1024_k24(lb):
    """ArF immersion annular 0.5-0.8, K = 24 (tol 0), 1024^2 at 1 nm, clear
    normalisation, level 0.3, a = 50 (steepness 15): a 16-clip batch through
    the fused band-limited step; clips 0 and 15 against the FP64 objective."""
    import torch
    from lithobat_b200 import ilt
    n, px, B = 1024, 1e-9, 16
    o = lb.OpticsConfig(wavelength=193e-9, NA=1.35, n_immersion=1.44, source_type="annular", sigma_inner=0.5,
                        sigma_outer=0.8, normalisation="clear")
    g = lb.GridConfig(n_pixels=n, pixel_size=px)
    k = lb.SOCSKernels.build(o, g, tol=0.0, max_kernels=24)
    ref = O.socs_build(o, g, tol=0.0, max_kernels=24)
    assert len(k) == len(ref) == 24
    e_w = float(np.abs(k.weights - ref.weights).max() / ref.weights[0])
    report("c4_socs_weights", e_w, time.perf_counter())
    assert e_w <= 1e-9
    assert k.clear == pytest.approx(ref.clear, rel=1e-9)
    rng = np.random.default_rng(500)
    targets = np.stack([lb.patterns.manhattan_clip(rng, n, px) for _ in range(B)]).astype(np.float32)
    theta = (0.5 * rng.standard_normal((B, n, n))).astype(np.float32)
    p = ilt.IltParams(scale=1.0 / k.clear, level=0.3, steepness=15.0, beta=4.0)
    b = ilt.IltBatch(k, torch.from_numpy(targets).cuda(), torch.from_numpy(theta).cuda(), p)
    assert b.fast
    b.check_status()
    cost, grad = b.cost.cpu().numpy(), b.grad_m.cpu().numpy()
    for c in (0, B - 1):
        t0 = time.perf_counter()
        m = O.mask_of(theta[c].astype(np.float64), 4.0, 0.0)
        rc, rg, _, _ = O.objective(ref, targets[c].astype(np.float64), m, 1.0 / ref.clear, 0.3, 0.0, 1.0, 15.0)
        e_c = abs(float(cost[c]) - rc) / abs(rc)
        e_g = rel(grad[c], rg)
        report(f"c4_ilt_1024_k24_clip{c}_cost", e_c, t0)
        report(f"c4_ilt_1024_k24_clip{c}_gradient", e_g, t0)
        assert e_c <= 1e-5
        assert e_g <= TOL_G


def test_c5_euv_2048_clip_in_an_uneven_batch(lb):
    """EUV 13.5 nm NA 0.33, dipole 0.6-0.9 opening 60 deg at source grid 43
    (204 points), 2 nm pixels: a 2048^2 clip imaged inside an uneven batch with
    256^2 and 1024^2 clips (the wide-pupil engine, 1024-point sub-transforms)."""
    from lithobat_b200.source import Source
    from lithobat_b200.uneven import UnevenAbbe
    import torch
    o = lb.OpticsConfig(wavelength=13.5e-9, NA=0.33, source_grid=43,
                        source_spec=Source.dipole(0.9, 0.6, opening_deg=60).to_dict())
    rng = np.random.default_rng(700)
    sizes = [256, 2048, 1024]
    masks = [lb.patterns.manhattan_clip(rng, s, 2e-9, n_rect=(20, 60), width_nm=(20.0, 80.0)) for s in sizes]
    run = UnevenAbbe(sizes, o, 2e-9, tune=False, graph=True)
    imgs = run([torch.from_numpy(m.astype(np.float32)).cuda() for m in masks])
    run.check_status()
    assert len(lb.source_points(o)) == 204

    class G:
        n_pixels, pixel_size = 2048, 2e-9
    t0 = time.perf_counter()
    ref = O.compute_aerial_image(masks[1], o, G)
    e = rel(imgs[1].cpu().numpy(), ref)
    report("c5_euv_dipole_2048_image", e, t0)
    assert e <= TOL_I
