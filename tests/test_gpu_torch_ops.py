"""torch.ops.litho.* on the GPU: against the reference's outputs (golden
fixtures) and against the Python entry points they share kernels with."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden

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


def _optics(lb, od):
    od = dict(od)
    od["zernike_coeffs"] = {int(k): v for k, v in (od.get("zernike_coeffs") or {}).items()}
    keep = {k: od[k] for k in lb.OpticsConfig.__dataclass_fields__ if k in od}
    return lb.OpticsConfig(**keep)


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_socs_forward_and_its_autograd_backward_match_the_reference(lb):
    """ilt_small: the reference's socs_fields intensity and socs_gradient of
    a sensitivity, through the operators and torch autograd."""
    import torch
    from lithobat_b200.torch_ops import socs_operands
    a, od, gd = load_golden("ilt_small")
    k = lb.SOCSKernels.build(_optics(lb, od), lb.GridConfig(**gd), tol=1e-6)
    table, w, h = socs_operands(k)
    m = torch.tensor(np.stack([a["mask"], a["mask3"]]), dtype=torch.float32, device="cuda", requires_grad=True)
    img = torch.ops.litho.socs_forward(m, table, w, h)
    e_i = rel(img[0].detach().cpu().numpy(), a["intensity"])
    sens = torch.tensor(np.stack([a["sens"], a["sens"] * 0.5]), dtype=torch.float32, device="cuda")
    (img * sens).sum().backward()
    e_g = rel(m.grad[0].cpu().numpy(), a["grad"])
    print(f"PARITY torch_ops_socs_forward {e_i:.3e} backward {e_g:.3e}")
    assert e_i <= TOL_I and e_g <= TOL_G
    # the second clip's gradient is linear in its sensitivity
    g1 = torch.ops.litho.socs_backward(m.detach()[1:], table, w, h, sens[1:] * 2.0)
    np.testing.assert_allclose(g1[0].cpu().numpy(), 2.0 * m.grad[1].cpu().numpy(), rtol=0,
                               atol=1e-6 * float(m.grad[1].abs().max()))


def test_socs_forward_equals_the_socs_image_path(lb):
    """The operator and SOCSKernels.raw (the Abbe engine with a kernel table)
    give the same images on a 1024^2 K=24 batch (complex masks too)."""
    import torch
    from lithobat_b200.torch_ops import socs_operands
    o = lb.OpticsConfig(wavelength=193e-9, NA=1.35, n_immersion=1.44, source_type="annular", sigma_inner=0.5,
                        sigma_outer=0.8, normalisation="clear")
    g = lb.GridConfig(n_pixels=1024, pixel_size=1e-9)
    k = lb.SOCSKernels.build(o, g, tol=0.0, max_kernels=24)
    table, w, h = socs_operands(k)
    rng = np.random.default_rng(5)
    masks = np.stack([lb.patterns.manhattan_clip(rng, 1024, 1e-9) for _ in range(3)]).astype(np.float32)
    md = torch.from_numpy(masks).cuda()
    a = torch.ops.litho.socs_forward(md, table, w, h)
    b, _pk = k.raw_batch(md)
    assert float((a - b).abs().max()) <= 1e-6 * float(b.abs().max())
    mc = (md * (0.25 + 0.5j)).to(torch.complex64)
    c = torch.ops.litho.socs_forward(mc, table, w, h)
    # a constant complex factor scales every intensity by its |.|^2 = 0.3125
    assert float((c - 0.3125 * b).abs().max()) <= 1e-5 * float(b.abs().max())
    bc, _ = k.raw_batch(mc)
    assert float((c - bc).abs().max()) <= 1e-6 * float(bc.abs().max())


@pytest.mark.parametrize("name", ["abbe_vector_te", "abbe_annular_aberrated", "abbe_dipole_exact_clear"])
def test_abbe_operator_and_device_clear(lb, name):
    import torch
    from lithobat_b200 import aerial
    from lithobat_b200.torch_ops import plan_tensor
    a, od, gd = load_golden(name)
    o, g = _optics(lb, od), lb.GridConfig(**gd)
    v = lb.config.optics_view(o)
    n = int(g.n_pixels)
    cplx = bool(np.iscomplexobj(a["mask"]))
    pd = aerial.plan_abbe([v], n, float(g.pixel_size), [[(v.defocus, v.image_index)]], 1.0, True, cplx)
    dev = torch.device("cuda", 0)
    table = aerial.pupil_table(pd, dev, torch.cuda.current_stream().cuda_stream)
    m = torch.tensor(np.asarray(a["mask"], dtype=np.complex64 if cplx else np.float32)[None], device=dev)
    img, peak = torch.ops.litho.abbe(m, plan_tensor(pd), pd._blob_dev, table, pd.n_out)
    assert rel(img[0].cpu().numpy(), a["raw"]) <= TOL_I
    assert float(peak[0]) == pytest.approx(float(a["peak"]), rel=TOL_I)
    clear = torch.ops.litho.abbe_clear(plan_tensor(pd), pd._blob_dev, pd.n_out)
    assert float(clear[0]) == pytest.approx(float(a["clear"]), rel=1e-12)
    assert float(clear[0]) == pytest.approx(float(pd.clears[0]), rel=1e-12)


def test_device_clear_of_a_mirrored_multi_plane_batch(lb):
    """litho_abbe_clear against the host FP64 clears for a multilayer (EUV)
    vector batch with two planes per clip."""
    import torch
    from lithobat_b200 import aerial
    from lithobat_b200.torch_ops import plan_tensor
    from lithobat_b200.source import Source
    o = lb.OpticsConfig(wavelength=13.5e-9, NA=0.33, source_grid=21, mask_model="multilayer",
                        imaging_model="vector", polarisation="unpolarised",
                        source_spec=Source.dipole(0.9, 0.6, opening_deg=60).to_dict())
    v = lb.config.optics_view(o)
    planes = [[(0.0, 1.0), (40e-9, 1.0)]] * 2
    pd = aerial.plan_abbe([v, v], 128, 2e-9, planes, 1.0, True, False)
    blob = torch.from_numpy(pd.blob).cuda()
    clear = torch.ops.litho.abbe_clear(plan_tensor(pd), blob, pd.n_out).cpu().numpy()
    np.testing.assert_allclose(clear, pd.clears, rtol=1e-12)
