"""Host-to-host pipelined imaging equals the one-call API batch by batch."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lithobat_b200
    return lithobat_b200


def test_pipeline_matches_one_call_api(lb):
    import torch
    from lithobat_b200.pipeline import AbbePipeline
    g = lb.GridConfig(n_pixels=128, pixel_size=2e-9)
    o = lb.OpticsConfig(NA=1.35, n_immersion=1.44, imaging_model="vector", polarisation="te",
                        source_type="annular", sigma_inner=0.5, sigma_outer=0.9, source_grid=9)
    rng = np.random.default_rng(0)
    batches = []
    for b in range(5):
        c = np.stack([lb.patterns.contact_array(128, 2e-9, p * 1e-9, p * 1e-9, 0.5 * p * 1e-9)
                      for p in rng.integers(50, 90, size=4)])
        batches.append(torch.from_numpy(lb.patterns.to_attenuated_psm(1.0 - c, 0.06, 180.0)
                                        .astype(np.complex64)).pin_memory())
    outs = [torch.empty((4, 128, 128), dtype=torch.float32).pin_memory() for _ in range(5)]
    pipe = AbbePipeline(o, g, 4, mask_complex=True, depth=2)
    pipe.run(batches, outs)
    for hin, hout in zip(batches, outs):
        ref, _, _ = lb.compute_aerial_batch(hin.cuda(), o, g)
        np.testing.assert_allclose(hout.numpy(), ref[:, 0].cpu().numpy(), rtol=0, atol=1e-6)
