"""The torch.ops.litho operators are registered and shape-check on meta
tensors (fake implementations; nothing runs, no GPU needed)."""

from __future__ import annotations

import torch

import lithobat_b200  # noqa: F401  (registers the operators)


def test_operators_are_registered():
    for name in ("abbe", "abbe_clear", "socs_forward", "socs_backward"):
        assert hasattr(torch.ops.litho, name), name


def test_fake_shapes():
    m = torch.empty((3, 64, 64), device="meta")
    table = torch.empty((5, 9), dtype=torch.complex64, device="meta")
    w = torch.empty((5,), dtype=torch.float64, device="meta")
    out = torch.ops.litho.socs_forward(m, table, w, 1)
    assert out.shape == (3, 64, 64) and out.dtype == torch.float32
    g = torch.ops.litho.socs_backward(m, table, w, 1, out)
    assert g.shape == (3, 64, 64) and g.dtype == torch.float32
    plan = torch.zeros(120, dtype=torch.uint8)
    blob = torch.empty(64, dtype=torch.uint8, device="meta")
    img, pk = torch.ops.litho.abbe(m, plan, blob, table, 6)
    assert img.shape == (6, 64, 64) and pk.shape == (6,)
    assert torch.ops.litho.abbe_clear(plan, blob, 6).shape == (6,)
