"""The imaging engine as PyTorch operators: ``torch.ops.litho.*``.

Each operator is a thin call into the C ABI of ``liblitho_b200.so`` on the
input's device and current stream; outputs and workspaces come from torch's
caching allocator. Fake (meta) implementations give output shapes without
running anything, and ``litho::socs_forward`` carries its adjoint as the
autograd formula, so SOCS imaging composes with torch autograd:

* ``litho::abbe(masks, plan, blob, table, n_out)`` -> (images, peaks): the
  Abbe sum of a planned batch (expose/aerial_image.py:_abbe_sum, :351-494,
  normalised per output as the plan says). ``plan`` is the 120-byte
  ``LithoAbbePlan`` as a CPU uint8 tensor, ``blob`` its device descriptors,
  ``table`` its pupil table (``aerial.pupil_table``).
* ``litho::abbe_clear(plan, blob, n_out)`` -> (n_out,) float64: the clear
  throughput of every output, in FP64 on the device.
* ``litho::socs_forward(masks, table, weights, h)`` -> raw SOCS intensity
  (C, N, N) (expose/hopkins.py:205-218, opc/ilt.py:227-231).
* ``litho::socs_backward(masks, table, weights, h, grad_image)`` -> d/dmasks
  of sum(grad_image * intensity) (opc/ilt.py:socs_gradient, :235-266).

Masks are (C, N, N) CUDA tensors: float32 (or complex64 for the forward
operators); table is (K, (2h+1)^2) complex64 (``SOCSKernels.table()``) and
weights (K,) float64 on the device.
"""

from __future__ import annotations

import ctypes as C

import torch
from torch import Tensor

from . import _native as nat


def _plan_struct(plan: Tensor) -> nat.AbbePlan:
    raw = bytes(plan.cpu().contiguous().numpy().tobytes())
    if len(raw) != C.sizeof(nat.AbbePlan):
        raise ValueError(f"plan must be the {C.sizeof(nat.AbbePlan)}-byte LithoAbbePlan, got {len(raw)} bytes")
    return nat.AbbePlan.from_buffer_copy(raw)


def plan_tensor(pd) -> Tensor:
    """The ``LithoAbbePlan`` of a planned batch as the CPU uint8 tensor the
    operators take."""
    return torch.frombuffer(bytearray(bytes(pd.plan)), dtype=torch.uint8)


def _stream(dev) -> int:
    return int(torch.cuda.current_stream(dev).cuda_stream)


def _ws(dev, nbytes: int) -> Tensor:
    # 256-byte aligned: the caching allocator's blocks are
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=dev)


@torch.library.custom_op("litho::abbe", mutates_args=())
def abbe(masks: Tensor, plan: Tensor, blob: Tensor, table: Tensor, n_out: int) -> tuple[Tensor, Tensor]:
    L = nat.lib()
    p = _plan_struct(plan)
    if p.n_out != n_out:
        raise ValueError(f"plan has {p.n_out} outputs, n_out says {n_out}")
    masks = masks.contiguous()
    dev = masks.device
    img = torch.empty((n_out, p.n, p.n), dtype=torch.float32, device=dev)
    peak = torch.empty((n_out,), dtype=torch.float32, device=dev)
    nb = C.c_size_t(0)
    nat.check("litho_abbe_workspace", L.litho_abbe_workspace(C.byref(p), C.byref(nb)))
    ws = _ws(dev, nb.value)
    nat.check("litho_abbe_tabled", L.litho_abbe_tabled(C.byref(p), blob.data_ptr(), table.data_ptr(),
                                                        masks.data_ptr(), img.data_ptr(), peak.data_ptr(),
                                                        ws.data_ptr(), ws.numel(), _stream(dev)))
    return img, peak


@abbe.register_fake
def _abbe_fake(masks, plan, blob, table, n_out):
    n = masks.shape[-1]
    return masks.new_empty((n_out, n, n), dtype=torch.float32), masks.new_empty((n_out,), dtype=torch.float32)


@torch.library.custom_op("litho::abbe_clear", mutates_args=())
def abbe_clear(plan: Tensor, blob: Tensor, n_out: int) -> Tensor:
    p = _plan_struct(plan)
    out = torch.empty((n_out,), dtype=torch.float64, device=blob.device)
    nat.check("litho_abbe_clear", nat.lib().litho_abbe_clear(C.byref(p), blob.data_ptr(), out.data_ptr(),
                                                              _stream(blob.device)))
    return out


@abbe_clear.register_fake
def _abbe_clear_fake(plan, blob, n_out):
    return blob.new_empty((n_out,), dtype=torch.float64)


def _check_table(table: Tensor, weights: Tensor, h: int) -> int:
    K = int(weights.numel())
    if table.dtype != torch.complex64 or tuple(table.shape) != (K, (2 * h + 1) ** 2):
        raise ValueError(f"table must be ({K}, {(2 * h + 1) ** 2}) complex64, got {tuple(table.shape)} {table.dtype}")
    if weights.dtype != torch.float64:
        raise ValueError("weights must be float64")
    return K


@torch.library.custom_op("litho::socs_forward", mutates_args=())
def socs_forward(masks: Tensor, table: Tensor, weights: Tensor, h: int) -> Tensor:
    L = nat.lib()
    K = _check_table(table, weights, h)
    m = masks.contiguous()
    C_, n = int(m.shape[0]), int(m.shape[-1])
    cplx = int(m.is_complex())
    dev = m.device
    nb = C.c_size_t(0)
    nat.check("litho_socs_forward_workspace", L.litho_socs_forward_workspace(C_, n, K, h, cplx, C.byref(nb)))
    ws = _ws(dev, nb.value)
    img = torch.empty((C_, n, n), dtype=torch.float32, device=dev)
    peak = torch.empty((C_,), dtype=torch.float32, device=dev)
    nat.check("litho_socs_forward", L.litho_socs_forward(
        table.contiguous().data_ptr(), weights.contiguous().data_ptr(), K, h, m.data_ptr(), cplx, C_, n, 0, 1.0,
        img.data_ptr(), peak.data_ptr(), ws.data_ptr(), ws.numel(), _stream(dev)))
    return img


@socs_forward.register_fake
def _socs_forward_fake(masks, table, weights, h):
    return masks.new_empty(tuple(masks.shape), dtype=torch.float32)


@torch.library.custom_op("litho::socs_backward", mutates_args=())
def socs_backward(masks: Tensor, table: Tensor, weights: Tensor, h: int, grad_image: Tensor) -> Tensor:
    L = nat.lib()
    K = _check_table(table, weights, h)
    m = masks.contiguous().to(torch.float32)
    g = grad_image.contiguous().to(torch.float32)
    C_, n = int(m.shape[0]), int(m.shape[-1])
    dev = m.device
    nb = C.c_size_t(0)
    nat.check("litho_socs_backward_workspace", L.litho_socs_backward_workspace(C_, n, K, h, C.byref(nb)))
    ws = _ws(dev, nb.value)
    out = torch.empty((C_, n, n), dtype=torch.float32, device=dev)
    nat.check("litho_socs_backward", L.litho_socs_backward(
        table.contiguous().data_ptr(), weights.contiguous().data_ptr(), K, h, m.data_ptr(), C_, n, g.data_ptr(),
        1.0, out.data_ptr(), ws.data_ptr(), ws.numel(), _stream(dev)))
    return out


@socs_backward.register_fake
def _socs_backward_fake(masks, table, weights, h, grad_image):
    return masks.new_empty(tuple(masks.shape), dtype=torch.float32)


def _socs_setup(ctx, inputs, output):
    masks, table, weights, h = inputs
    ctx.save_for_backward(masks, table, weights)
    ctx.h = h


def _socs_grad(ctx, grad_image):
    masks, table, weights = ctx.saved_tensors
    return socs_backward(masks, table, weights, ctx.h, grad_image), None, None, None


socs_forward.register_autograd(_socs_grad, setup_context=_socs_setup)


def socs_operands(kernels):
    """(table, weights, h) of a ``SOCSKernels`` set for the SOCS operators."""
    w = getattr(kernels, "_weights_dev", None)
    table = kernels.table()
    if w is None or w.device != table.device:
        w = torch.from_numpy(kernels.weights.copy()).to(table.device)
        kernels._weights_dev = w
    return table, w, kernels.halfwidth


__all__ = ["abbe", "abbe_clear", "plan_tensor", "socs_backward", "socs_forward", "socs_operands"]
