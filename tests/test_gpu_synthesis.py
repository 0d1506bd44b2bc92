"""Band-limited synthesis through the C ABI (litho_band_synthesis) against
numpy's inverse FFT of the same Hermitian box, over box half-widths, grid
sizes and batch sizes that reach every synthesis engine: the tensor-core GEMM
(large batches; K padded to 16), the pair FFT,
the direct kernel and the wide scatter + FFT.

Bar: max |I_gpu - I_ref| / max |I_ref| <= 1e-5 (FP32 result; the tensor-core
path splits operands into FP16 hi + lo).
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from lithobat_b200 import _native as nat
    return torch, nat


def _hermitian_box(rng, h, n_fields):
    G = 2 * h + 1
    b = rng.standard_normal((n_fields, G, G)) + 1j * rng.standard_normal((n_fields, G, G))
    g = np.arange(-h, h + 1)
    b *= np.exp(-np.hypot(g[None, :, None], g[None, None, :]) / max(h, 1))[...]
    b = 0.5 * (b + np.conj(b[:, ::-1, ::-1]))      # B(-g) = conj B(g)
    b[:, h, h] = np.abs(b[:, h, h]) * 10
    return b


def _reference(box, n):
    F, G, _ = box.shape
    h = G // 2
    spec = np.zeros((F, n, n), complex)
    for iy, gy in enumerate(range(-h, h + 1)):
        for ix, gx in enumerate(range(-h, h + 1)):
            spec[:, gy % n, gx % n] += box[:, iy, ix]
    return np.fft.ifft2(spec).real * n * n


def _fields_for_tensor_cores(n):
    """Fields that make the batch large enough for the tensor-core engine
    (about 16 output tiles of 128 x 256 per SM)."""
    return -(-16 * 148 // ((n // 256) * (n // 128)))


@pytest.mark.parametrize("n,h,big", [(256, 0, True), (256, 3, True), (1024, 14, True), (512, 20, True),
                                     (256, 31, True), (2048, 9, True), (4096, 5, True),
                                     (256, 1, False), (1024, 14, False), (2048, 9, False),
                                     (128, 7, False), (512, 40, False), (1024, 100, False), (2048, 200, False),
                                     (2048, 400, False), (256, 100, False)])
def test_band_synthesis_matches_numpy(env, n, h, big):
    torch, nat = env
    L = nat.lib()
    rng = np.random.default_rng(n + h)
    F = _fields_for_tensor_cores(n) if big else 3
    box = _hermitian_box(rng, h, F)
    check = sorted({0, F // 2, F - 1})
    want = _reference(box[check], n)
    dev = torch.device("cuda", torch.cuda.current_device())
    bx = torch.from_numpy(box.astype(np.complex64)).to(dev)
    nb = C.c_size_t(0)
    nat.check("litho_band_synthesis_workspace", L.litho_band_synthesis_workspace(F, n, C.byref(nb)))
    ws = torch.empty(nb.value, dtype=torch.uint8, device=dev)
    out = torch.empty((F, n, n), dtype=torch.float32, device=dev)
    nat.check("litho_band_synthesis", L.litho_band_synthesis(
        bx.data_ptr(), F, n, h, 0, out.data_ptr(), ws.data_ptr(), ws.numel(), torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert int(ws[:4].view(torch.int32).item()) == 0          # no wait gave up
    got = out[check].double().cpu().numpy()
    err = float(np.abs(got - want).max() / np.abs(want).max())
    assert err <= 1e-5, err


@pytest.mark.parametrize("n,bm,cplx", [(1024, 200, False), (1024, 300, True), (2048, 100, False),
                                       (2048, 400, False), (2048, 250, True), (4096, 60, False), (256, 100, True)])
def test_band_spectrum_matches_numpy(env, n, bm, cplx):
    """litho_band_spectrum (rows, then columns of its own output) against
    numpy's fft2 restricted to |kx|, |ky| <= bm, including bands wide enough
    for the full-row transforms."""
    torch, nat = env
    L = nat.lib()
    rng = np.random.default_rng(n + bm)
    F = 2
    x = rng.standard_normal((F, n, n))
    if cplx:
        x = x + 1j * rng.standard_normal((F, n, n))
    k = np.arange(-bm, bm + 1) % n
    want = np.fft.fft2(x)[:, k][:, :, k] / (n * n)
    dev = torch.device("cuda", torch.cuda.current_device())
    xd = torch.from_numpy(x.astype(np.complex64 if cplx else np.float32)).to(dev)
    nb = C.c_size_t(0)
    nat.check("litho_band_spectrum_workspace", L.litho_band_spectrum_workspace(F, n, bm, C.byref(nb)))
    ws = torch.empty(nb.value, dtype=torch.uint8, device=dev)
    out = torch.empty((F, (2 * bm + 1) ** 2), dtype=torch.complex64, device=dev)
    nat.check("litho_band_spectrum", L.litho_band_spectrum(
        xd.data_ptr(), int(cplx), F, n, bm, 1.0 / (n * n), out.data_ptr(), ws.data_ptr(), ws.numel(),
        torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    got = out.cpu().numpy().astype(np.complex128).reshape(F, 2 * bm + 1, 2 * bm + 1)
    err = float(np.abs(got - want).max() / np.abs(want).max())
    assert err <= 1e-5, err
