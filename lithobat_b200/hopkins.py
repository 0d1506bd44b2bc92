"""Sum of coherent systems (SOCS): the drop-in for ``litho_sim.expose.hopkins``.

``SOCSKernels.build(optics, grid, tol, max_kernels)`` mirrors
``expose/hopkins.py:SOCSKernels.build`` (:103-198) and ``.raw`` / ``.image``
mirror ``:205-223``. The decomposition runs on the GPU (``litho_socs_build``:
pupil matrix in FP64, Gram matrix on the tensor cores, FP64 Jacobi, kernels
and weights in FP64); the forward image runs through the band-limited
pipeline of ``aerial.py`` with the eigen-kernels as its table, one coherent
system per kernel.

Differences from the reference, all below the 1e-5 image tolerance:
* eigenpairs come from the S x S Gram matrix G = conj(A) A^T instead of the
  n_band x n_band TCC (same non-zero spectrum, kernels A^T u / sqrt(lambda));
* weights are the FP64 Rayleigh quotients |A^T u|^2;
* at most min(n_source, n_band) kernels, none below 1e-10 x lambda_max: the
  reference's eigh also returns round-off eigenvalues (down to ~1e-34 x
  lambda_max) which it keeps when ``tol=0``; they carry no image.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native as nat
from .aerial import normalisation_scale, run_abbe
from .config import optics_view
from .source import source_points

NOISE_FLOOR = 1e-10


def band_bins(n: int, pixel_size: float, k_max: float):
    """Signed (kx, ky) bins of the SOCS band |f| <= 2 k_max (1 + 1e-9), in the
    order numpy's nonzero visits them (hopkins.py:144-146), plus their
    physical frequencies."""
    f = np.fft.fftfreq(n, d=pixel_size)
    FX, FY = np.meshgrid(f, f)
    rows, cols = np.nonzero(np.hypot(FX, FY) <= 2.0 * k_max + 1e-9 * k_max)
    signed = lambda i: np.where(i <= (n - 1) // 2, i, i - n)  # noqa: E731
    return signed(cols).astype(np.int32), signed(rows).astype(np.int32), FX[rows, cols], FY[rows, cols]


def aperture_mask(fxb, fyb, src, k_max: float, chunk: int = 64) -> np.ndarray:
    """inside[s, b]: hypot(f_b - f_s) / k_max <= 1, the reference's own test
    (hopkins.py:157-159), in float64 on the host."""
    S = len(src)
    out = np.zeros((S, fxb.size), dtype=np.uint8)
    for s0 in range(0, S, chunk):
        dx = fxb[None, :] - src.fx[s0:s0 + chunk, None]
        dy = fyb[None, :] - src.fy[s0:s0 + chunk, None]
        out[s0:s0 + chunk] = (np.hypot(dx, dy) / k_max <= 1.0)
    return out


class SOCSKernels:
    """The eigen-kernels of one optical state, ready to image any mask."""

    def __init__(self, *, weights, clear, energy_kept, n_band, n_source, optics, grid, band_kx, band_ky,
                 phi_dev, gram_sweeps=None):
        self.weights = np.asarray(weights, dtype=np.float64)
        self.clear = float(clear)
        self.energy_kept = float(energy_kept)
        self.n_band = int(n_band)
        self.n_source = int(n_source)
        self.optics = optics
        self.grid = grid
        self.band_kx = band_kx
        self.band_ky = band_ky
        self._phi = phi_dev          # (K, n_band) complex128 on the device, unit norm
        self.gram_sweeps = gram_sweeps
        self._plans: dict = {}
        self._table = None
        self._tcc = None             # band TCC blob (device), False where it does not fit

    def __len__(self) -> int:
        return int(self.weights.size)

    def subset(self, index) -> "SOCSKernels":
        """The kernels at ``index`` (a slice or index array) as kernels of their
        own: same optics, grid, band and clear (the full set's open-frame
        intensity, so normalisation is unchanged). Images and gradients are
        linear in the kernel set, so the parts of a partition sum to the
        whole (the SOCS split of one clip over several GPUs)."""
        import torch
        idx = np.arange(len(self))[index]
        sel = torch.from_numpy(idx.astype(np.int64)).to(self._phi.device)
        return SOCSKernels(weights=self.weights[idx], clear=self.clear, energy_kept=self.energy_kept,
                           n_band=self.n_band, n_source=self.n_source, optics=self.optics, grid=self.grid,
                           band_kx=self.band_kx, band_ky=self.band_ky, phi_dev=self._phi.index_select(0, sel),
                           gram_sweeps=self.gram_sweeps)

    @staticmethod
    def supports(optics) -> bool:
        v = optics_view(optics)
        return v.imaging_model.lower() == "scalar" and v.mask_model == "thin"

    # ------------------------------------------------------------------
    @classmethod
    def build(cls, optics, grid, tol: float = 1e-8, max_kernels: int | None = None,
              gram: str = "tensor") -> "SOCSKernels":
        """Decompose the optics into kernels (hopkins.py:103-198).

        gram: "tensor" assembles the Gram matrix on the tcgen05 tensor cores
        (TF32 split into hi + lo, FP32 accumulate, FP64 reduction); "fp64"
        assembles it on the CUDA cores in FP64 (a check)."""
        if not cls.supports(optics):
            v = optics_view(optics)
            raise ValueError(
                "SOCS kernels apply to the scalar thin-mask process only; got "
                f"imaging_model={v.imaging_model!r}, mask_model={v.mask_model!r}. "
                "Use compute_aerial_image for those.")
        torch = nat.require_cuda()
        L = nat.lib()
        v = optics_view(optics)
        n, px = int(grid.n_pixels), float(grid.pixel_size)
        k_max = v.NA / v.wavelength
        src = source_points(v)
        S = len(src)
        kx, ky, fxb, fyb = band_bins(n, px, k_max)
        nb = int(kx.size)
        inside = aperture_mask(fxb, fyb, src, k_max)
        dev = torch.device("cuda", torch.cuda.current_device())
        pupil = np.zeros(1, dtype=nat.PUPIL_DTYPE)
        pupil["wavelength"], pupil["NA"] = v.wavelength, v.NA
        pupil["defocus"], pupil["n_image"] = v.defocus, v.image_index
        zern = np.zeros(21)
        for j, c in v.zernike:
            if 1 <= j <= 21:
                zern[j - 1] = c
        pupil["zernike"] = zern
        pupil["exact_defocus"] = int(v.exact_defocus)
        pupil["has_zernike"] = int(bool(np.any(zern != 0.0)))
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        d_pupil = t(pupil.view(np.uint8))
        d_fx, d_fy, d_w = t(src.fx), t(src.fy), t(src.weight)
        d_kx, d_ky, d_in = t(kx), t(ky), t(inside)
        phi = torch.empty((S, nb), dtype=torch.complex128, device=dev)
        lam = torch.empty(S, dtype=torch.float64, device=dev)
        ws_bytes = C.c_size_t(0)
        nat.check("litho_socs_workspace", L.litho_socs_workspace(S, nb, C.byref(ws_bytes)))
        ws = torch.empty(ws_bytes.value, dtype=torch.uint8, device=dev)
        s = nat.stream_ptr(torch, dev)
        mode = {"tensor": 0, "fp64": 1}[gram]
        nat.check("litho_socs_build", L.litho_socs_build(
            d_pupil.data_ptr(), d_fx.data_ptr(), d_fy.data_ptr(), d_w.data_ptr(), S, d_kx.data_ptr(),
            d_ky.data_ptr(), nb, d_in.data_ptr(), n, px, mode, phi.data_ptr(), lam.data_ptr(), None,
            ws.data_ptr(), ws.numel(), s))
        sweeps = C.c_int(0)
        nat.check("litho_socs_status", L.litho_socs_status(S, nb, ws.data_ptr(), C.byref(sweeps), s))
        lam_h = lam.cpu().numpy()
        order = np.argsort(lam_h, kind="stable")[::-1]
        ev = lam_h[order]
        lmax = ev[0] if ev.size else 0.0
        keep = (ev > (tol * lmax if ev.size else 0.0)) & (ev > 0.0) & (ev > NOISE_FLOOR * lmax)
        keep[min(S, nb):] = False
        if max_kernels is not None:
            keep[max_kernels:] = False
        idx = order[keep]
        lam_k = ev[keep]
        sel = torch.from_numpy(idx.copy()).to(dev)
        phi_k = phi.index_select(0, sel) / torch.from_numpy(np.sqrt(lam_k)).to(dev)[:, None]
        # open frame: a clear mask has only the DC order (hopkins.py:188-191)
        dc = np.nonzero((kx == 0) & (ky == 0))[0]
        if dc.size and lam_k.size:
            d = phi_k[:, int(dc[0])].cpu().numpy()
            clear = float(np.sum(lam_k * np.abs(d) ** 2))
        else:
            clear = 0.0
        trace = float(np.sum(src.weight * inside.sum(axis=1)))   # trace of the TCC, exactly
        kept = float(lam_k.sum() / trace) if trace > 0 else 1.0
        return cls(weights=lam_k, clear=clear, energy_kept=kept, n_band=nb, n_source=S, optics=optics,
                   grid=grid, band_kx=kx, band_ky=ky, phi_dev=phi_k, gram_sweeps=int(sweeps.value))

    # ------------------------------------------------------------------
    @property
    def kernels(self) -> np.ndarray:
        """(K, N, N) complex128 kernels on the full FFT grid, zero off the band
        (the reference's ``SOCSKernels.kernels``). Materialised on demand."""
        n = int(self.grid.n_pixels)
        out = np.zeros((len(self), n, n), dtype=np.complex128)
        out[:, self.band_ky % n, self.band_kx % n] = self._phi.cpu().numpy()
        return out

    @property
    def halfwidth(self) -> int:
        return int(max(np.abs(self.band_kx).max(), np.abs(self.band_ky).max()))

    def table(self):
        """Kernel table for the band-limited engine: (K, (2h+1)^2) complex64."""
        if self._table is None:
            torch = nat.require_cuda()
            h = self.halfwidth
            side = 2 * h + 1
            pos = torch.from_numpy(((self.band_ky + h) * side + (self.band_kx + h)).astype(np.int64)).to(
                self._phi.device)
            tab = torch.zeros((len(self), side * side), dtype=torch.complex64, device=self._phi.device)
            tab[:, pos] = self._phi.to(torch.complex64)
            self._table = tab.contiguous()
        return self._table

    def tcc(self):
        """The band TCC of these kernels on the device (``litho_socs_tcc_build``:
        T(f, f') = sum_k lambda_k conj phi_k(f) phi_k(f') in FP64, stored as
        complex64 with its index maps), built once; None where it would not
        stay resident in L2 (wide bands), and the per-kernel engines serve."""
        if self._tcc is False:
            return None
        if self._tcc is None:
            torch = nat.require_cuda()
            L = nat.lib()
            nb, h = int(self.band_kx.size), self.halfwidth
            nbytes = C.c_size_t(0)
            st = L.litho_socs_tcc_bytes(nb, h, C.byref(nbytes))
            if st == nat.LITHO_E_UNSUPPORTED:
                self._tcc = False
                return None
            nat.check("litho_socs_tcc_bytes", st)
            dev = self._phi.device
            buf = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
            kx = torch.from_numpy(self.band_kx.astype(np.int32)).to(dev)
            ky = torch.from_numpy(self.band_ky.astype(np.int32)).to(dev)
            lam = torch.from_numpy(self.weights.copy()).to(dev)
            bad = torch.zeros((1,), dtype=torch.int32, device=dev)
            phi = self._phi.contiguous()
            nat.check("litho_socs_tcc_build", L.litho_socs_tcc_build(
                phi.data_ptr(), lam.data_ptr(), len(self), kx.data_ptr(), ky.data_ptr(), nb, h, buf.data_ptr(),
                buf.numel(), bad.data_ptr(), nat.stream_ptr(torch, dev)))
            if int(bad.item()):
                raise nat.LithoError("litho_socs_tcc_build", nat.LITHO_E_BAND,
                                     "a band point lies outside the kernel box")
            self._tcc = buf
        return self._tcc

    def _plan(self, n_clips: int, mask_complex: bool, norm_mode: tuple):
        key = (n_clips, mask_complex, norm_mode)
        pd = self._plans.get(key)
        if pd is None:
            from .aerial import plan_from_table
            pd = plan_from_table(int(self.grid.n_pixels), float(self.grid.pixel_size), n_clips, self.weights,
                                 self.halfwidth, mask_complex, norm_mode)
            self._plans[key] = pd
        return pd

    def raw_batch(self, masks_dev, norm_mode=(0, 1.0)):
        """(C, N, N) float32 images and (C,) raw peaks for device masks."""
        pd = self._plan(int(masks_dev.shape[0]), bool(masks_dev.is_complex()), norm_mode)
        pd._table_dev = self.table()
        return run_abbe(pd, masks_dev)

    def raw(self, mask):
        """(raw, peak, clear), the reference's ``SOCSKernels.raw`` (hopkins.py:205-218)."""
        n = int(self.grid.n_pixels)
        if tuple(np.shape(mask)[-2:]) != (n, n) or np.ndim(mask) != 2:
            raise ValueError(f"mask must be {(n, n)} for these kernels, got {tuple(np.shape(mask))}")
        torch = nat.require_cuda()
        from .aerial import _as_device_masks, _is_torch
        md = _as_device_masks(torch, mask, n)
        img, pk = self.raw_batch(md)
        if not _is_torch(mask):
            from .aerial import check_status
            check_status(self._plan(1, bool(md.is_complex()), (0, 1.0)), md.device)
        a = img[0] if _is_torch(mask) else img[0].cpu().numpy().astype(np.float64)
        return a, float(pk[0]), self.clear

    def image(self, mask, dose: float = 1.0):
        """The aerial image, normalised as ``optics.normalisation`` says and dosed."""
        raw, peak, clear = self.raw(mask)
        return raw * normalisation_scale(optics_view(self.optics).normalisation, peak, clear, dose)


__all__ = ["SOCSKernels", "band_bins", "aperture_mask"]
