"""Inverse lithography on the B200: the drop-in for ``litho_sim.opc.ilt``'s hot path.

* :func:`socs_fields`   — opc/ilt.py:208-232 (fields kept, intensity)
* :func:`socs_gradient` — opc/ilt.py:235-266 (the hand-written SOCS adjoint)
* :class:`Objective`    — opc/ilt.py:292-360 (relaxed resist, blur, TV, discreteness)
* :func:`mask_of`, :func:`grad_theta` — opc/ilt.py:368-389
* :class:`IltBatch`     — one fused ILT iteration (opc/ilt.py:576-596) for a batch
  of clips, entirely on the device: grad_theta, Adam, the beta anneal, mask_of
  and the objective's forward and adjoint
* :class:`SocsImage`    — ``torch.autograd.Function``: forward = SOCS intensity,
  backward = the adjoint
* :func:`run_ilt`       — the solve loop (opc/ilt.py:397-621), host-driven

Every stage is a C-ABI call into ``liblitho_b200.so`` (band spectra, coarse
SOCS forward and adjoint, band synthesis, objective, Adam, Gaussian blur).
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _native as nat
from .aerial import _as_device_masks, _is_torch, normalisation_scale, plan_from_table
from .config import optics_view
from .hopkins import SOCSKernels

N_PART = 64   # partial-sum blocks per clip for costs / pattern errors
KERNEL_HMAX_FUSED = 15   # widest kernel band (bins) of the on-chip SOCS adjoint


def band_limited_ok(n: int, h: int) -> bool:
    """Can the band-limited ILT stages serve kernels of half-width h on an
    n x n grid (on chip up to 15 bins, else a coarse grid of 128..1024 <= n)?"""
    if h <= KERNEL_HMAX_FUSED:
        return True
    from .aerial import coarse_grid
    L = coarse_grid(h)
    return 128 <= L <= 1024 and L <= n <= 4096 and (n & (n - 1)) == 0


def gaussian_weights(sigma: float, truncate: float = 4.0) -> np.ndarray:
    """scipy.ndimage's 1-D Gaussian (order 0): radius int(truncate sigma + 0.5),
    exp(-x^2 / (2 sigma^2)) normalised to unit sum, in float64."""
    r = int(truncate * float(sigma) + 0.5)
    x = np.arange(-r, r + 1, dtype=np.float64)
    w = np.exp(-0.5 / (float(sigma) ** 2) * x ** 2)
    return w / w.sum()


class _Stages:
    """Device stages bound to one set of SOCS kernels and one batch size.

    The image and adjoint band boxes come from the band TCC
    (``litho_socs_tcc_image`` / ``litho_socs_tcc_adjoint``) when the kernels'
    TCC stays resident in L2 and ``use_tcc`` allows it, else from the
    per-kernel coarse-grid engines (``litho_coarse_image``,
    ``litho_socs_adjoint``)."""

    def __init__(self, kernels: SOCSKernels, n_clips: int, use_tcc: bool = True):
        self.torch = nat.require_cuda()
        self.L = nat.lib()
        self.k = kernels
        self.n = int(kernels.grid.n_pixels)
        self.h = kernels.halfwidth
        self.C = int(n_clips)
        self.dev = kernels._phi.device
        self.side = 2 * self.h + 1
        self.pd = plan_from_table(self.n, float(kernels.grid.pixel_size), self.C, kernels.weights, self.h, False)
        self.blob = self.torch.from_numpy(self.pd.blob).to(self.dev)
        self.table = kernels.table()
        self.tcc = kernels.tcc() if use_tcc else None
        self.nb = int(kernels.band_kx.size)
        self._ws = {}
        self._blur = {}
        self._obj_counters = None     # litho_ilt_objective_totals' per-field block counters
        self._imgobj_ok = None

    def stream(self):
        return nat.stream_ptr(self.torch, self.dev)

    def ws(self, tag, nbytes):
        t = self._ws.get(tag)
        if t is None or t.numel() < nbytes:
            t = self.torch.empty(max(int(nbytes), 256), dtype=self.torch.uint8, device=self.dev)
            self._ws[tag] = t
        return t

    # -- transforms ---------------------------------------------------------
    def band(self, fields, bm: int, scale: float, tag: str = "band", out=None):
        """(F, (2bm+1)^2) complex64 band boxes of F dense fields (into ``out``
        when given)."""
        torch, L = self.torch, self.L
        F = int(fields.shape[0])
        nb = C.c_size_t(0)
        nat.check("litho_band_spectrum_workspace", L.litho_band_spectrum_workspace(F, self.n, bm, C.byref(nb)))
        ws = self.ws(tag, nb.value)
        if out is None:
            out = torch.empty((F, (2 * bm + 1) ** 2), dtype=torch.complex64, device=self.dev)
        nat.check("litho_band_spectrum", L.litho_band_spectrum(
            fields.data_ptr(), int(fields.is_complex()), F, self.n, bm, scale, out.data_ptr(), ws.data_ptr(),
            ws.numel(), self.stream()))
        return out

    def synth(self, box, h: int, complex_out: bool):
        torch, L = self.torch, self.L
        F = int(box.shape[0])
        nb = C.c_size_t(0)
        nat.check("litho_band_synthesis_workspace", L.litho_band_synthesis_workspace(F, self.n, C.byref(nb)))
        ws = self.ws("synth", nb.value)
        out = torch.empty((F, self.n, self.n), dtype=torch.complex64 if complex_out else torch.float32,
                          device=self.dev)
        nat.check("litho_band_synthesis", L.litho_band_synthesis(
            box.data_ptr(), F, self.n, h, int(complex_out), out.data_ptr(), ws.data_ptr(), ws.numel(),
            self.stream()))
        return out

    def mask_box(self, masks, out=None):
        return self.band(masks, self.h, 1.0 / (self.n * self.n), tag="band_mask", out=out)

    # workspaces whose first word is a device status (litho_band_spectrum,
    # litho_band_synthesis: LITHO_E_TIMEOUT when a bounded wait gave up); one
    # per call site of a step, so a step's every call keeps its own word
    STATUS_TAGS = ("band_mask", "band", "synth", "imgobj_band")

    def check_status(self) -> None:
        """Synchronise and raise ``LithoError`` if a bounded wait inside the
        latest band spectrum or synthesis call of any kind gave up."""
        self.torch.cuda.synchronize(self.dev)
        for tag in self.STATUS_TAGS:
            t = self._ws.get(tag)
            if t is not None:
                st = int(t[:4].view(self.torch.int32).item())
                if st:
                    nat.check(f"litho_band_{'synthesis' if tag == 'synth' else 'spectrum'}", st)

    def image_box(self, mbox):
        """Band box (C, (4h+1)^2) of the raw SOCS intensity from the mask band boxes."""
        torch, L = self.torch, self.L
        if self.tcc is not None:
            G = 4 * self.h + 1
            bbox = torch.empty((self.C, G * G), dtype=torch.complex64, device=self.dev)
            nat.check("litho_socs_tcc_image", L.litho_socs_tcc_image(
                self.tcc.data_ptr(), self.nb, self.h, mbox.data_ptr(), self.C, bbox.data_ptr(), self.stream()))
            return bbox
        nb = C.c_size_t(0)
        nat.check("litho_abbe_workspace", L.litho_abbe_workspace(C.byref(self.pd.plan), C.byref(nb)))
        ws = self.ws("coarse", nb.value)
        G = 4 * self.h + 1
        bbox = torch.empty((self.C, G * G), dtype=torch.complex64, device=self.dev)
        nat.check("litho_coarse_image", L.litho_coarse_image(
            C.byref(self.pd.plan), self.blob.data_ptr(), self.table.data_ptr(), mbox.data_ptr(), bbox.data_ptr(),
            ws.data_ptr(), ws.numel(), self.stream()))
        return bbox

    def image(self, mbox):
        """Raw SOCS intensity (C, N, N) from the mask band boxes."""
        return self.synth(self.image_box(mbox), 2 * self.h, False)

    def fields(self, mbox):
        """(C, K, N, N) complex64 coherent fields E_k = F^-1(phi_k F(m))."""
        K = len(self.k)
        boxes = (self.table[None, :, :] * mbox[:, None, :]).reshape(self.C * K, -1).contiguous()
        return self.synth(boxes, self.h, True).view(self.C, K, self.n, self.n)

    def adjoint(self, sens, scale: float = 1.0, mbox=None, field_boxes=None):
        """d/dm of sum_x sens(x) I(x): (C, N, N) float32 (opc/ilt.py:262-266)."""
        gbox = self.band(sens, 2 * self.h, scale / (self.n * self.n))
        return self.synth(self.adjoint_box(gbox, mbox, field_boxes), self.h, False)

    def adjoint_box(self, gbox, mbox=None, field_boxes=None, out=None):
        """Band box (C, (2h+1)^2) of the mask gradient from the band box of
        scale * dJ/dI on |g| <= 2h (already divided by N^2); into ``out``
        when given."""
        torch, L = self.torch, self.L
        hbox = out if out is not None else torch.empty((self.C, self.side * self.side), dtype=torch.complex64,
                                                       device=self.dev)
        if self.tcc is not None and field_boxes is None and mbox is not None:
            nat.check("litho_socs_tcc_adjoint", L.litho_socs_tcc_adjoint(
                self.tcc.data_ptr(), self.nb, self.h, mbox.data_ptr(), gbox.data_ptr(), self.C, hbox.data_ptr(),
                self.stream()))
            return hbox
        nb = C.c_size_t(0)
        nat.check("litho_socs_adjoint_workspace", L.litho_socs_adjoint_workspace(
            self.C, self.pd.plan.n_items, self.h, C.byref(nb)))
        ws = self.ws("adjoint", nb.value)
        nat.check("litho_socs_adjoint", L.litho_socs_adjoint(
            C.byref(self.pd.plan), self.blob.data_ptr(), self.table.data_ptr(),
            None if mbox is None else mbox.data_ptr(),
            None if field_boxes is None else field_boxes.data_ptr(), gbox.data_ptr(), hbox.data_ptr(),
            ws.data_ptr(), ws.numel(), self.stream()))
        return hbox

    # -- the fast step (no blur, smoothing or penalties) --------------------
    def fast_ok(self, p) -> bool:
        return (p.sigma_px < 1e-3 and p.smooth_px < 1e-3 and p.weight_tv == 0.0 and p.weight_discrete == 0.0
                and self.n % 4 == 0)

    def objective_split(self, mbox, target, scale, level, sign, steepness, want_signed=True, out_hbox=None,
                        out_cost=None, out_perr=None):
        """The objective from the mask band boxes, keeping only band boxes
        between steps: (cost (C,), gradient band box (C, (2h+1)^2), signed or
        None, perr (C,)). Synthesis of the image, the per-pixel resist, the
        band of dJ/dI, the adjoint to the gradient's band box. ``out_*``:
        write into these tensors (views of a larger batch's state)."""
        ibox = self.image_box(mbox)
        cost, gbox, signed, perr = self.objective_from_box(ibox, target, scale, level, sign, steepness, want_signed,
                                                           out_cost, out_perr)
        hbox = self.adjoint_box(gbox, mbox, out=out_hbox)
        return cost, hbox, signed, perr

    def objective_from_box(self, ibox, target, scale, level, sign, steepness, want_signed=True, out_cost=None,
                           out_perr=None):
        """The resist objective of the image whose band box (C, (4h+1)^2) is
        ``ibox``: (cost (C,), band box of scale * dJ/dI / N^2 on |g| <= 2h,
        signed or None, perr (C,))."""
        torch, L = self.torch, self.L
        a = steepness / max(abs(level), 1e-12)
        if self._obj_counters is None:
            self._obj_counters = torch.zeros((self.C,), dtype=torch.int32, device=self.dev)
        cost = out_cost if out_cost is not None else torch.empty((self.C,), dtype=torch.float64, device=self.dev)
        perr = out_perr if out_perr is not None else torch.empty((self.C,), dtype=torch.int64, device=self.dev)
        if not want_signed and self.image_objective_band_ok() and target.data_ptr() % 16 == 0:
            # the image is synthesised straight into the objective and dJ/dI
            # straight into its band rows (neither is stored)
            nb = C.c_size_t(0)
            nat.check("litho_ilt_image_objective_band_workspace", L.litho_ilt_image_objective_band_workspace(
                self.C, self.n, 2 * self.h, 2 * self.h, C.byref(nb)))
            ws = self.ws("imgobj_band", nb.value)
            G = 4 * self.h + 1
            gbox = torch.empty((self.C, G * G), dtype=torch.complex64, device=self.dev)
            nat.check("litho_ilt_image_objective_band", L.litho_ilt_image_objective_band(
                ibox.data_ptr(), self.C, self.n, 2 * self.h, target.data_ptr(), float(scale), float(level),
                float(sign), float(a), 2 * self.h, float(scale) / (self.n * self.n), gbox.data_ptr(),
                self._obj_counters.data_ptr(), cost.data_ptr(), perr.data_ptr(), ws.data_ptr(), ws.numel(),
                self.stream()))
            return cost, gbox, None, perr
        if not want_signed and self.image_objective_ok() and target.data_ptr() % 16 == 0:
            # the image is synthesised straight into the objective (never stored)
            nb = C.c_size_t(0)
            nat.check("litho_ilt_image_objective_workspace", L.litho_ilt_image_objective_workspace(
                self.C, self.n, 2 * self.h, C.byref(nb)))
            ws = self.ws("imgobj", nb.value)
            dfield = torch.empty((self.C, self.n, self.n), dtype=torch.float32, device=self.dev)
            nat.check("litho_ilt_image_objective", L.litho_ilt_image_objective(
                ibox.data_ptr(), self.C, self.n, 2 * self.h, target.data_ptr(), float(scale), float(level),
                float(sign), float(a), dfield.data_ptr(), self._obj_counters.data_ptr(), cost.data_ptr(),
                perr.data_ptr(), ws.data_ptr(), ws.numel(), self.stream()))
            gbox = self.band(dfield, 2 * self.h, float(scale) / (self.n * self.n))
            return cost, gbox, None, perr
        raw = self.synth(ibox, 2 * self.h, False)
        dfield = torch.empty_like(raw)
        signed = torch.empty_like(raw) if want_signed else None
        cpart = torch.empty((self.C, N_PART), dtype=torch.float64, device=self.dev)
        ppart = torch.empty((self.C, N_PART), dtype=torch.int32, device=self.dev)
        nat.check("litho_ilt_objective_totals", L.litho_ilt_objective_totals(
            raw.data_ptr(), target.data_ptr(), self.C, self.n, float(scale), float(level), float(sign), float(a),
            dfield.data_ptr(), None if signed is None else signed.data_ptr(), cpart.data_ptr(), ppart.data_ptr(),
            N_PART, self._obj_counters.data_ptr(), cost.data_ptr(), perr.data_ptr(), self.stream()))
        gbox = self.band(dfield, 2 * self.h, float(scale) / (self.n * self.n))
        return cost, gbox, signed, perr

    def image_objective_band_ok(self) -> bool:
        """Whether litho_ilt_image_objective_band serves this grid and band."""
        if getattr(self, "_imgobj_band_ok", None) is None:
            nb = C.c_size_t(0)
            st = self.L.litho_ilt_image_objective_band_workspace(self.C, self.n, 2 * self.h, 2 * self.h, C.byref(nb))
            if st not in (0, nat.LITHO_E_UNSUPPORTED):
                nat.check("litho_ilt_image_objective_band_workspace", st)
            self._imgobj_band_ok = st == 0
        return self._imgobj_band_ok

    def image_objective_ok(self) -> bool:
        """Whether litho_ilt_image_objective serves this grid and band."""
        if self._imgobj_ok is None:
            nb = C.c_size_t(0)
            st = self.L.litho_ilt_image_objective_workspace(self.C, self.n, 2 * self.h, C.byref(nb))
            if st not in (0, nat.LITHO_E_UNSUPPORTED):
                nat.check("litho_ilt_image_objective_workspace", st)
            self._imgobj_ok = st == 0
        return self._imgobj_ok

    def update_split(self, hbox, theta, m1, m2, beta, beta_next, step, b1, b2, eps, it):
        """dJ/dm from its band box -> dJ/dtheta -> Adam (theta, m1, m2 in
        place) -> the next mask; returns (its band box, the mask)."""
        g = self.synth(hbox, self.h, False)
        mask = self.torch.empty_like(theta)
        nat.check("litho_ilt_update", self.L.litho_ilt_update(
            g.data_ptr(), g.numel(), float(beta), float(beta_next), float(step), float(b1), float(b2), float(eps),
            int(it), theta.data_ptr(), m1.data_ptr(), m2.data_ptr(), mask.data_ptr(), self.stream()))
        return self.mask_box(mask), mask

    # -- elementwise ----------------------------------------------------------
    def blur(self, x, sigma_px: float):
        if sigma_px < 1e-3:
            return x
        torch, L = self.torch, self.L
        key = float(sigma_px)
        w = self._blur.get(key)
        if w is None:
            wt = gaussian_weights(sigma_px)
            w = (torch.from_numpy(wt.astype(np.float32)).to(self.dev), (wt.size - 1) // 2)
            self._blur[key] = w
        out = torch.empty_like(x)
        tmp = torch.empty_like(x)
        nat.check("litho_gaussian_blur", L.litho_gaussian_blur(
            x.data_ptr(), out.data_ptr(), tmp.data_ptr(), int(x.shape[0]), self.n, w[0].data_ptr(), w[1],
            self.stream()))
        return out

    def mask_of(self, theta, beta: float, smooth_px: float):
        f = self.blur(theta, smooth_px)
        m = self.torch.empty_like(theta)
        nat.check("litho_ilt_mask", self.L.litho_ilt_mask(f.data_ptr(), f.numel(), float(beta), m.data_ptr(),
                                                           self.stream()))
        return m

    def grad_theta(self, grad_m, mask, beta: float, smooth_px: float):
        q = self.torch.empty_like(grad_m)
        nat.check("litho_ilt_theta_grad", self.L.litho_ilt_theta_grad(
            grad_m.data_ptr(), mask.data_ptr(), grad_m.numel(), float(beta), q.data_ptr(), self.stream()))
        return self.blur(q, smooth_px)

    def objective(self, mask, target, scale, level, sigma_px, sign, steepness, weight_tv, weight_discrete,
                  want_signed=True):
        """Device _Objective: (cost (C,), grad (C,N,N), signed, perr (C,)) — all on the device."""
        torch, L = self.torch, self.L
        mbox = self.mask_box(mask)
        raw = self.image(mbox)
        fld = self.blur(raw, sigma_px)
        a = steepness / max(abs(level), 1e-12)
        dfield = torch.empty_like(raw)
        signed = torch.empty_like(raw) if want_signed else None
        cpart = torch.empty((self.C, N_PART), dtype=torch.float64, device=self.dev)
        ppart = torch.empty((self.C, N_PART), dtype=torch.int32, device=self.dev)
        nat.check("litho_ilt_objective", L.litho_ilt_objective(
            fld.data_ptr(), target.data_ptr(), self.C, self.n, float(scale), float(level), float(sign), float(a),
            dfield.data_ptr(), None if signed is None else signed.data_ptr(), cpart.data_ptr(), ppart.data_ptr(),
            N_PART, self.stream()))
        dint = self.blur(dfield, sigma_px)
        grad = self.adjoint(dint, scale=float(scale), mbox=mbox)
        npix = float(self.n * self.n)
        cost = cpart.sum(dim=1) / npix
        if weight_tv > 0.0 or weight_discrete > 0.0:
            pc = torch.empty((self.C, N_PART), dtype=torch.float64, device=self.dev)
            nat.check("litho_ilt_penalties", L.litho_ilt_penalties(
                mask.data_ptr(), self.C, self.n, float(weight_tv), float(weight_discrete), grad.data_ptr(),
                pc.data_ptr(), N_PART, self.stream()))
            cost = cost + pc.sum(dim=1)
        return cost, grad, signed, ppart.sum(dim=1)


class _PlainStages(_Stages):
    """The same objective through the plain full-grid SOCS forward and
    adjoint (one 2-D FFT per kernel and direction), for comparison."""

    def __init__(self, kernels: SOCSKernels, n_clips: int):
        super().__init__(kernels, n_clips, use_tcc=False)
        torch = self.torch
        self.phi = kernels._phi.to(torch.complex64).contiguous()
        self.lam = (C.c_float * len(kernels))(*[float(x) for x in kernels.weights])
        self.bkx = torch.from_numpy(kernels.band_kx).to(self.dev)
        self.bky = torch.from_numpy(kernels.band_ky).to(self.dev)
        self._fields = None

    def _pws(self):
        nb = C.c_size_t(0)
        nat.check("litho_plain_socs_workspace", self.L.litho_plain_socs_workspace(self.C, self.n, C.byref(nb)))
        return self.ws("plain", nb.value)

    def objective(self, mask, target, scale, level, sigma_px, sign, steepness, weight_tv, weight_discrete,
                  want_signed=True):
        torch, L = self.torch, self.L
        K = len(self.k)
        if self._fields is None:
            self._fields = torch.empty((K, self.C, self.n, self.n), dtype=torch.complex64, device=self.dev)
        raw = torch.empty((self.C, self.n, self.n), dtype=torch.float32, device=self.dev)
        ws = self._pws()
        nat.check("litho_plain_socs_forward", L.litho_plain_socs_forward(
            mask.data_ptr(), self.C, self.n, K, self.phi.data_ptr(), self.lam, self.bkx.data_ptr(),
            self.bky.data_ptr(), self.phi.shape[1], self._fields.data_ptr(), raw.data_ptr(), ws.data_ptr(),
            ws.numel(), self.stream()))
        fld = self.blur(raw, sigma_px)
        a = steepness / max(abs(level), 1e-12)
        dfield = torch.empty_like(raw)
        signed = torch.empty_like(raw) if want_signed else None
        cpart = torch.empty((self.C, N_PART), dtype=torch.float64, device=self.dev)
        ppart = torch.empty((self.C, N_PART), dtype=torch.int32, device=self.dev)
        nat.check("litho_ilt_objective", L.litho_ilt_objective(
            fld.data_ptr(), target.data_ptr(), self.C, self.n, float(scale), float(level), float(sign), float(a),
            dfield.data_ptr(), None if signed is None else signed.data_ptr(), cpart.data_ptr(), ppart.data_ptr(),
            N_PART, self.stream()))
        sens = self.blur(dfield, sigma_px) * float(scale)
        grad = torch.empty_like(raw)
        nat.check("litho_plain_socs_adjoint", L.litho_plain_socs_adjoint(
            self._fields.data_ptr(), sens.data_ptr(), self.C, self.n, K, self.phi.data_ptr(), self.lam,
            self.bkx.data_ptr(), self.bky.data_ptr(), self.phi.shape[1], grad.data_ptr(), ws.data_ptr(),
            ws.numel(), self.stream()))
        cost = cpart.sum(dim=1) / float(self.n * self.n)
        if weight_tv > 0.0 or weight_discrete > 0.0:
            pc = torch.empty((self.C, N_PART), dtype=torch.float64, device=self.dev)
            nat.check("litho_ilt_penalties", L.litho_ilt_penalties(
                mask.data_ptr(), self.C, self.n, float(weight_tv), float(weight_discrete), grad.data_ptr(),
                pc.data_ptr(), N_PART, self.stream()))
            cost = cost + pc.sum(dim=1)
        return cost, grad, signed, ppart.sum(dim=1)


_STAGES: dict = {}


def stages(kernels: SOCSKernels, n_clips: int, engine: str = "fused") -> _Stages:
    key = (id(kernels), int(n_clips), engine)
    st = _STAGES.get(key)
    if st is None or st.k is not kernels:
        if len(_STAGES) > 16:
            _STAGES.clear()
        # the band-limited stages cover kernel bands up to 15 bins on chip (a
        # 64-point coarse grid) and wider ones on coarse grids of 128..1024
        # points; bands wider than that run both directions on the full grid
        if engine not in ("fused", "coarse", "plain"):
            raise ValueError(f"engine must be 'fused', 'coarse' or 'plain', got {engine!r}")
        fused = engine != "plain" and band_limited_ok(int(kernels.grid.n_pixels), kernels.halfwidth)
        st = _Stages(kernels, n_clips, use_tcc=engine == "fused") if fused else _PlainStages(kernels, n_clips)
        _STAGES[key] = st
    return st


# ---------------------------------------------------------------------------
# drop-in functions
# ---------------------------------------------------------------------------


class SocsFields(np.ndarray):
    """The (K, N, N) complex fields of :func:`socs_fields`; also carries the
    mask's band spectrum so :func:`socs_gradient` needs no second transform."""

    def __array_finalize__(self, obj):
        self._mbox = getattr(obj, "_mbox", None)
        self._kernels = getattr(obj, "_kernels", None)


def _check_mask(kernels, mask):
    n = int(kernels.grid.n_pixels)
    if tuple(np.shape(mask)) != (n, n):
        raise ValueError(f"mask must be {(n, n)} for these kernels, got {tuple(np.shape(mask))}")


def socs_fields(kernels: SOCSKernels, mask):
    """(fields (K, N, N) complex128, intensity (N, N) float64) — opc/ilt.py:208-232."""
    _check_mask(kernels, mask)
    st = stages(kernels, 1)
    torch = st.torch
    md = _as_device_masks(torch, mask, st.n)
    mbox = st.mask_box(md)
    inten = st.image(mbox)[0]
    f = st.fields(mbox)[0]
    if _is_torch(mask):
        return f, inten
    st.check_status()
    out = f.cpu().numpy().astype(np.complex128).view(SocsFields)
    out._mbox = mbox
    out._kernels = kernels
    return out, inten.cpu().numpy().astype(np.float64)


def socs_gradient(kernels: SOCSKernels, fields, sensitivity):
    """d/dm of sum_x sensitivity(x) I(x), (N, N) float64 — opc/ilt.py:235-266."""
    st = stages(kernels, 1)
    torch = st.torch
    g = _as_device_masks(torch, np.asarray(sensitivity, dtype=np.float64) if not _is_torch(sensitivity)
                         else sensitivity, st.n)
    mbox = getattr(fields, "_mbox", None)
    if mbox is not None and getattr(fields, "_kernels", None) is kernels:
        grad = st.adjoint(g, mbox=mbox)[0]
    else:
        fl = fields if _is_torch(fields) else torch.from_numpy(np.asarray(fields).astype(np.complex64)).to(st.dev)
        if st.h > KERNEL_HMAX_FUSED:
            # wide kernel bands: the coarse-grid adjoint recomputes the fields from
            # the mask, which these fields do not come with; use them directly
            grad = _plain_adjoint(stages(kernels, 1, "plain"), fl.reshape(-1, 1, st.n, st.n).contiguous(), g)[0]
            return grad if _is_torch(sensitivity) else grad.cpu().numpy().astype(np.float64)
        fb = st.band(fl.reshape(-1, st.n, st.n).contiguous(), st.h, 1.0 / (st.n * st.n))
        grad = st.adjoint(g, field_boxes=fb)[0]
    if _is_torch(sensitivity):
        return grad
    st.check_status()
    return grad.cpu().numpy().astype(np.float64)


def _plain_adjoint(pst, fields, sens):
    """Full-grid SOCS adjoint of given fields (K, C, N, N) complex64: (C, N, N)."""
    torch, L = pst.torch, pst.L
    grad = torch.empty(sens.shape, dtype=torch.float32, device=pst.dev)
    ws = pst._pws()
    nat.check("litho_plain_socs_adjoint", L.litho_plain_socs_adjoint(
        fields.data_ptr(), sens.data_ptr(), pst.C, pst.n, len(pst.k), pst.phi.data_ptr(), pst.lam,
        pst.bkx.data_ptr(), pst.bky.data_ptr(), pst.phi.shape[1], grad.data_ptr(), ws.data_ptr(), ws.numel(),
        pst.stream()))
    return grad


@dataclass
class Objective:
    """The cost, its gradient and the signed field in one pass (opc/ilt.py:292-360)."""

    kernels: SOCSKernels
    target: np.ndarray
    scale: float
    level: float
    sigma_px: float
    sign: float
    steepness: float
    weight_tv: float = 0.0
    weight_discrete: float = 0.0

    def __call__(self, mask):
        st = stages(self.kernels, 1)
        torch = st.torch
        md = _as_device_masks(torch, mask, st.n)
        tg = _as_device_masks(torch, self.target, st.n)
        cost, grad, signed, perr = st.objective(md, tg, self.scale, self.level, self.sigma_px, self.sign,
                                                self.steepness, self.weight_tv, self.weight_discrete)
        st.check_status()
        if _is_torch(mask):
            return float(cost[0]), grad[0], signed[0], int(perr[0])
        return (float(cost[0]), grad[0].cpu().numpy().astype(np.float64),
                signed[0].cpu().numpy().astype(np.float64), int(perr[0]))


def mask_of(theta, beta: float, smooth_px: float, kernels: SOCSKernels | None = None, grid=None):
    """sigma(beta G(theta)) on the device (opc/ilt.py:368-378)."""
    torch = nat.require_cuda()
    th = _as_device_masks(torch, theta, int(np.shape(theta)[-1]))
    n = int(th.shape[-1])
    st = _ElementwiseStages(n, th.device)
    m = st.mask_of(th, beta, smooth_px)
    return m[0] if _is_torch(theta) else m[0].cpu().numpy().astype(np.float64)


def grad_theta(grad_mask, mask, beta: float, smooth_px: float):
    """dJ/dtheta from dJ/dm (opc/ilt.py:381-389)."""
    torch = nat.require_cuda()
    n = int(np.shape(mask)[-1])
    gm = _as_device_masks(torch, grad_mask, n)
    mk = _as_device_masks(torch, mask, n)
    st = _ElementwiseStages(n, gm.device)
    q = st.grad_theta(gm, mk, beta, smooth_px)
    return q[0] if _is_torch(grad_mask) else q[0].cpu().numpy().astype(np.float64)


class _ElementwiseStages(_Stages):
    """The elementwise and blur stages, without kernels."""

    def __init__(self, n: int, dev):  # noqa: D401 - deliberately not calling super
        self.torch = nat.require_cuda()
        self.L = nat.lib()
        self.n = n
        self.dev = dev
        self._ws = {}
        self._blur = {}


# ---------------------------------------------------------------------------
# autograd
# ---------------------------------------------------------------------------


def _socs_image_function():
    import torch

    class SocsImage(torch.autograd.Function):
        """Raw SOCS intensity of a batch of masks; backward is the adjoint.

        forward(masks (C, N, N) float32 CUDA, kernels) -> (C, N, N) float32;
        backward(dL/dI) -> dL/dmasks (opc/ilt.py:262-266 for every clip)."""

        @staticmethod
        def forward(ctx, masks, kernels):
            st = stages(kernels, int(masks.shape[0]))
            mbox = st.mask_box(masks.contiguous())
            ctx.st = st
            ctx.save_for_backward(mbox)
            return st.image(mbox)

        @staticmethod
        def backward(ctx, grad_out):
            (mbox,) = ctx.saved_tensors
            g = ctx.st.adjoint(grad_out.contiguous().to(torch.float32), mbox=mbox)
            return g, None

    return SocsImage


_SOCS_IMAGE = None


def socs_image(masks, kernels: SOCSKernels):
    """Differentiable SOCS intensity (``torch.autograd.Function``)."""
    global _SOCS_IMAGE
    if _SOCS_IMAGE is None:
        _SOCS_IMAGE = _socs_image_function()
    return _SOCS_IMAGE.apply(masks, kernels)


def __getattr__(name):
    if name == "SocsImage":
        global _SOCS_IMAGE
        if _SOCS_IMAGE is None:
            _SOCS_IMAGE = _socs_image_function()
        return _SOCS_IMAGE
    raise AttributeError(name)


# ---------------------------------------------------------------------------
# fused batched iteration and the solve loop
# ---------------------------------------------------------------------------


@dataclass
class IltParams:
    """The objective and optimiser settings of a solve (opc/ilt.py:397-576)."""

    scale: float
    level: float
    sign: float = 1.0
    sigma_px: float = 0.0
    steepness: float = 12.0
    weight_tv: float = 0.0
    weight_discrete: float = 0.0
    smooth_px: float = 0.0
    step: float = 0.4
    beta: float = 4.0
    growth: float = 1.0
    b1: float = 0.9
    b2: float = 0.999
    eps: float = 1e-8


def default_lanes(n_clips: int) -> int:
    """Parallel clip groups of a graph-replayed fast step: two once a group
    still has 4 clips to keep its pixel passes wide."""
    return 2 if n_clips >= 8 else 1


def _lane_ranges(n_clips: int, lanes: int):
    base, extra = divmod(n_clips, lanes)
    out, a = [], 0
    for r in range(lanes):
        b = a + base + (1 if r < extra else 0)
        out.append((a, b))
        a = b
    return out


class IltBatch:
    """A batch of ILT solves advanced together on the device.

    state: theta, Adam moments (float32), the current mask and gradient.
    ``step()`` is one iteration of opc/ilt.py:576-596: grad_theta, Adam, the
    beta anneal, mask_of and the objective (SOCS forward + adjoint).

    Without blurs, smoothing or penalties (the common ILT setting) the step
    keeps the gradient as its band box between steps and does dJ/dtheta,
    Adam and the next mask in one pixel pass (``fast``); ``grad_m`` is then
    synthesised on demand. ``fast=False`` forces the stage-by-stage path."""

    def __init__(self, kernels: SOCSKernels, targets, theta0, params: IltParams, engine: str = "fused",
                 fast: bool | None = None, lanes: int | None = None):
        self.st = stages(kernels, int(theta0.shape[0]), engine)
        C = int(theta0.shape[0])
        #: clip groups the graph-replayed fast step runs on parallel branches
        self.lanes = max(1, min(C, int(lanes) if lanes is not None else default_lanes(C)))
        torch = self.st.torch
        n = self.st.n
        self.p = params
        self.target = _as_device_masks(torch, targets, n)
        self.theta = _as_device_masks(torch, theta0, n).clone()
        self.m1 = torch.zeros_like(self.theta)
        self.m2 = torch.zeros_like(self.theta)
        self.beta = float(params.beta)
        self.it = 0
        can = type(self.st) is _Stages and self.st.fast_ok(params)
        self.fast = can if fast is None else (bool(fast) and can)
        self._mask = self.st.mask_of(self.theta, self.beta, params.smooth_px)
        self._grad_m = None
        self._graph = None
        if self.fast:
            self.mbox = self.st.mask_box(self._mask)
            self.cost, self.hbox, self.signed, self.perr = self._objective_fast(True)
        else:
            self.cost, self._grad_m, self.signed, self.perr = self._objective(self._mask)

    def _objective(self, mask, want_signed=True):
        p = self.p
        return self.st.objective(mask, self.target, p.scale, p.level, p.sigma_px, p.sign, p.steepness,
                                 p.weight_tv, p.weight_discrete, want_signed=want_signed)

    def _objective_fast(self, want_signed):
        p = self.p
        return self.st.objective_split(self.mbox, self.target, p.scale, p.level, p.sign, p.steepness, want_signed)

    def check_status(self) -> None:
        """Synchronise and raise ``LithoError`` if a bounded device wait gave
        up in the latest step (its results are then invalid)."""
        for st in getattr(self, "_lane_st", None) or [self.st]:
            st.check_status()

    @property
    def mask(self):
        if self._mask is None:
            self._mask = self.st.mask_of(self.theta, self.beta, self.p.smooth_px)
        return self._mask

    @property
    def grad_m(self):
        if self._grad_m is None:
            self._grad_m = self.st.synth(self.hbox, self.st.h, False)
        return self._grad_m

    def run(self, n_steps: int, graph: bool = True):
        """``n_steps`` steps without the signed field; returns the last cost.

        The fast step is recorded once as a CUDA graph (its beta annealing and
        Adam counter kept in device memory, ``litho_ilt_update_sched``) and
        replayed, which removes the launch gaps between its ~15 kernels; the
        results are those of ``step()``. Other configurations step eagerly."""
        n_steps = int(n_steps)
        if n_steps <= 0:
            return self.cost
        if not (self.fast and graph):
            for _ in range(n_steps):
                self.step(want_signed=False)
            return self.cost
        if self._graph is None:
            if self.it == 0:          # the first step allocates the stages' workspaces
                self.step(want_signed=False)
                n_steps -= 1
            self._capture()
        for _ in range(n_steps):
            self._graph.replay()
            self.it += 1
            self.beta = self.beta * self.p.growth
        self.signed = None
        return self.cost

    def _capture(self):
        """Record one fast step as a CUDA graph. The clips are split into
        ``self.lanes`` groups, each with its own stages (workspaces) and step
        schedule, recorded on parallel branches of the graph: a lane's
        latency-bound coarse-grid kernels then overlap another lane's
        pixel passes. Clips are independent, so the results are those of one
        lane; every kernel's arithmetic is per clip."""
        torch = self.st.torch
        p = self.p
        C = int(self.theta.shape[0])
        ranges = [(a, b) for a, b in _lane_ranges(C, self.lanes) if b > a]
        sched = np.zeros(1, dtype=nat.ILT_SCHED_DTYPE)
        sched["beta"] = sched["beta_next"] = self.beta
        sched["growth"] = p.growth
        sched["it"] = self.it
        self._sched = [torch.from_numpy(sched.view(np.uint8).copy()).to(self.st.dev) for _ in ranges]
        hbox = torch.empty_like(self.hbox)
        hbox.copy_(self.hbox)
        self.hbox = hbox
        lane_st = [self.st] if len(ranges) == 1 else [_Stages(self.st.k, b - a, use_tcc=self.st.tcc is not None)
                                                      for a, b in ranges]
        mask = torch.empty_like(self.theta)
        mbox = torch.empty((C, self.st.side * self.st.side), dtype=torch.complex64, device=self.st.dev)
        cost = torch.empty((C,), dtype=torch.float64, device=self.st.dev)
        perr = torch.empty((C,), dtype=torch.int64, device=self.st.dev)
        if len(ranges) > 1:
            # the lanes' first calls size their workspaces outside the capture
            for st, (a, b) in zip(lane_st, ranges):
                mb = st.mask_box(self._mask[a:b])
                st.objective_split(mb, self.target[a:b], p.scale, p.level, p.sign, p.steepness, want_signed=False)
                st.synth(self.hbox[a:b], st.h, False)
        torch.cuda.synchronize(self.st.dev)
        streams = [torch.cuda.Stream(device=self.st.dev) for _ in ranges]
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            main = torch.cuda.current_stream(self.st.dev)
            for s in streams:
                s.wait_stream(main)
            for st, s, sch, (a, b) in zip(lane_st, streams, self._sched, ranges):
                with torch.cuda.stream(s):
                    grad = st.synth(self.hbox[a:b], st.h, False)
                    nat.check("litho_ilt_update_sched", st.L.litho_ilt_update_sched(
                        grad.data_ptr(), grad.numel(), sch.data_ptr(), float(p.step), float(p.b1), float(p.b2),
                        float(p.eps), self.theta[a:b].data_ptr(), self.m1[a:b].data_ptr(), self.m2[a:b].data_ptr(),
                        mask[a:b].data_ptr(), st.stream()))
                    st.mask_box(mask[a:b], out=mbox[a:b])
                    st.objective_split(mbox[a:b], self.target[a:b], p.scale, p.level, p.sign, p.steepness,
                                       want_signed=False, out_hbox=self.hbox[a:b], out_cost=cost[a:b],
                                       out_perr=perr[a:b])
            for s in streams:
                main.wait_stream(s)
        self._graph = g
        self._lane_st = lane_st
        self._mask, self.mbox, self.cost, self.perr = mask, mbox, cost, perr
        self._grad_m = None

    def step(self, want_signed: bool = True):
        if self._graph is not None:
            raise RuntimeError("this batch steps by graph replay (run()); make a new IltBatch to step eagerly")
        p = self.p
        self.it += 1
        if self.fast:
            beta_next = self.beta * p.growth
            self.mbox, self._mask = self.st.update_split(self.hbox, self.theta, self.m1, self.m2, self.beta,
                                                         beta_next, p.step, p.b1, p.b2, p.eps, self.it)
            self.beta = beta_next
            self._grad_m = None
            self.cost, self.hbox, self.signed, self.perr = self._objective_fast(want_signed)
            return self.cost
        gt = self.st.grad_theta(self.grad_m, self.mask, self.beta, p.smooth_px)
        nat.check("litho_ilt_adam", self.st.L.litho_ilt_adam(
            gt.data_ptr(), gt.numel(), float(p.step), float(p.b1), float(p.b2), float(p.eps), self.it,
            self.theta.data_ptr(), self.m1.data_ptr(), self.m2.data_ptr(), self.st.stream()))
        self.beta *= p.growth
        self._mask = self.st.mask_of(self.theta, self.beta, p.smooth_px)
        self.cost, self._grad_m, self.signed, self.perr = self._objective(self._mask, want_signed)
        return self.cost


@dataclass
class ILTResult:
    mask: np.ndarray
    theta: np.ndarray
    target: np.ndarray
    history: list = field(default_factory=list)
    iterations: int = 0
    converged: bool = False


def run_ilt(target, kernels: SOCSKernels, *, level: float, dose: float = 1.0, sign: float = 1.0,
            diffusion_sigma: float = 0.0, initial=None, max_iter: int = 120, step: float = 0.4, tol: float = 1e-7,
            beta: float = 4.0, beta_final: float | None = 12.0, initial_grey: float = 0.9, steepness: float = 12.0,
            weight_tv: float = 0.0, weight_discrete: float = 0.0, smooth: float = 0.0, progress=None) -> ILTResult:
    """Solve for the mask that prints ``target`` (opc/ilt.py:run_ilt, :397-621).

    The print model is given by its parts: SOCS ``kernels`` (whose optics set
    the normalisation, which must not be 'peak'), resist ``level`` and
    ``diffusion_sigma`` [m], ``dose``, and ``sign`` (+1 clear tone, -1 dark)."""
    v = optics_view(kernels.optics)
    if v.normalisation.lower() == "peak":
        raise ValueError("inverse lithography needs a mask-independent normalisation; 'peak' rescales the "
                         "image by whatever the current mask's brightest point happens to be, which moves the "
                         "objective every step. Use normalisation='clear'.")
    n = int(kernels.grid.n_pixels)
    tgt = np.asarray(target, dtype=np.float64)
    if tgt.shape != (n, n):
        raise ValueError(f"target must be {(n, n)} for this grid, got {tgt.shape}")
    if smooth < 0.0:
        raise ValueError(f"smooth is a length and cannot be negative, got {smooth:g}")
    px = float(kernels.grid.pixel_size)
    smooth_px = float(smooth / px)
    scale = normalisation_scale(v.normalisation, 1.0, kernels.clear, dose)
    p = float(np.clip(initial_grey, 0.5 + 1e-3, 1.0 - 1e-6))
    m0 = 0.5 + (np.clip(tgt, 0.0, 1.0) - 0.5) * (2.0 * p - 1.0) if initial is None else \
        np.clip(np.asarray(initial, dtype=np.float64), 1.0 - p, p)
    theta0 = np.log(m0 / (1.0 - m0)) / beta
    growth = 1.0 if beta_final is None or max_iter <= 1 else (beta_final / beta) ** (1.0 / (max_iter - 1))
    params = IltParams(scale=scale, level=level, sign=sign, sigma_px=float(diffusion_sigma / px),
                       steepness=steepness, weight_tv=weight_tv, weight_discrete=weight_discrete,
                       smooth_px=smooth_px, step=step, beta=beta, growth=growth)
    b = IltBatch(kernels, tgt[None], theta0[None], params)
    b.check_status()
    lit = int((b.signed > 0).sum())
    if lit == 0 or lit == n * n:
        raise ValueError(f"the initial mask prints {'nothing' if lit == 0 else 'everywhere'} — no contour "
                         f"exists, so the objective has no gradient. Size the dose first.")
    hist = [{"iteration": 0, "cost": float(b.cost[0]), "pattern_error": int(b.perr[0]), "beta": b.beta,
             "grad_norm": float(b.grad_m.double().norm())}]
    if progress is not None:
        progress({"iteration": 0, "mask": b.mask[0].cpu().numpy(), "signed": b.signed[0].cpu().numpy()})
    prev, converged, taken = np.inf, False, 0
    for it in range(1, max_iter + 1):
        b.step()
        taken = it
        b.check_status()
        cost = float(b.cost[0])
        hist.append({"iteration": it, "cost": cost, "pattern_error": int(b.perr[0]), "beta": b.beta,
                     "grad_norm": float(b.grad_m.double().norm())})
        if progress is not None:
            progress({"iteration": it, "mask": b.mask[0].cpu().numpy(), "signed": b.signed[0].cpu().numpy()})
        if abs(prev - cost) < tol:
            converged = True
            break
        prev = cost
    return ILTResult(mask=b.mask[0].cpu().numpy().astype(np.float64),
                     theta=b.theta[0].cpu().numpy().astype(np.float64), target=tgt > 0.5, history=hist,
                     iterations=taken, converged=converged)


__all__ = ["Objective", "IltBatch", "IltParams", "ILTResult", "SocsFields", "gaussian_weights", "grad_theta",
           "mask_of", "run_ilt", "socs_fields", "socs_gradient", "socs_image"]
