"""Uneven batches: clips of several sizes imaged by one CUDA-graph replay,
and ILT over clips of several sizes.

The reference images clips one call at a time, whatever their size
(expose/aerial_image.py:502-548). Here the clips of a batch are grouped by
grid size; every group gets its own plan, pupil table, static input/output
buffers and workspace, the launch sequences of all groups are captured once
in a CUDA graph, and each batch is one replay. The work-item size of every
group (source points per thread block, the unit the coarse kernels
schedule) is picked by timing the candidates on the group's own clips the
first time a (grid, pupil width, clip count) combination is seen.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as nat
from .aerial import coarse_grid, disc_halfwidth, fused_supported, plan_abbe, pupil_table
from .config import optics_view

#: candidates for jobs (source points x states) per work item: on-chip coarse
#: grids (L <= 64), and the wide-pupil engine (one L x L partial per item)
ITEM_CANDIDATES = (2, 4, 8, 16, 32)
WIDE_ITEM_CANDIDATES = (8, 16, 32)
_TUNED: dict = {}


@dataclass
class _Group:
    n: int
    index: list            # positions of this group's clips in the batch
    pd: object
    masks: object          # (C, N, N) static device input
    image: object          # (C, N, N) static device output
    peak: object
    ws: object
    table: object
    items: int


def _run_group(torch, L, g: _Group, stream: int) -> None:
    nat.check("litho_abbe_tabled", L.litho_abbe_tabled(
        C.byref(g.pd.plan), g.pd._blob_dev.data_ptr(), g.table.data_ptr(), g.masks.data_ptr(), g.image.data_ptr(),
        g.peak.data_ptr(), g.ws.data_ptr(), g.ws.numel(), stream))


class UnevenAbbe:
    """Abbe images of a batch of clips of mixed sizes (one optics, one pixel size).

    sizes: the grid side of every clip, in batch order. ``__call__`` takes the
    masks (a list of (N_i, N_i) device tensors or arrays) and returns the
    images as a list of (N_i, N_i) float32 device tensors (views of the
    group's output buffer, overwritten by the next call)."""

    def __init__(self, sizes, optics, pixel_size: float, *, mask_complex: bool = False, dose: float = 1.0,
                 return_raw: bool = False, graph: bool = True, tune: bool = True, device=None):
        torch = nat.require_cuda()
        self.torch, self.L = torch, nat.lib()
        self.dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.sizes = [int(n) for n in sizes]
        self.view = optics_view(optics)
        self.px = float(pixel_size)
        self.complex = bool(mask_complex)
        self.dose, self.return_raw = float(dose), bool(return_raw)
        by_n: dict = {}
        for i, n in enumerate(self.sizes):
            by_n.setdefault(n, []).append(i)
        dt = torch.complex64 if self.complex else torch.float32
        self.groups = []
        for n in sorted(by_n):
            idx = by_n[n]
            masks = torch.zeros((len(idx), n, n), dtype=dt, device=self.dev)
            self.groups.append(self._group(n, idx, masks, 8))
        self.tuned = {}
        if tune:
            self._tune()
        self.graph = None
        if graph:
            self._capture()

    # ------------------------------------------------------------------
    def _group(self, n, idx, masks, items) -> _Group:
        torch, L = self.torch, self.L
        v = self.view
        pd = plan_abbe([v] * len(idx), n, self.px, [[(v.defocus, v.image_index)]] * len(idx), self.dose,
                       self.return_raw, self.complex, items_per_job_group=items)
        if not fused_supported(n, int(pd.plan.L)):
            raise NotImplementedError(f"{n}^2 clips need the full-grid engine, which this batch runner does not "
                                      "capture; image them with compute_aerial_batch")
        pd._blob_dev = torch.from_numpy(pd.blob).to(self.dev)
        s = nat.stream_ptr(torch, self.dev)
        table = pupil_table(pd, self.dev, s)
        nb = C.c_size_t(0)
        nat.check("litho_abbe_workspace", L.litho_abbe_workspace(C.byref(pd.plan), C.byref(nb)))
        ws = torch.empty(max(nb.value, 256), dtype=torch.uint8, device=self.dev)
        image = torch.empty((len(idx), n, n), dtype=torch.float32, device=self.dev)
        peak = torch.empty((len(idx),), dtype=torch.float32, device=self.dev)
        return _Group(n, idx, pd, masks, image, peak, ws, table, items)

    def _tune(self) -> None:
        """Per group, time each work-item size on the group's clips (two runs
        after one warm-up, CUDA events) and keep the fastest."""
        torch = self.torch
        for k, g in enumerate(self.groups):
            h = disc_halfwidth(self.view.NA, self.view.wavelength, g.n, self.px)[1]
            key = (g.n, h, coarse_grid(h), len(g.index), repr(self.view))
            best = _TUNED.get(key)
            if best is None:
                times = {}
                for items in (ITEM_CANDIDATES if coarse_grid(h) <= 64 else WIDE_ITEM_CANDIDATES):
                    cand = self._group(g.n, g.index, g.masks, items)
                    s = nat.stream_ptr(torch, self.dev)
                    _run_group(torch, self.L, cand, s)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    for _ in range(2):
                        _run_group(torch, self.L, cand, s)
                    e1.record()
                    torch.cuda.synchronize()
                    times[items] = e0.elapsed_time(e1) / 2
                    del cand
                best = min(times, key=times.get)
                _TUNED[key] = best
                self.tuned[g.n] = {"items_per_block": best, "ms": times}
            else:
                self.tuned[g.n] = {"items_per_block": best}
            if best != g.items:
                self.groups[k] = self._group(g.n, g.index, g.masks, best)

    def _launch_all(self) -> None:
        s = nat.stream_ptr(self.torch, self.dev)
        for g in self.groups:
            _run_group(self.torch, self.L, g, s)

    def _capture(self) -> None:
        torch = self.torch
        self._launch_all()                       # first launches (lazy set-up) outside the capture
        torch.cuda.synchronize()
        side = torch.cuda.Stream(device=self.dev)
        side.wait_stream(torch.cuda.current_stream(self.dev))
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=side):
            self._launch_all()
        torch.cuda.synchronize()

    # ------------------------------------------------------------------
    def load(self, masks) -> None:
        """Copy the batch's masks into the groups' input buffers."""
        torch = self.torch
        if len(masks) != len(self.sizes):
            raise ValueError(f"expected {len(self.sizes)} masks, got {len(masks)}")
        for g in self.groups:
            for j, i in enumerate(g.index):
                m = masks[i]
                t = m if isinstance(m, torch.Tensor) else torch.from_numpy(np.asarray(m))
                if tuple(t.shape) != (g.n, g.n):
                    raise ValueError(f"mask {i} must be {(g.n, g.n)}, got {tuple(t.shape)}")
                g.masks[j].copy_(t.to(g.masks.dtype), non_blocking=True)

    def run(self) -> None:
        """Image the loaded masks (one graph replay, or the launches in order)."""
        if self.graph is not None:
            self.graph.replay()
        else:
            self._launch_all()

    def __call__(self, masks):
        self.load(masks)
        self.run()
        out = [None] * len(self.sizes)
        for g in self.groups:
            for j, i in enumerate(g.index):
                out[i] = g.image[j]
        return out

    def check_status(self) -> None:
        """Synchronise and raise ``LithoError`` if a bounded device wait gave
        up in the latest run of any size group (its images are then invalid)."""
        self.torch.cuda.synchronize(self.dev)
        for g in self.groups:
            st = int(g.ws[:4].view(self.torch.int32).item())
            if st:
                nat.check("litho_abbe_tabled", st)

    def peaks(self):
        out = [None] * len(self.sizes)
        for g in self.groups:
            for j, i in enumerate(g.index):
                out[i] = g.peak[j]
        return out


class UnevenIlt:
    """ILT of a batch of clips of mixed sizes (one optics, one pixel size):
    the clips are grouped by grid size, each group has its own SOCS kernels
    (built once, on the device) and is stepped as one ``IltBatch``.

    targets, theta0: lists of (N_i, N_i) arrays or device tensors, in batch
    order. params(kernels) -> IltParams for a group (its normalisation scale
    depends on the group's kernels)."""

    def __init__(self, targets, theta0, optics, pixel_size: float, params, *, max_kernels: int | None = 24,
                 tol: float = 0.0):
        from .config import GridConfig
        from .hopkins import SOCSKernels
        from .ilt import IltBatch
        torch = nat.require_cuda()
        self.torch = torch
        if len(targets) != len(theta0):
            raise ValueError(f"{len(targets)} targets for {len(theta0)} initial fields")
        self.sizes = [int(np.shape(t)[-1]) for t in targets]
        by_n: dict = {}
        for i, n in enumerate(self.sizes):
            by_n.setdefault(n, []).append(i)
        self.groups = []
        for n in sorted(by_n):
            idx = by_n[n]
            k = SOCSKernels.build(optics, GridConfig(n_pixels=n, pixel_size=pixel_size), tol=tol,
                                  max_kernels=max_kernels)

            def stack(xs):
                ts = [x if isinstance(x, torch.Tensor) else torch.from_numpy(np.asarray(x, dtype=np.float32))
                      for x in xs]
                return torch.stack([t.to(torch.float32).cuda() for t in ts])
            b = IltBatch(k, stack([targets[i] for i in idx]), stack([theta0[i] for i in idx]), params(k))
            self.groups.append((n, idx, k, b))

    def step(self, want_signed: bool = False):
        """One ILT iteration of every clip; returns the costs in batch order (device)."""
        cost = [None] * len(self.sizes)
        for _n, idx, _k, b in self.groups:
            c = b.step(want_signed=want_signed)
            for j, i in enumerate(idx):
                cost[i] = c[j]
        return cost

    def theta(self):
        out = [None] * len(self.sizes)
        for _n, idx, _k, b in self.groups:
            for j, i in enumerate(idx):
                out[i] = b.theta[j]
        return out


def compute_aerial_uneven(masks, optics, pixel_size: float, dose: float = 1.0, return_raw: bool = False):
    """Images of clips of mixed sizes in one call (one CUDA-graph replay);
    numpy in -> list of numpy float64 out, torch in -> list of torch float32."""
    torch = nat.require_cuda()
    is_t = [isinstance(m, torch.Tensor) for m in masks]
    cplx = any((m.is_complex() if isinstance(m, torch.Tensor) else np.iscomplexobj(m)) for m in masks)
    run = UnevenAbbe([int(np.shape(m)[-1]) for m in masks], optics, pixel_size, mask_complex=cplx, dose=dose,
                     return_raw=return_raw, graph=True, tune=False)
    imgs = run(masks)
    return [im.clone() if t else im.cpu().numpy().astype(np.float64) for im, t in zip(imgs, is_t)]


__all__ = ["UnevenAbbe", "UnevenIlt", "compute_aerial_uneven", "ITEM_CANDIDATES"]
