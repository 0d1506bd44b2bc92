"""Imaging over several GPUs: one process per GPU.

Three ways to spread the work, by what the workload has many of:

* Many clips (the batched workloads): clips are sharded, each rank images its
  own, and only results travel. ``shard_plan`` balances ranks by cost (pixels
  x coherent systems, so uneven clip sizes spread evenly), deterministically,
  so every rank computes the same plan without communicating;
  ``gather_tensors`` reassembles the outputs in input order with tensor
  all-gathers (NCCL on the GPU, gloo on the CPU).
* One large image: its source points are split over ranks
  (``source_ranges``). The Abbe sum is linear in the source set
  (expose/aerial_image.py:421-486 loops over source points and adds), so each
  rank sums its share into the image's band box ((4h+1)^2 complex values,
  30 KB at 1024^2 against 4 MB for the image), one all-reduce adds the
  shares, and every rank synthesises the image; the peak is taken after the
  reduction and the clear throughput is the full source's (host, FP64).
* One ILT clip: its SOCS kernels are split over ranks (``kernel_ranges``).
  The intensity and the adjoint are both sums over kernels
  (opc/ilt.py:227-231, :262-266), so each rank forms its kernels' part of the
  image's band box and, after the objective, its part of the gradient's band
  box; one all-reduce after each. The optimiser state is replicated: every
  rank takes the same Adam step on the same reduced gradient.

No TMA multicast is involved: the exchanged band boxes go through NCCL
all-reduces into each rank's own memory before any kernel reads them.
"""

from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def shard_plan(costs: Sequence[float], world: int) -> list[list[int]]:
    """Assign item indices to `world` ranks, largest first onto the least
    loaded rank (ties to the lower rank); each rank's list is in input order."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def clip_cost(n_pixels: int, n_systems: int = 1) -> float:
    """Relative cost of imaging one clip: its pixels times coherent systems."""
    return float(n_pixels) * float(n_pixels) * float(max(1, n_systems))


def contiguous_ranges(count: int, world: int) -> list[tuple[int, int]]:
    """Split range(count) into `world` contiguous (start, stop) ranges whose
    lengths differ by at most one (the first count % world ranks get one
    more); ranks past `count` get empty ranges."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    if count < 0:
        raise ValueError("count must be >= 0")
    base, extra = divmod(int(count), int(world))
    out, a = [], 0
    for r in range(world):
        b = a + base + (1 if r < extra else 0)
        out.append((a, b))
        a = b
    return out


def source_ranges(n_sources: int, world: int) -> list[tuple[int, int]]:
    """Source points of one image per rank (every point costs the same:
    one coherent system per state and field component)."""
    return contiguous_ranges(n_sources, world)


def kernel_ranges(n_kernels: int, world: int) -> list[tuple[int, int]]:
    """SOCS kernels of one clip per rank."""
    return contiguous_ranges(n_kernels, world)


def run_sharded(items: Sequence, costs: Sequence[float], fn: Callable[[list], list], rank: int, world: int):
    """Run fn on this rank's share of `items`; returns (indices, results)."""
    mine = shard_plan(costs, world)[rank]
    out = fn([items[i] for i in mine]) if mine else []
    if len(out) != len(mine):
        raise RuntimeError(f"rank {rank}: fn returned {len(out)} results for {len(mine)} items")
    return mine, list(out)


def _comm_device(group):
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def gather_tensors(n_items: int, mine: list[int], results: list, group=None) -> list:
    """All-gather every rank's (indices, tensors) and return all items'
    tensors in input order, on every rank, as tensors on the communication
    device (the current GPU for NCCL, the CPU for gloo).

    Results may differ in shape (uneven clip sizes) but share one dtype. Two
    collectives: an all-gather of each rank's sizes, then one of its
    zero-padded payload (headers + flattened values)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    dev = _comm_device(group)
    if len(mine) != len(results):
        raise ValueError(f"{len(mine)} indices for {len(results)} results")
    dtypes = {r.dtype for r in results}
    if len(dtypes) > 1:
        raise ValueError(f"results must share one dtype, got {sorted(map(str, dtypes))}")
    # header per item: index, ndim, then 4 dims (unused ones 1)
    head = torch.zeros((len(mine), 6), dtype=torch.int64)
    for j, (i, r) in enumerate(zip(mine, results)):
        if r.dim() > 4:
            raise ValueError("results of at most 4 dimensions")
        head[j, 0], head[j, 1] = int(i), r.dim()
        head[j, 2:2 + r.dim()] = torch.tensor(list(r.shape), dtype=torch.int64)
    code_of, dtype_of = _dtype_tables()
    dt = results[0].dtype if results else torch.float32
    if results and dt not in code_of:
        raise ValueError(f"unsupported result dtype {dt}")
    dts = torch.tensor([code_of[dt] if results else -1], dtype=torch.int64, device=dev)
    flat = torch.cat([r.detach().reshape(-1).to(dev) for r in results]) if results else torch.zeros(0, device=dev)
    sizes = torch.tensor([len(mine), flat.numel()], dtype=torch.int64, device=dev)
    all_sizes = [torch.zeros_like(sizes) for _ in range(world)]
    dist.all_gather(all_sizes, sizes, group=group)
    all_dts = [torch.zeros_like(dts) for _ in range(world)]
    dist.all_gather(all_dts, dts, group=group)
    codes = {int(d.item()) for d in all_dts} - {-1}
    if len(codes) > 1:
        raise ValueError("ranks returned results of different dtypes")
    if codes:
        dt = dtype_of[codes.pop()]
    max_items = max(int(s[0]) for s in all_sizes)
    max_vals = max(int(s[1]) for s in all_sizes)
    hbuf = torch.zeros((max(max_items, 1), 6), dtype=torch.int64, device=dev)
    hbuf[:len(mine)] = head.to(dev)
    vbuf = torch.zeros(max(max_vals, 1), dtype=dt, device=dev)
    vbuf[:flat.numel()] = flat.to(dt)
    hs = [torch.zeros_like(hbuf) for _ in range(world)]
    vs = [torch.zeros_like(vbuf) for _ in range(world)]
    dist.all_gather(hs, hbuf, group=group)
    real = (lambda t: torch.view_as_real(t)) if dt.is_complex else (lambda t: t)  # noqa: E731
    dist.all_gather([real(v) for v in vs], real(vbuf), group=group)
    hs = [h.cpu() for h in hs]
    full: list = [None] * n_items
    seen = 0
    for r in range(world):
        cnt = int(all_sizes[r][0])
        off = 0
        for j in range(cnt):
            i, nd = int(hs[r][j, 0]), int(hs[r][j, 1])
            shape = [int(x) for x in hs[r][j, 2:2 + nd]]
            numel = int(np.prod(shape)) if shape else 1
            if not 0 <= i < n_items or full[i] is not None:
                raise RuntimeError(f"item {i} out of range or produced by two ranks")
            full[i] = vs[r][off:off + numel].reshape(shape)
            off += numel
            seen += 1
    if seen != n_items:
        raise RuntimeError(f"gathered {seen} of {n_items} results")
    return full


def _dtype_tables():
    """dtype <-> small integer code, for agreeing on a payload dtype."""
    import torch
    code = {torch.float32: 0, torch.float64: 1, torch.complex64: 2, torch.complex128: 3, torch.int32: 4,
            torch.int64: 5, torch.uint8: 6, torch.float16: 7, torch.bfloat16: 8}
    return code, {v: k for k, v in code.items()}


def gather_results(n_items: int, mine: list[int], results: list, group=None) -> list:
    """``gather_tensors`` for results given as numpy arrays or tensors;
    returns numpy arrays when the inputs were numpy (on every rank)."""
    import torch
    as_np = all(not isinstance(r, torch.Tensor) for r in results)
    ts = [r if isinstance(r, torch.Tensor) else torch.as_tensor(np.asarray(r)) for r in results]
    full = gather_tensors(n_items, mine, ts, group)
    return [t.cpu().numpy() for t in full] if as_np else full


# ---------------------------------------------------------------------------
# one image split by source points
# ---------------------------------------------------------------------------


def _all_reduce_sum(t, group):
    import torch
    import torch.distributed as dist
    buf = torch.view_as_real(t) if t.is_complex() else t
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    return t


def split_abbe_image(partial: Callable, finish: Callable, n_sources: int, group=None):
    """The Abbe image of one clip with its source points split over the
    ranks of `group`.

    partial((start, stop)) -> this rank's share as a tensor (on the GPU: the
    image band box; ``None`` for an empty range, replaced by zeros like the
    other ranks' shares). finish(reduced) -> whatever the caller wants from
    the whole sum (on the GPU: the synthesised raw image). Every rank calls
    this with the same arguments; the result is identical on every rank."""
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    rngs = source_ranges(n_sources, world)
    a, b = rngs[rank]
    share = partial((a, b)) if b > a else None
    if share is None:
        # the shape comes from a rank with sources (rank 0 always has some)
        share = partial((0, 1)).zero_()
    return finish(_all_reduce_sum(share, group))


class GpuAbbeSplit:
    """The GPU halves of ``split_abbe_image`` for one clip and one plane:
    ``partial`` sums a range of source points into the image's band box
    (band DFT of the mask, then the coarse-grid accumulation), ``finish``
    synthesises the raw image from the reduced box; ``image`` normalises it
    as ``compute_aerial_image`` does, with the peak of the reduced image and
    the full source's clear throughput."""

    def __init__(self, mask, optics, grid, dose: float = 1.0):
        from . import _native as nat
        from .aerial import _as_device_masks, fused_supported, plan_abbe, pupil_table
        from .config import optics_view
        from .source import source_points
        self.torch = nat.require_cuda()
        self.nat, self.L = nat, nat.lib()
        self.v = optics_view(optics)
        self.n, self.px = int(grid.n_pixels), float(grid.pixel_size)
        self.dose = float(dose)
        self.mask = _as_device_masks(self.torch, mask, self.n)
        self.dev = self.mask.device
        self.plane = [(self.v.defocus, self.v.image_index)]
        self.n_sources = len(source_points(self.v))
        full = plan_abbe([self.v], self.n, self.px, [self.plane], 1.0, True, bool(self.mask.is_complex()))
        if not fused_supported(self.n, int(full.plan.L)):
            raise NotImplementedError("the source split runs on the band-limited engines")
        self.clear = float(full.clears[0])
        self.h = int(full.plan.h)
        self._plan_abbe, self._pupil_table = plan_abbe, pupil_table

    def partial(self, rng):
        import ctypes as C
        torch, nat, L = self.torch, self.nat, self.L
        pd = self._plan_abbe([self.v], self.n, self.px, [self.plane], 1.0, True, bool(self.mask.is_complex()),
                             sources=rng)
        if int(pd.plan.h) != self.h:
            raise RuntimeError("source ranges disagree on the pupil half-width")
        s = nat.stream_ptr(torch, self.dev)
        table = self._pupil_table(pd, self.dev, s)
        bm, n = int(pd.plan.bm), self.n
        nb = C.c_size_t(0)
        nat.check("litho_band_spectrum_workspace", L.litho_band_spectrum_workspace(1, n, bm, C.byref(nb)))
        ws = nat.Workspace.get(torch, self.dev, nb.value, tag="split_band")
        mb = torch.empty(((2 * bm + 1) ** 2,), dtype=torch.complex64, device=self.dev)
        nat.check("litho_band_spectrum", L.litho_band_spectrum(
            self.mask.data_ptr(), int(self.mask.is_complex()), 1, n, bm, 1.0 / (n * n), mb.data_ptr(),
            ws.data_ptr(), ws.numel(), s))
        nat.check("litho_abbe_workspace", L.litho_abbe_workspace(C.byref(pd.plan), C.byref(nb)))
        wsc = nat.Workspace.get(torch, self.dev, nb.value, tag="split_coarse")
        G = 4 * self.h + 1
        box = torch.empty((G * G,), dtype=torch.complex64, device=self.dev)
        nat.check("litho_coarse_image", L.litho_coarse_image(
            C.byref(pd.plan), pd._blob_dev.data_ptr(), table.data_ptr(), mb.data_ptr(), box.data_ptr(),
            wsc.data_ptr(), wsc.numel(), s))
        return box

    def finish(self, box):
        import ctypes as C
        torch, nat, L = self.torch, self.nat, self.L
        n = self.n
        nb = C.c_size_t(0)
        nat.check("litho_band_synthesis_workspace", L.litho_band_synthesis_workspace(1, n, C.byref(nb)))
        ws = nat.Workspace.get(torch, self.dev, nb.value, tag="split_synth")
        raw = torch.empty((n, n), dtype=torch.float32, device=self.dev)
        nat.check("litho_band_synthesis", L.litho_band_synthesis(
            box.data_ptr(), 1, n, 2 * self.h, 0, raw.data_ptr(), ws.data_ptr(), ws.numel(),
            nat.stream_ptr(torch, self.dev)))
        return raw

    def image(self, group=None, return_raw: bool = False):
        """(raw, peak, clear) with ``return_raw``, else the normalised, dosed
        image, the same on every rank."""
        from .aerial import normalisation_scale
        raw = split_abbe_image(self.partial, self.finish, self.n_sources, group)
        peak = float(raw.max())
        if return_raw:
            return raw, peak, self.clear
        return raw * normalisation_scale(self.v.normalisation, peak, self.clear, self.dose)


# ---------------------------------------------------------------------------
# one ILT clip split by SOCS kernels
# ---------------------------------------------------------------------------


def split_socs_objective(engine, masks, group=None):
    """Objective value and gradient of one batch of clips with the SOCS
    kernels split over the ranks of `group` (each rank's engine holds its
    kernels only):

        p = engine.forward(masks)       this rank's part of the image
        all-reduce(p)                   the whole image (every rank)
        cost, s = engine.objective(p)   replicated: the resist objective
        q = engine.adjoint(s)           this rank's part of the gradient
        all-reduce(q)
        return cost, engine.gradient(q)

    On the GPU p and q are band boxes (``GpuSocsSplit``)."""
    p = _all_reduce_sum(engine.forward(masks), group)
    cost, sens = engine.objective(p)
    q = _all_reduce_sum(engine.adjoint(sens), group)
    return cost, engine.gradient(q)


class GpuSocsSplit:
    """The GPU engine of ``split_socs_objective``: the band-limited ILT stages
    of this rank's kernels (``SOCSKernels.subset``), band boxes exchanged.

    forward(masks) -> image band boxes (C, (4h+1)^2) of this rank's kernels;
    objective(ibox) -> (cost (C,), band box of dJ/dI); adjoint(gbox) -> this
    rank's part of the gradient's band box (C, (2h+1)^2); gradient(hbox) ->
    dJ/dm (C, N, N) float32."""

    def __init__(self, kernels_local, targets, scale: float, level: float, sign: float = 1.0,
                 steepness: float = 12.0):
        import torch

        from .aerial import _as_device_masks
        from .ilt import stages
        n = int(kernels_local.grid.n_pixels)
        self.targets = _as_device_masks(torch, targets, n)
        self.st = stages(kernels_local, int(self.targets.shape[0]))
        self.args = (float(scale), float(level), float(sign), float(steepness))
        self._mbox = None

    def forward(self, masks):
        self._mbox = self.st.mask_box(masks)
        return self.st.image_box(self._mbox)

    def objective(self, ibox):
        cost, gbox, _signed, _perr = self.st.objective_from_box(ibox, self.targets, *self.args, want_signed=False)
        return cost, gbox

    def adjoint(self, gbox):
        return self.st.adjoint_box(gbox, self._mbox)

    def gradient(self, hbox):
        return self.st.synth(hbox, self.st.h, False)


__all__ = ["GpuAbbeSplit", "GpuSocsSplit", "clip_cost", "contiguous_ranges", "gather_results", "gather_tensors",
           "kernel_ranges", "run_sharded", "shard_plan", "source_ranges", "split_abbe_image",
           "split_socs_objective"]
