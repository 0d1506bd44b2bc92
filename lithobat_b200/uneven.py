"""Uneven batches: clips of several sizes imaged in one call, and ILT over
clips of several sizes.

The reference images clips one call at a time, whatever their size
(expose/aerial_image.py:502-548). Here the clips of a batch are grouped by
grid size; every group gets its own plan, pupil table, static input/output
buffers and workspace. With the default "queue" engine one
``litho_uneven_run`` images the whole batch: the coherent transforms of every
wide-pupil group (coarse grids of 128 points and more) are drained by ONE
persistent kernel from a device work queue of (jobs, pass A) and (work item,
row block, pass B) tasks across all groups, and groups on the on-chip coarse
grids run their own engine. The call is captured once as a CUDA graph and
each batch is one replay. The sizes of each group (jobs per work item, the
pass-A buffer slot and slots in flight, the tile of each kind of task) are
searched on the group's own clips the first time a (device, grid, pupil
width, clip count, optics) combination is seen, and persist in a JSON file.
"""

from __future__ import annotations

import ctypes as C
import dataclasses
import hashlib
import json
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _native as nat
from .aerial import coarse_grid, disc_halfwidth, fused_supported, plan_abbe, pupil_table
from .config import optics_view

#: candidates for jobs (source points x states) per work item: on-chip coarse
#: grids (L <= 64), and the wide-pupil engine (one L x L partial per item)
ITEM_CANDIDATES = (2, 4, 8, 16, 32)
WIDE_ITEM_CANDIDATES = (8, 16, 32)
#: the work queue's search space for wide groups, searched one knob at a time
#: (coordinate descent from the defaults, two sweeps)
QUEUE_SEARCH = {
    "items": (8, 16, 32),           # jobs per work item (source points per pass-B task)
    "slot_kib": (0, 65536, 262144, 1048576, 2097152),  # pass-A buffer per chunk of items (0: the library's
                                                       # size, 16 transforms per resident block)
    "b_rows": (1, 2, 4),            # row blocks per pass-B task (its tile height)
    "a_units": (48, 96, 192),       # warp transforms per pass-A task (its tile width)
    "n_slots": (2, 3, 4),           # chunks in flight
}
_TUNED: dict = {}
TUNE_CACHE_ENV = "LITHO_TUNE_CACHE"


@dataclass(frozen=True)
class QueueTune:
    """Work-queue sizes of one wide group (litho_b200.h: LithoUnevenGroup)."""
    items: int = 16
    slot_kib: int = 0
    n_slots: int = 2
    a_units: int = 96
    b_rows: int = 0


def tune_cache_path() -> Path:
    """The JSON file tuned sizes persist in: $LITHO_TUNE_CACHE, else
    ~/.cache/lithobat_b200/uneven_tune.json."""
    p = os.environ.get(TUNE_CACHE_ENV)
    return Path(p) if p else Path.home() / ".cache" / "lithobat_b200" / "uneven_tune.json"


def _load_cache(path: Path) -> dict:
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def _store_cache(path: Path, key: str, value: dict) -> None:
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        data = _load_cache(path)
        data[key] = value
        tmp = path.with_suffix(path.suffix + ".tmp")
        tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
        tmp.replace(path)
    except OSError:
        pass   # a read-only home: the sizes are still kept for this process


def tune_key(device_name: str, n: int, h: int, L: int, clips: int, view) -> str:
    """Cache key of one size group: device, grid side, pupil half-width,
    coarse grid, clip count and the optics."""
    digest = hashlib.sha1(repr(view).encode()).hexdigest()[:16]
    return f"{device_name}|n={n}|h={h}|L={L}|clips={clips}|optics={digest}"


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
    tune: QueueTune | None = None
    cg: object = None      # nat.UnevenGroup of the queue engine (raw addresses of the tensors here)
    blob: object = None    # the plan's device blob the descriptors point to


def _run_group(torch, L, g: _Group, stream: int) -> None:
    nat.check("litho_abbe_tabled", L.litho_abbe_tabled(
        C.byref(g.pd.plan), g.pd._blob_dev.data_ptr(), g.table.data_ptr(), g.masks.data_ptr(), g.image.data_ptr(),
        g.peak.data_ptr(), g.ws.data_ptr(), g.ws.numel(), stream))


def queue_schedule(L, cgroups) -> tuple[np.ndarray, int]:
    """The work queue's task list (QUEUE_TASK_DTYPE) and counter count for an
    array of nat.UnevenGroup (host only: reads the plans' host blobs)."""
    n = len(cgroups)
    nt, nc = C.c_int(0), C.c_int(0)
    nat.check("litho_uneven_schedule", L.litho_uneven_schedule(cgroups, n, None, 0, C.byref(nt), C.byref(nc)))
    tasks = np.zeros(max(nt.value, 1), dtype=nat.QUEUE_TASK_DTYPE)
    nat.check("litho_uneven_schedule", L.litho_uneven_schedule(
        cgroups, n, tasks.ctypes.data, tasks.size, C.byref(nt), C.byref(nc)))
    return tasks[:nt.value], nc.value


class _Queue:
    """Device copy of a schedule plus the queue's workspace."""

    def __init__(self, torch, L, dev, groups: list):
        self.arr = (nat.UnevenGroup * len(groups))(*[g.cg for g in groups])
        tasks, self.n_counters = queue_schedule(L, self.arr)
        self.n_tasks = int(tasks.size)
        self.tasks_host = tasks
        self.tasks = torch.from_numpy(tasks.view(np.uint8).copy()).to(dev) if self.n_tasks else None
        nb = C.c_size_t(0)
        nat.check("litho_uneven_queue_workspace", L.litho_uneven_queue_workspace(self.n_counters, C.byref(nb)))
        self.ws = torch.zeros(max(nb.value, 256), dtype=torch.uint8, device=dev)
        self.n_groups = len(groups)

    def launch(self, L, stream: int) -> None:
        nat.check("litho_uneven_run", L.litho_uneven_run(
            self.arr, self.n_groups, self.tasks.data_ptr() if self.tasks is not None else None, self.n_tasks,
            self.n_counters, self.ws.data_ptr(), self.ws.numel(), stream))


class UnevenAbbe:
    """Abbe images of a batch of clips of mixed sizes (one optics, one pixel size).

    sizes: the grid side of every clip, in batch order. ``__call__`` takes the
    masks (a list of (N_i, N_i) device tensors or arrays) and returns the
    images as a list of (N_i, N_i) float32 device tensors (views of the
    group's output buffer, overwritten by the next call).

    engine "queue" (default): one ``litho_uneven_run`` per batch — the
    coherent passes of every wide-pupil group drained by one persistent kernel
    from a device work queue, coarse-grid groups on their on-chip engine.
    engine "groups": one ``litho_abbe_tabled`` launch sequence per group.
    Either way the whole batch is captured once as a CUDA graph. ``tune``
    searches each group's sizes on its own clips the first time a (device,
    grid, pupil width, clip count, optics) combination is seen, and keeps the
    result in memory and in the JSON file of ``tune_cache_path()``."""

    def __init__(self, sizes, optics, pixel_size: float, *, mask_complex: bool = False, dose: float = 1.0,
                 return_raw: bool = False, graph: bool = True, tune: bool = True, device=None,
                 engine: str = "queue", tune_cache: str | os.PathLike | None = None):
        torch = nat.require_cuda()
        if engine not in ("queue", "groups"):
            raise ValueError(f"engine must be 'queue' or 'groups', got {engine!r}")
        self.torch, self.L = torch, nat.lib()
        self.dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.engine = engine
        self.cache_path = Path(tune_cache) if tune_cache is not None else tune_cache_path()
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
            self.groups.append(self._group(n, idx, masks, 8, QueueTune()))
        self.tuned = {}
        if tune:
            self._tune()
        self.queue = _Queue(torch, self.L, self.dev, self.groups) if engine == "queue" else None
        self.graph = None
        if graph:
            self._capture()

    # ------------------------------------------------------------------
    def _wide(self, n: int) -> bool:
        h = disc_halfwidth(self.view.NA, self.view.wavelength, n, self.px)[1]
        return coarse_grid(h) > 64

    def _group(self, n, idx, masks, items, tune: QueueTune) -> _Group:
        torch, L = self.torch, self.L
        v = self.view
        queued = self.engine == "queue" and self._wide(n)
        pd = plan_abbe([v] * len(idx), n, self.px, [[(v.defocus, v.image_index)]] * len(idx), self.dose,
                       self.return_raw, self.complex, items_per_job_group=tune.items if queued else items)
        if not fused_supported(n, int(pd.plan.L)):
            raise NotImplementedError(f"{n}^2 clips need the full-grid engine, which this batch runner does not "
                                      "capture; image them with compute_aerial_batch")
        # plans are cached and shared between runners and tuning candidates:
        # keep the plan's device blob (the queue's descriptors hold its raw
        # address, so it must never be replaced while a group uses it)
        blob_dev = getattr(pd, "_blob_dev", None)
        if blob_dev is None or blob_dev.device != self.dev:
            blob_dev = torch.from_numpy(pd.blob).to(self.dev)
            pd._blob_dev = blob_dev
        s = nat.stream_ptr(torch, self.dev)
        table = pupil_table(pd, self.dev, s)
        image = torch.empty((len(idx), n, n), dtype=torch.float32, device=self.dev)
        peak = torch.empty((len(idx),), dtype=torch.float32, device=self.dev)
        nb = C.c_size_t(0)
        cg = None
        if self.engine == "queue":
            cg = nat.UnevenGroup(plan=pd.plan, blob_host=pd.blob.ctypes.data, blob_dev=blob_dev.data_ptr(),
                                 table_dev=table.data_ptr(), masks_dev=masks.data_ptr(), image_dev=image.data_ptr(),
                                 peak_dev=peak.data_ptr(), workspace_dev=None, ws_bytes=0,
                                 slot_kib=tune.slot_kib, n_slots=tune.n_slots, a_units=tune.a_units,
                                 b_rows=tune.b_rows)
            nat.check("litho_uneven_group_workspace", L.litho_uneven_group_workspace(C.byref(cg), C.byref(nb)))
        else:
            nat.check("litho_abbe_workspace", L.litho_abbe_workspace(C.byref(pd.plan), C.byref(nb)))
        ws = torch.empty(max(nb.value, 256), dtype=torch.uint8, device=self.dev)
        if cg is not None:
            cg.workspace_dev = ws.data_ptr()
            cg.ws_bytes = ws.numel()
        return _Group(n, idx, pd, masks, image, peak, ws, table, items, tune if queued else None, cg, blob_dev)

    def _time(self, launch, reps: int = 2) -> float:
        torch = self.torch
        launch()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            launch()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def _search_items(self, g: _Group) -> tuple[dict, dict]:
        """Work-item size of a group run by litho_abbe_tabled: every candidate."""
        torch = self.torch
        times = {}
        cands = ITEM_CANDIDATES if not self._wide(g.n) else WIDE_ITEM_CANDIDATES
        for items in cands:
            cand = self._group(g.n, g.index, g.masks, items, QueueTune())
            s = nat.stream_ptr(torch, self.dev)
            times[items] = self._time(lambda: _run_group(torch, self.L, cand, s))
            del cand
        best = min(times, key=times.get)
        return {"items_per_block": best}, {str(k): v for k, v in times.items()}

    def _search_queue(self, g: _Group) -> tuple[dict, dict]:
        """Queue sizes of a wide group, each candidate run as a one-group
        queue on the group's clips: coordinate descent over QUEUE_SEARCH."""
        torch, L = self.torch, self.L
        times: dict = {}

        def measure(t: QueueTune) -> float:
            key = dataclasses.astuple(t)
            if key not in times:
                cand = self._group(g.n, g.index, g.masks, t.items, t)
                q = _Queue(torch, L, self.dev, [cand])
                s = nat.stream_ptr(torch, self.dev)
                times[key] = self._time(lambda: q.launch(L, s))
                del q, cand
            return times[key]

        cur = QueueTune()
        best = measure(cur)
        for _sweep in range(2):
            moved = False
            for knob, values in QUEUE_SEARCH.items():
                for val in values:
                    t = dataclasses.replace(cur, **{knob: val})
                    ms = measure(t)
                    if ms < best * 0.99:
                        cur, best, moved = t, ms, True
            if not moved:
                break
        out = dataclasses.asdict(cur)
        out["items_per_block"] = cur.items
        return out, {"best_ms": best, "candidates": len(times)}

    def _tune(self) -> None:
        """Per group: the cached sizes of its (device, grid, pupil width, clip
        count, optics, engine) key, else a search on the group's own clips."""
        torch = self.torch
        name = torch.cuda.get_device_name(self.dev)
        cache = _load_cache(self.cache_path)
        for k, g in enumerate(self.groups):
            h = disc_halfwidth(self.view.NA, self.view.wavelength, g.n, self.px)[1]
            queued = self.engine == "queue" and self._wide(g.n)
            key = tune_key(name, g.n, h, coarse_grid(h), len(g.index), self.view) + (
                "|queue" if queued else "|launches")
            best = _TUNED.get(key) or cache.get(key)
            if best is None:
                best, info = self._search_queue(g) if queued else self._search_items(g)
                _TUNED[key] = best
                _store_cache(self.cache_path, key, best)
                self.tuned[g.n] = {**best, "ms": info, "source": "search"}
            else:
                _TUNED[key] = best
                self.tuned[g.n] = {**best, "source": "cache"}
            if queued:
                t = QueueTune(**{f.name: int(best[f.name]) for f in dataclasses.fields(QueueTune)})
                self.groups[k] = self._group(g.n, g.index, g.masks, t.items, t)
            elif int(best["items_per_block"]) != g.items:
                self.groups[k] = self._group(g.n, g.index, g.masks, int(best["items_per_block"]), QueueTune())

    def _launch_all(self) -> None:
        s = nat.stream_ptr(self.torch, self.dev)
        if self.queue is not None:
            self.queue.launch(self.L, s)
            return
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
        up in the latest run of any size group or of the work queue (its
        images are then invalid)."""
        self.torch.cuda.synchronize(self.dev)
        words = [(g.ws, "litho_abbe_tabled") for g in self.groups]
        if self.queue is not None:
            words.append((self.queue.ws, "litho_uneven_run"))
        for ws, fn in words:
            st = int(ws[:4].view(self.torch.int32).item())
            if st:
                nat.check(fn, st)

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

    def run(self, n_steps: int):
        """``n_steps`` ILT iterations of every clip without the signed field;
        returns the costs in batch order (device). Each group steps by
        ``IltBatch.run`` (its fast step recorded once as a CUDA graph and
        replayed), and the groups' replays go on parallel streams, so the
        small groups' kernels overlap the large groups' passes. Groups are
        independent, so the iterates are those of ``step()``."""
        torch = self.torch
        n_steps = int(n_steps)
        if n_steps > 0 and any(b._graph is None for _n, _i, _k, b in self.groups):
            for _n, _i, _k, b in self.groups:   # the first call records each group's graph (one step)
                b.run(1)
            n_steps -= 1
        if n_steps > 0:
            if getattr(self, "_streams", None) is None:
                self._streams = [torch.cuda.Stream() for _ in self.groups]
            main = torch.cuda.current_stream()
            for s in self._streams:
                s.wait_stream(main)
            for (_n, _i, _k, b), s in zip(self.groups, self._streams):
                with torch.cuda.stream(s):
                    b.run(n_steps)
            for s in self._streams:
                main.wait_stream(s)
        cost = [None] * len(self.sizes)
        for _n, idx, _k, b in self.groups:
            for j, i in enumerate(idx):
                cost[i] = b.cost[j]
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
                     return_raw=return_raw, graph=False, tune=False)
    imgs = run(masks)
    return [im.clone() if t else im.cpu().numpy().astype(np.float64) for im, t in zip(imgs, is_t)]


__all__ = ["UnevenAbbe", "UnevenIlt", "compute_aerial_uneven", "ITEM_CANDIDATES", "QUEUE_SEARCH", "QueueTune",
           "queue_schedule", "tune_cache_path"]
