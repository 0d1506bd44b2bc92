"""Host-to-host imaging of a stream of mask batches with the copies overlapped.

A caller whose masks live in host memory (the reference's numpy callers:
opc/model.py, analysis/process_window.py, the CLI) pays the host link for every
batch: 8 bytes per complex mask pixel in, 4 bytes per image pixel out. Run one
batch at a time and the GPU idles while the link works. ``AbbePipeline`` keeps
``depth`` device slots and three CUDA streams: while batch i is imaged, batch
i+1 is uploaded and batch i-1 downloaded, ordered by events, so a stream of
batches runs at the link's pace rather than at link + compute.
"""

from __future__ import annotations

import ctypes as C

from . import _native as nat
from .aerial import fused_supported, plan_abbe, pupil_table
from .config import optics_view


class AbbePipeline:
    """Images batches of ``batch`` clips (one optics, one grid) from pinned
    host tensors into pinned host tensors.

    ``run(inputs, outputs)``: inputs[i] (batch, N, N) float32 or complex64
    pinned CPU tensors, outputs[i] (batch, N, N) float32 pinned CPU tensors
    (the same tensor may appear several times in either list; an output is
    complete once ``run`` returns). ``run`` raises ``LithoError`` if a bounded
    wait inside any batch's kernels gave up (``LITHO_E_TIMEOUT``).

    ``level_masks=True``: inputs are level maps, (batch, N, N) uint8 indices
    into ``run(..., levels=...)``, a (batch, n_levels) complex64 tensor shared
    by every batch of the run (``litho_abbe_levels``): one byte per pixel over
    the host link instead of eight for complex masks."""

    def __init__(self, optics, grid, batch: int, mask_complex: bool, dose: float = 1.0, return_raw: bool = False,
                 depth: int = 2, device=None, level_masks: bool = False):
        torch = nat.require_cuda()
        self.torch, self.L = torch, nat.lib()
        self.dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        v = optics_view(optics)
        self.n = n = int(grid.n_pixels)
        self.batch = int(batch)
        self.levels = bool(level_masks)
        self.complex = bool(mask_complex) or self.levels
        self.pd = plan_abbe([v] * self.batch, n, float(grid.pixel_size), [[(v.defocus, v.image_index)]] * self.batch,
                            float(dose), bool(return_raw), self.complex)
        if not fused_supported(n, int(self.pd.plan.L)):
            raise NotImplementedError("the pipeline runs the band-limited engines only")
        blob = getattr(self.pd, "_blob_dev", None)   # plans are cached and shared: keep an existing copy
        if blob is None or blob.device != self.dev:
            self.pd._blob_dev = torch.from_numpy(self.pd.blob).to(self.dev)
        self.table = pupil_table(self.pd, self.dev, nat.stream_ptr(torch, self.dev))
        nb = C.c_size_t(0)
        nat.check("litho_abbe_workspace", self.L.litho_abbe_workspace(C.byref(self.pd.plan), C.byref(nb)))
        self.ws = torch.empty(max(nb.value, 256), dtype=torch.uint8, device=self.dev)
        if self.levels and int(self.pd.plan.L) > 64:
            raise NotImplementedError("level-map masks run on the coarse-grid engines only")
        dt = torch.uint8 if self.levels else (torch.complex64 if self.complex else torch.float32)
        self.depth = max(2, int(depth))
        self.d_in = [torch.empty((self.batch, n, n), dtype=dt, device=self.dev) for _ in range(self.depth)]
        self.d_out = [torch.empty((self.batch, n, n), dtype=torch.float32, device=self.dev) for _ in range(self.depth)]
        self.d_peak = [torch.empty((self.batch,), dtype=torch.float32, device=self.dev) for _ in range(self.depth)]
        self.s_in = torch.cuda.Stream(device=self.dev)
        self.s_run = torch.cuda.Stream(device=self.dev)
        self.s_out = torch.cuda.Stream(device=self.dev)
        # the workspace's status word (offset 0) is cleared by every call; the
        # worst status of a run is kept here, read once the run has synchronised
        self._status = self.ws[:4].view(torch.int32)
        self._worst = torch.zeros((1,), dtype=torch.int32, device=self.dev)

    def run(self, inputs, outputs, levels=None) -> None:
        torch, L = self.torch, self.L
        if len(inputs) != len(outputs):
            raise ValueError(f"{len(inputs)} input batches for {len(outputs)} outputs")
        if self.levels:
            if levels is None or tuple(levels.shape[:1]) != (self.batch,) or levels.dim() != 2:
                raise ValueError(f"level-map inputs need levels of shape ({self.batch}, n_levels)")
            with torch.cuda.stream(self.s_in):
                d_lv = levels.to(self.dev, torch.complex64, non_blocking=True).contiguous()
            self.s_run.wait_stream(self.s_in)
        ev = torch.cuda.Event
        read_done = [None] * self.depth    # compute finished reading d_in[slot]
        sent = [None] * self.depth         # download of d_out[slot] finished
        for i, (hin, hout) in enumerate(zip(inputs, outputs)):
            k = i % self.depth
            with torch.cuda.stream(self.s_in):
                if read_done[k] is not None:
                    self.s_in.wait_event(read_done[k])
                self.d_in[k].copy_(hin, non_blocking=True)
                loaded = ev()
                loaded.record(self.s_in)
            with torch.cuda.stream(self.s_run):
                self.s_run.wait_event(loaded)
                if sent[k] is not None:
                    self.s_run.wait_event(sent[k])
                if self.levels:
                    nat.check("litho_abbe_levels", L.litho_abbe_levels(
                        C.byref(self.pd.plan), self.pd._blob_dev.data_ptr(), self.table.data_ptr(),
                        self.d_in[k].data_ptr(), d_lv.data_ptr(), int(d_lv.shape[1]), self.d_out[k].data_ptr(),
                        self.d_peak[k].data_ptr(), self.ws.data_ptr(), self.ws.numel(), int(self.s_run.cuda_stream)))
                else:
                    nat.check("litho_abbe_tabled", L.litho_abbe_tabled(
                        C.byref(self.pd.plan), self.pd._blob_dev.data_ptr(), self.table.data_ptr(),
                        self.d_in[k].data_ptr(), self.d_out[k].data_ptr(), self.d_peak[k].data_ptr(),
                        self.ws.data_ptr(), self.ws.numel(), int(self.s_run.cuda_stream)))
                torch.maximum(self._worst, self._status, out=self._worst)
                done = ev()
                done.record(self.s_run)
                read_done[k] = done
            with torch.cuda.stream(self.s_out):
                self.s_out.wait_event(done)
                hout.copy_(self.d_out[k], non_blocking=True)
                fin = ev()
                fin.record(self.s_out)
                sent[k] = fin
        self.s_out.synchronize()
        self.s_run.synchronize()
        worst = int(self._worst.item())
        if worst:
            self._worst.zero_()
            nat.check("litho_abbe_tabled", worst)


__all__ = ["AbbePipeline"]
