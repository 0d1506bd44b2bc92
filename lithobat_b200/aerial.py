"""Partially coherent aerial images on the B200: the drop-in Abbe entry points.

Public functions mirror ``litho_sim.expose.aerial_image``:

* :func:`compute_aerial_image` — ``compute_aerial_image(mask, optics, grid,
  dose=1.0, return_raw=False)`` (aerial_image.py:502-548)
* :func:`compute_aerial_planes` — several (defocus, n_image) planes in one
  pass (aerial_image.py:551-587)
* :func:`normalisation_scale` — the one scalar of a normalisation
  (aerial_image.py:217-241)
* :func:`compute_aerial_batch` — many clips (each with its own optics) and
  planes in one launch sequence; the batched form the drop-in calls reduce to.

numpy inputs give numpy float64 outputs, as the reference returns; torch CUDA
inputs give torch float32 CUDA outputs and never leave the device. The work
runs in ``liblitho_b200.so``; there is no CPU path.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _native as nat
from .config import IMAGING_MODELS, NORMALISATIONS, optics_view
from .pupil import clear_throughput, jones_states
from .source import source_points

#: expose/aerial_image.py:73 — the sign of the tilt a source point applies to
#: the mask; the engine evaluates the pupil at f - f_s exactly as the reference.
SOURCE_TILT_SIGN = -1.0


def normalisation_scale(mode: str, peak: float, clear: float, dose: float = 1.0) -> float:
    """The single constant that turns a raw Abbe sum into a dosed image."""
    m = mode.lower()
    if m == "peak":
        return dose / peak if peak > 0 else dose
    if m == "clear":
        return dose / clear if clear > 0 else dose
    if m == "none":
        return dose
    raise ValueError(f"normalisation must be 'peak', 'clear' or 'none', got '{mode}'")


def disc_halfwidth(NA: float, wavelength: float, n: int, pixel_size: float) -> tuple[float, int]:
    """Pupil radius R in frequency bins, and the integer half-width h of the
    box around a source point's nearest bin that contains its whole disc."""
    R = (NA / wavelength) * n * pixel_size
    return R, int(math.floor(R + 0.5 + 1e-9 * (1.0 + R)))


@dataclass
class AbbePlanData:
    plan: nat.AbbePlan
    blob: np.ndarray
    clears: np.ndarray           # (n_out,) float64
    n_out: int
    jobs: int
    transforms: int              # coherent transforms (jobs x components)


def _validate_view(v) -> None:
    if v.imaging_model.lower() not in IMAGING_MODELS:
        raise ValueError(f"imaging_model must be 'scalar' or 'vector', got '{v.imaging_model}'")
    if v.normalisation.lower() not in NORMALISATIONS:
        raise ValueError(f"normalisation must be 'peak', 'clear' or 'none', got '{v.normalisation}'")
    if v.mask_model.lower() != "thin":
        raise ValueError(
            f"mask_model={v.mask_model!r}: this engine images thin (Kirchhoff) masks only; "
            "thick-mask spectra are outside the accelerated path")


def plan_abbe(views: Sequence, n: int, pixel_size: float, planes: Sequence[Sequence[tuple]],
              dose: float, return_raw: bool, mask_complex: bool, items_per_job_group: int = 4) -> AbbePlanData:
    """Build the device descriptors of one batched Abbe sum.

    views[c] is the optics of clip c, planes[c] its list of (defocus, n_image).
    Every clip must have the same number of planes.
    """
    C = len(views)
    P = len(planes[0])
    if any(len(p) != P for p in planes):
        raise ValueError("every clip needs the same number of planes")
    val = 1.0 / (n * pixel_size)
    pupils = np.zeros(C * P, dtype=nat.PUPIL_DTYPE)
    job_rows = []
    clears = np.zeros(C * P, dtype=np.float64)
    h = 0
    vec_any = False
    for c, v in enumerate(views):
        _validate_view(v)
        vector = v.imaging_model.lower() == "vector"
        vec_any |= vector
        exact = v.exact_defocus or vector
        src = source_points(v)
        _, hc = disc_halfwidth(v.NA, v.wavelength, n, pixel_size)
        h = max(h, hc)
        zern = np.zeros(21)
        for j, coef in v.zernike:
            if 1 <= j <= 21:
                zern[j - 1] = coef
        cxs = np.rint(src.fx / val).astype(np.int64)
        cys = np.rint(src.fy / val).astype(np.int64)
        for p, (dz, n_img) in enumerate(planes[c]):
            k = c * P + p
            pupils[k]["wavelength"] = v.wavelength
            pupils[k]["NA"] = v.NA
            pupils[k]["defocus"] = float(dz)
            pupils[k]["n_image"] = float(n_img)
            pupils[k]["zernike"] = zern
            pupils[k]["exact_defocus"] = int(exact)
            pupils[k]["vector"] = int(vector)
            pupils[k]["obliquity"] = int(v.obliquity)
            pupils[k]["has_zernike"] = int(bool(np.any(zern != 0.0)))
            clears[k] = clear_throughput(src, v, float(n_img), vector)
            for s in range(len(src)):
                states = jones_states(v.polarisation, float(src.phi[s])) if vector else [(0.0, 0.0, 1.0)]
                for jx, jy, wp in states:
                    job_rows.append((src.fx[s], src.fy[s], jx, jy, src.weight[s] * wp, k, c, k,
                                     cxs[s], cys[s], 3 if vector else 1))
    if not job_rows:
        raise ValueError("the source has no points")
    jobs = np.zeros(len(job_rows), dtype=nat.JOB_DTYPE)
    arr = np.array(job_rows, dtype=object)
    for i, name in enumerate(nat.JOB_DTYPE.names):
        jobs[name] = arr[:, i].astype(nat.JOB_DTYPE[name])
    # jobs are already grouped by output (k); chunk each output's run
    n_out = C * P
    items, out_items = [], [0]
    per = max(1, int(items_per_job_group))
    starts = np.searchsorted(jobs["out"], np.arange(n_out + 1), side="left")
    for o in range(n_out):
        b, e = int(starts[o]), int(starts[o + 1])
        for j in range(b, e, per):
            items.append((o, j, min(j + per, e), 0))
        out_items.append(len(items))
    items = np.array(items, dtype=np.int32).view(nat.ITEM_DTYPE).reshape(-1)
    out_items = np.array(out_items, dtype=np.int32)
    norm = np.zeros(n_out, dtype=nat.NORM_DTYPE)
    for c, v in enumerate(views):
        for p in range(P):
            k = c * P + p
            if return_raw:
                norm[k] = (0, 1.0)
            else:
                m = v.normalisation.lower()
                if m == "peak":
                    norm[k] = (1, dose)
                else:
                    norm[k] = (0, normalisation_scale(m, 1.0, clears[k], dose))
    bm = int(max(np.abs(jobs["cx"]).max(), np.abs(jobs["cy"]).max())) + h
    blob, offs = nat.blob([jobs, pupils, items, out_items, norm])
    plan = nat.AbbePlan(
        n=n, n_clips=C, n_out=n_out, n_jobs=len(jobs), n_items=len(items), n_pupils=len(pupils),
        h=h, bm=bm, L=32, mask_complex=int(mask_complex), ncomp_max=3 if vec_any else 1, flags=0,
        pixel_size=pixel_size, off_jobs=offs[0], off_pupils=offs[1], off_items=offs[2],
        off_out_items=offs[3], off_norm=offs[4])
    if 4 * h + 1 > 32:
        raise NotImplementedError(
            f"pupil radius {h} bins needs a coarse grid above 32; this build serves 4h+1 <= 32")
    transforms = int(np.sum(jobs["ncomp"]))
    return AbbePlanData(plan, blob, clears, n_out, len(jobs), transforms)


# ---------------------------------------------------------------------------
# running
# ---------------------------------------------------------------------------


def _as_device_masks(torch, masks, n: int):
    """(C, N, N) device tensor, float32 or complex64; complex with zero
    imaginary part is sent as real (the spectrum is the same)."""
    if isinstance(masks, torch.Tensor):
        t = masks
        if t.dim() == 2:
            t = t.unsqueeze(0)
        dev = t.device if t.is_cuda else torch.device("cuda", torch.cuda.current_device())
        t = t.to(dev)
    else:
        a = np.asarray(masks)
        if a.ndim == 2:
            a = a[None]
        if np.iscomplexobj(a):
            a = a.astype(np.complex64) if not np.all(a.imag == 0) else a.real.astype(np.float32)
        else:
            a = a.astype(np.float32)
        t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    if t.is_complex():
        if not bool(torch.any(t.imag != 0)):
            t = t.real
        else:
            t = t.to(torch.complex64)
    if not t.is_complex():
        t = t.to(torch.float32)
    if t.shape[-2:] != (n, n):
        raise ValueError(f"mask must be {(n, n)} for this grid, got {tuple(t.shape[-2:])}")
    return t.contiguous()


def run_abbe(pd: AbbePlanData, masks_dev, out=None, peak=None, stream=None):
    """Launch one planned Abbe batch; returns (images (n_out, N, N), peaks (n_out,))."""
    torch = nat.require_cuda()
    L = nat.lib()
    dev = masks_dev.device
    n = pd.plan.n
    if out is None:
        out = torch.empty((pd.n_out, n, n), dtype=torch.float32, device=dev)
    if peak is None:
        peak = torch.empty((pd.n_out,), dtype=torch.float32, device=dev)
    import ctypes as C
    ws_bytes = C.c_size_t(0)
    nat.check("litho_abbe_workspace", L.litho_abbe_workspace(C.byref(pd.plan), C.byref(ws_bytes)))
    ws = nat.Workspace.get(torch, dev, ws_bytes.value)
    blob = getattr(pd, "_blob_dev", None)
    if blob is None or blob.device != dev:
        blob = torch.from_numpy(pd.blob).to(dev)
        pd._blob_dev = blob
    s = stream if stream is not None else nat.stream_ptr(torch, dev)
    nat.check("litho_abbe", L.litho_abbe(C.byref(pd.plan), blob.data_ptr(), masks_dev.data_ptr(),
                                          out.data_ptr(), peak.data_ptr(), ws.data_ptr(),
                                          ws.numel(), s))
    return out, peak


def _grid(grid):
    return int(grid.n_pixels), float(grid.pixel_size)


def compute_aerial_batch(masks, optics, grid, planes=None, dose: float = 1.0, return_raw: bool = False):
    """Abbe images of a batch of clips on the GPU.

    masks: (C, N, N) numpy array or torch tensor (real or complex).
    optics: one optics object for all clips, or a sequence of C of them.
    planes: None (each clip's own defocus / image index), a list of
        (defocus, n_image) shared by all clips, or a list of C such lists.
    Returns (images, peaks, clears): images (C, P, N, N) float32 CUDA tensor,
    peaks (C, P) raw maxima, clears (C, P) float64 numpy.
    """
    torch = nat.require_cuda()
    n, px = _grid(grid)
    md = _as_device_masks(torch, masks, n)
    Cn = md.shape[0]
    views = [optics_view(o) for o in optics] if isinstance(optics, (list, tuple)) else \
        [optics_view(optics)] * Cn
    if len(views) != Cn:
        raise ValueError(f"{len(views)} optics for {Cn} clips")
    if planes is None:
        pl = [[(v.defocus, v.image_index)] for v in views]
    elif len(planes) and isinstance(planes[0], (list, tuple)) and len(planes[0]) and \
            isinstance(planes[0][0], (list, tuple)):
        pl = [list(p) for p in planes]
    else:
        pl = [list(planes)] * Cn
    pd = plan_abbe(views, n, px, pl, dose, return_raw, md.is_complex())
    img, pk = run_abbe(pd, md)
    P = len(pl[0])
    return img.view(Cn, P, n, n), pk.view(Cn, P), pd.clears.reshape(Cn, P)


def _is_torch(x) -> bool:
    try:
        import torch
        return isinstance(x, torch.Tensor)
    except ImportError:  # pragma: no cover
        return False


def compute_aerial_image(mask, optics, grid, dose: float = 1.0, return_raw: bool = False):
    """Drop-in for ``litho_sim.expose.compute_aerial_image`` (aerial_image.py:502-548).

    Returns the (N, N) image normalised as ``optics.normalisation`` says and
    multiplied by ``dose``; with ``return_raw`` the tuple (raw, peak, clear)."""
    v = optics_view(optics)
    img, pk, cl = compute_aerial_batch(mask, optics, grid, [(v.defocus, v.image_index)], dose,
                                       return_raw)
    a = img[0, 0]
    if not _is_torch(mask):
        a = a.cpu().numpy().astype(np.float64)
    if return_raw:
        return a, float(pk[0, 0]), float(cl[0, 0])
    return a


def compute_aerial_planes(mask, optics, grid, planes: Sequence[tuple[float, float]], dose: float = 1.0):
    """Drop-in for ``compute_aerial_planes`` (aerial_image.py:551-587): (P, N, N),
    each plane normalised on its own."""
    img, _pk, _cl = compute_aerial_batch(mask, optics, grid, [tuple(p) for p in planes], dose, False)
    out = img[0]
    return out if _is_torch(mask) else out.cpu().numpy().astype(np.float64)
