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

import ctypes
import math
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _native as nat
from .config import IMAGING_MODELS, NORMALISATIONS, optics_view
from . import multilayer
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


def coarse_grid(h: int) -> int:
    """The coarse grid side: the smallest power of two L >= 32 with L >= 4h + 1,
    on which |E|^2 of a (2h+1)^2 spectrum is exact."""
    L = 32
    while L < 4 * h + 1:
        L *= 2
    return L


def fused_supported(n: int, L: int) -> bool:
    """Can the band-limited engine run this grid? (L <= 64 on chip; 128..1024
    through the wide engine, which also needs a power-of-two N >= L.)"""
    if L <= 64:
        return True
    return L <= 1024 and L <= n <= 4096 and (n & (n - 1)) == 0


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
    if v.mask_model.lower() not in ("thin", "multilayer"):
        raise ValueError(
            f"mask_model={v.mask_model!r}: this engine images thin (Kirchhoff) masks, on their own or on "
            "a multilayer mirror; rigorous (FDTD) near fields are outside the accelerated path")


_PLANS: dict = {}


def plan_abbe(views: Sequence, n: int, pixel_size: float, planes: Sequence[Sequence[tuple]],
              dose: float, return_raw: bool, mask_complex: bool, items_per_job_group: int = 0,
              sources: tuple[int, int] | None = None) -> AbbePlanData:
    """Build (or fetch from a small cache) the device descriptors of one
    batched Abbe sum. views[c] is the optics of clip c, planes[c] its list of
    (defocus, n_image); every clip has the same number of planes. ``sources``
    (start, stop) keeps only those source points of every clip (in the
    reference's order): the plan then sums part of the Abbe sum, and its
    ``clears`` are that part's share of the clear throughput."""
    key = (tuple(repr(v) for v in views), n, pixel_size, tuple(tuple(map(tuple, p)) for p in planes),
           float(dose), bool(return_raw), bool(mask_complex), items_per_job_group,
           None if sources is None else (int(sources[0]), int(sources[1])))
    hit = _PLANS.get(key)
    if hit is not None:
        return hit
    pd = _plan_abbe(views, n, pixel_size, planes, dose, return_raw, mask_complex, items_per_job_group, sources)
    if len(_PLANS) > 32:
        _PLANS.clear()
    _PLANS[key] = pd
    return pd


def _source_slice(src, sources):
    if sources is None:
        return src
    a, b = int(sources[0]), int(sources[1])
    if not 0 <= a < b <= len(src):
        raise ValueError(f"source range {sources} outside the {len(src)} source points")
    return type(src)(weight=src.weight[a:b], fx=src.fx[a:b], fy=src.fy[a:b], phi=src.phi[a:b], grid=src.grid)


def _plan_abbe(views, n, pixel_size, planes, dose, return_raw, mask_complex, items_per_job_group, sources=None):
    C = len(views)
    P = len(planes[0])
    if any(len(p) != P for p in planes):
        raise ValueError("every clip needs the same number of planes")
    val = 1.0 / (n * pixel_size)
    pupils = np.zeros(C * P, dtype=nat.PUPIL_DTYPE)
    clears = np.zeros(C * P, dtype=np.float64)
    h = 0
    vec_any = False
    cols = {k: [] for k in nat.JOB_DTYPE.names}
    slot_of_state: dict = {}     # (optics, plane) -> first slot of its (source, state) run
    slot_reps: list[np.ndarray] = []
    n_tab = 0
    n_jobs = 0
    mirror_rows = np.zeros(C * P, dtype=nat.MIRROR_DTYPE)
    mirror_tabs: list = []       # distinct reflection tables, in first-use order
    for c, v in enumerate(views):
        _validate_view(v)
        mirror, m_scale = None, None
        if v.mask_model.lower() == "multilayer":
            mirror = multilayer.mirror_table(multilayer.stack_for(v), v.wavelength)
            if not any(t is mirror for t in mirror_tabs):
                mirror_tabs.append(mirror)
        vector = v.imaging_model.lower() == "vector"
        vec_any |= vector
        exact = v.exact_defocus or vector
        src = _source_slice(source_points(v), sources)
        S = len(src)
        if S == 0:
            raise ValueError("the source has no points")
        if mirror is not None:
            m_scale = multilayer.clear_scales(v, src)
            cxs, cys = multilayer.chief_ray_sines(v)
            m_idx = next(i for i, t in enumerate(mirror_tabs) if t is mirror)
        _, hc = disc_halfwidth(v.NA, v.wavelength, n, pixel_size)
        h = max(h, hc)
        zern = np.zeros(21)
        for j, coef in v.zernike:
            if 1 <= j <= 21:
                zern[j - 1] = coef
        # incoherent states of every source point (one for scalar / polarised)
        st = [jones_states(v.polarisation, float(ph)) for ph in src.phi] if vector else [[(0.0, 0.0, 1.0)]] * S
        nst = len(st[0])
        jxy = np.array(st, dtype=np.float64).reshape(S * nst, 3)
        s_idx = np.repeat(np.arange(S), nst)
        vkey = repr(v)
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
            clears[k] = clear_throughput(src, v, float(n_img), vector, m_scale)
            if mirror is not None:
                mirror_rows[k] = (v.wavelength, v.reduction, multilayer.SOURCE_TILT_SIGN, cxs, cys,
                                  mirror.theta.size, m_idx, 0)
            m = S * nst
            skey = (vkey, float(dz), float(n_img))
            base = slot_of_state.get(skey)
            if base is None:
                base = n_tab
                slot_of_state[skey] = base
                slot_reps.append(n_jobs + np.arange(m, dtype=np.int32))
                n_tab += m
            cols["fsx"].append(src.fx[s_idx]); cols["fsy"].append(src.fy[s_idx])
            cols["jx"].append(jxy[:, 0]); cols["jy"].append(jxy[:, 1])
            cols["weight"].append(src.weight[s_idx] * jxy[:, 2])
            cols["pupil"].append(np.full(m, k)); cols["clip"].append(np.full(m, c))
            cols["out"].append(np.full(m, k))
            cols["cx"].append(np.rint(src.fx / val).astype(np.int64)[s_idx])
            cols["cy"].append(np.rint(src.fy / val).astype(np.int64)[s_idx])
            cols["ncomp"].append(np.full(m, 3 if vector else 1))
            cols["tab"].append(base + np.arange(m))
            n_jobs += m
    jobs = np.zeros(n_jobs, dtype=nat.JOB_DTYPE)
    for name in nat.JOB_DTYPE.names:
        jobs[name] = np.concatenate(cols[name]).astype(nat.JOB_DTYPE[name])
    slots = np.concatenate(slot_reps).astype(np.int32)
    # jobs are grouped by output (k); chunk each output's run into work items
    # (0: as many jobs per item as keeps about two waves of blocks, at most 32)
    n_out = C * P
    L = coarse_grid(h)
    if items_per_job_group:
        per = int(items_per_job_group)
    elif L > 64:
        per = 8   # wide engine: one partial L x L image per item
    else:
        per = min(32, max(1, n_jobs // (2 * 4 * 148)))
    starts = np.searchsorted(jobs["out"], np.arange(n_out + 1), side="left")
    item_rows, out_items = [], [0]
    for o in range(n_out):
        b0, e0 = int(starts[o]), int(starts[o + 1])
        for j in range(b0, e0, per):
            item_rows.append((o, j, min(j + per, e0), 0))
        out_items.append(len(item_rows))
    items = np.array(item_rows, dtype=np.int32).view(nat.ITEM_DTYPE).reshape(-1)
    out_items = np.array(out_items, dtype=np.int32)
    norm = np.zeros(n_out, dtype=nat.NORM_DTYPE)
    for c, v in enumerate(views):
        for p in range(P):
            k = c * P + p
            if return_raw:
                norm[k] = (0, 1.0)
            elif v.normalisation.lower() == "peak":
                norm[k] = (1, dose)
            else:
                norm[k] = (0, normalisation_scale(v.normalisation, 1.0, clears[k], dose))
    bm = int(max(np.abs(jobs["cx"]).max(), np.abs(jobs["cy"]).max())) + h
    arrays = [jobs, pupils, items, out_items, norm, slots]
    if mirror_tabs:
        arrays.append(_mirror_segment(mirror_rows, mirror_tabs))
    blob, offs = nat.blob(arrays)
    plan = nat.AbbePlan(
        n=n, n_clips=C, n_out=n_out, n_jobs=n_jobs, n_items=len(items), n_pupils=len(pupils),
        h=h, bm=bm, L=L, mask_complex=int(mask_complex), ncomp_max=3 if vec_any else 1, n_tab=n_tab,
        pixel_size=pixel_size, off_jobs=offs[0], off_pupils=offs[1], off_items=offs[2],
        off_out_items=offs[3], off_norm=offs[4], off_slots=offs[5],
        mirrored=int(bool(mirror_tabs)), off_mirrors=offs[6] if mirror_tabs else 0)
    transforms = int(np.sum(jobs["ncomp"]))
    return AbbePlanData(plan, blob, clears, n_out, n_jobs, transforms)


def _mirror_segment(rows: np.ndarray, tabs: list) -> np.ndarray:
    """LithoMirror[n_pupils] followed by each distinct reflection table
    (float64 theta, |r|, arg r), 16-byte aligned; rows' ``pad`` field holds
    the table index on entry and is cleared here."""
    head = (rows.nbytes + 15) & ~15
    offs, size = [], head
    for t in tabs:
        offs.append(size)
        size += (3 * t.theta.size * 8 + 15) & ~15
    seg = np.zeros(size, dtype=np.uint8)
    out = rows.copy()
    for k in range(out.size):
        if out[k]["n_theta"]:
            out[k]["off_table"] = offs[int(out[k]["pad"])]
        out[k]["pad"] = 0
    seg[:rows.nbytes] = out.view(np.uint8)
    for o, t in zip(offs, tabs):
        seg[o:o + 3 * t.theta.size * 8] = np.concatenate([t.theta, t.mag, t.phase]).astype("<f8").view(np.uint8)
    return seg


def plan_from_table(n: int, pixel_size: float, n_clips: int, weights, h: int, mask_complex: bool,
                    norm_mode=(0, 1.0), items_per_job_group: int = 0) -> AbbePlanData:
    """Plan that images every clip with K unshifted coherent systems whose
    spectra are given by a caller-built table (the SOCS forward,
    hopkins.py:215-217): job (clip c, kernel k) has weight weights[k] and
    table slot k; there is no pupil to evaluate."""
    K = len(weights)
    if K == 0:
        raise ValueError("no kernels to image with")
    L = coarse_grid(h)
    jobs = np.zeros(n_clips * K, dtype=nat.JOB_DTYPE)
    jobs["weight"] = np.tile(np.asarray(weights, dtype=np.float64), n_clips)
    jobs["clip"] = np.repeat(np.arange(n_clips), K)
    jobs["out"] = jobs["clip"]
    jobs["ncomp"] = 1
    jobs["tab"] = np.tile(np.arange(K), n_clips)
    pupils = np.zeros(1, dtype=nat.PUPIL_DTYPE)
    pupils["wavelength"], pupils["NA"], pupils["n_image"] = 1.0, 1.0, 1.0
    slots = np.arange(K, dtype=np.int32)
    # 0: two jobs per item (one per warp of the L = 64 kernels) until there are
    # enough items to fill the GPU, then up to 8
    per = int(items_per_job_group) or (8 if L > 64 else min(8, max(2, (n_clips * K) // (4 * 148))))
    item_rows, out_items = [], [0]
    for c in range(n_clips):
        for j in range(c * K, (c + 1) * K, per):
            item_rows.append((c, j, min(j + per, (c + 1) * K), 0))
        out_items.append(len(item_rows))
    items = np.array(item_rows, dtype=np.int32).view(nat.ITEM_DTYPE).reshape(-1)
    out_items = np.array(out_items, dtype=np.int32)
    norm = np.zeros(n_clips, dtype=nat.NORM_DTYPE)
    norm["mode"], norm["scale"] = norm_mode
    blob, offs = nat.blob([jobs, pupils, items, out_items, norm, slots])
    plan = nat.AbbePlan(
        n=n, n_clips=n_clips, n_out=n_clips, n_jobs=len(jobs), n_items=len(items), n_pupils=1, h=h, bm=h, L=L,
        mask_complex=int(mask_complex), ncomp_max=1, n_tab=K, pixel_size=pixel_size, off_jobs=offs[0],
        off_pupils=offs[1], off_items=offs[2], off_out_items=offs[3], off_norm=offs[4], off_slots=offs[5])
    return AbbePlanData(plan, blob, np.zeros(n_clips), n_clips, len(jobs), len(jobs))


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


ENGINES = ("fused", "plain")


def pupil_table(pd: AbbePlanData, dev, stream: int):
    """The plan's pupil table on `dev`, built once (it depends on the optics
    and source only) and kept with the plan."""
    torch = nat.require_cuda()
    t = getattr(pd, "_table_dev", None)
    if t is not None and t.device == dev:
        return t
    import ctypes as C
    L = nat.lib()
    nb = C.c_size_t(0)
    nat.check("litho_abbe_table_bytes", L.litho_abbe_table_bytes(C.byref(pd.plan), C.byref(nb)))
    t = torch.empty(max(nb.value, 16), dtype=torch.uint8, device=dev)
    blob = getattr(pd, "_blob_dev", None)
    if blob is None or blob.device != dev:
        blob = torch.from_numpy(pd.blob).to(dev)
        pd._blob_dev = blob
    nat.check("litho_abbe_pupil_table", L.litho_abbe_pupil_table(C.byref(pd.plan), blob.data_ptr(),
                                                                  t.data_ptr(), stream))
    pd._table_dev = t
    return t


def plain_batch_size(pd: AbbePlanData, budget_bytes: int = 2 << 30) -> int:
    """Coherent systems the plain engine transforms per batch (HBM budget)."""
    per = pd.plan.ncomp_max * pd.plan.n * pd.plan.n * 8
    return int(max(1, min(pd.jobs, budget_bytes // per)))


def run_abbe(pd: AbbePlanData, masks_dev, out=None, peak=None, stream=None, engine: str = "fused"):
    """Launch one planned Abbe batch; returns (images (n_out, N, N), peaks (n_out,)).

    engine "fused" is the band-limited on-chip engine; "plain" transforms every
    coherent system on the full N x N grid (the comparison baseline)."""
    torch = nat.require_cuda()
    L = nat.lib()
    dev = masks_dev.device
    n = pd.plan.n
    if engine not in ENGINES:
        raise ValueError(f"engine must be one of {ENGINES}, got {engine!r}")
    if engine == "fused" and not fused_supported(n, int(pd.plan.L)):
        engine = "plain"   # pupil wider than the grid allows a coarse grid for: full-grid GPU engine
    if out is None:
        out = torch.empty((pd.n_out, n, n), dtype=torch.float32, device=dev)
    if peak is None:
        peak = torch.empty((pd.n_out,), dtype=torch.float32, device=dev)
    import ctypes as C
    ws_bytes = C.c_size_t(0)
    if engine == "fused":
        nat.check("litho_abbe_workspace", L.litho_abbe_workspace(C.byref(pd.plan), C.byref(ws_bytes)))
    else:
        batch = plain_batch_size(pd)
        nat.check("litho_abbe_plain_workspace",
                  L.litho_abbe_plain_workspace(C.byref(pd.plan), batch, C.byref(ws_bytes)))
    ws = nat.Workspace.get(torch, dev, ws_bytes.value, tag=engine)
    blob = getattr(pd, "_blob_dev", None)
    if blob is None or blob.device != dev:
        blob = torch.from_numpy(pd.blob).to(dev)
        pd._blob_dev = blob
    s = stream if stream is not None else nat.stream_ptr(torch, dev)
    if engine == "fused":
        table = pupil_table(pd, dev, s)
        nat.check("litho_abbe_tabled", L.litho_abbe_tabled(C.byref(pd.plan), blob.data_ptr(), table.data_ptr(),
                                                            masks_dev.data_ptr(), out.data_ptr(), peak.data_ptr(),
                                                            ws.data_ptr(), ws.numel(), s))
    else:
        nat.check("litho_abbe_plain", L.litho_abbe_plain(C.byref(pd.plan), batch, blob.data_ptr(),
                                                          masks_dev.data_ptr(), out.data_ptr(),
                                                          peak.data_ptr(), ws.data_ptr(), ws.numel(), s))
    return out, peak


SYNTHESIS = ("direct", "row_pairs", "tensor_cores", "wide")


class LevelMasks:
    """Masks given as level maps: ``index`` (C, N, N) uint8 (numpy or a torch
    tensor, any device) indexing each clip's complex ``levels`` (C, n_levels),
    n_levels <= 256. Binary masks (0/1) and attenuated phase-shift masks
    (1 and sqrt(T) e^{i phase}, mask/patterns.py) have two levels, so a clip
    travels to the device and through HBM at one byte per pixel instead of
    eight; the images are those of the complex masks the levels spell out."""

    def __init__(self, index, levels):
        self.index = index
        self.levels = np.asarray(levels, dtype=np.complex64) if not _is_torch(levels) else levels
        shape = tuple(index.shape)
        if len(shape) != 3 or shape[1] != shape[2]:
            raise ValueError(f"index must be (C, N, N), got {shape}")
        lv = tuple(self.levels.shape)
        if len(lv) != 2 or lv[0] != shape[0] or not 1 <= lv[1] <= 256:
            raise ValueError(f"levels must be ({shape[0]}, n_levels <= 256), got {lv}")

    @staticmethod
    def from_masks(masks, max_levels: int = 256) -> "LevelMasks":
        """Factor (C, N, N) masks (host arrays) into a level map and each
        clip's distinct values; raises ValueError past ``max_levels``."""
        m = np.asarray(masks)
        if m.ndim == 2:
            m = m[None]
        C = m.shape[0]
        index = np.empty(m.shape, dtype=np.uint8)
        uniq = []
        for c in range(C):
            u, inv = np.unique(m[c].astype(np.complex64).ravel(), return_inverse=True)
            if u.size > max_levels:
                raise ValueError(f"clip {c} has {u.size} distinct values, more than {max_levels} levels")
            uniq.append(u)
            index[c] = inv.reshape(m.shape[1:]).astype(np.uint8)
        nl = max(u.size for u in uniq)
        levels = np.zeros((C, nl), dtype=np.complex64)
        for c, u in enumerate(uniq):
            levels[c, :u.size] = u
        return LevelMasks(index, levels)

    def expand(self) -> np.ndarray:
        """The complex64 masks (host) the levels spell out."""
        idx = self.index.cpu().numpy() if _is_torch(self.index) else np.asarray(self.index)
        lv = self.levels.cpu().numpy() if _is_torch(self.levels) else self.levels
        return np.take_along_axis(lv[:, None, :], idx.reshape(idx.shape[0], 1, -1).astype(np.int64),
                                  axis=2).reshape(idx.shape).astype(np.complex64)


def run_abbe_levels(pd: AbbePlanData, index_dev, levels_dev, out=None, peak=None, stream=None):
    """``run_abbe`` for level-map masks (``litho_abbe_levels``): index_dev
    (C, N, N) uint8 and levels_dev (C, n_levels) complex64 on the device."""
    torch = nat.require_cuda()
    L = nat.lib()
    dev = index_dev.device
    n = pd.plan.n
    if index_dev.dtype != torch.uint8 or tuple(index_dev.shape) != (pd.plan.n_clips, n, n):
        raise ValueError(f"index must be uint8 {(pd.plan.n_clips, n, n)}, got {index_dev.dtype} {tuple(index_dev.shape)}")
    if levels_dev.dtype != torch.complex64 or levels_dev.dim() != 2 or levels_dev.shape[0] != pd.plan.n_clips:
        raise ValueError("levels must be complex64 (n_clips, n_levels)")
    if out is None:
        out = torch.empty((pd.n_out, n, n), dtype=torch.float32, device=dev)
    if peak is None:
        peak = torch.empty((pd.n_out,), dtype=torch.float32, device=dev)
    import ctypes as C
    ws_bytes = C.c_size_t(0)
    nat.check("litho_abbe_workspace", L.litho_abbe_workspace(C.byref(pd.plan), C.byref(ws_bytes)))
    ws = nat.Workspace.get(torch, dev, ws_bytes.value, tag="fused")
    blob = getattr(pd, "_blob_dev", None)
    if blob is None or blob.device != dev:
        blob = torch.from_numpy(pd.blob).to(dev)
        pd._blob_dev = blob
    s = stream if stream is not None else nat.stream_ptr(torch, dev)
    table = pupil_table(pd, dev, s)
    lv = levels_dev.contiguous()
    nat.check("litho_abbe_levels", L.litho_abbe_levels(
        C.byref(pd.plan), blob.data_ptr(), table.data_ptr(), index_dev.data_ptr(), lv.data_ptr(), int(lv.shape[1]),
        out.data_ptr(), peak.data_ptr(), ws.data_ptr(), ws.numel(), s))
    return out, peak


def engine_info(pd: AbbePlanData) -> dict:
    """Which engine and image synthesis ``run_abbe`` uses for this plan
    (``litho_abbe_engine``)."""
    info = (ctypes.c_int32 * 2)()
    nat.check("litho_abbe_engine", nat.lib().litho_abbe_engine(ctypes.byref(pd.plan), info, 2))
    return {"engine": "coarse" if info[0] == 1 else "wide", "synthesis": SYNTHESIS[info[1]]}


def check_status(pd: AbbePlanData, dev, engine: str = "fused", stream=None) -> None:
    """Synchronise and raise if a bounded wait inside the last fused Abbe
    call on this device's workspace gave up (its images are then invalid)."""
    if engine != "fused" or not fused_supported(pd.plan.n, int(pd.plan.L)):
        return
    torch = nat.require_cuda()
    ws = nat.Workspace.get(torch, dev, 0, tag="fused")
    s = stream if stream is not None else nat.stream_ptr(torch, dev)
    nat.check("litho_abbe_status", nat.lib().litho_abbe_status(ctypes.byref(pd.plan), ws.data_ptr(), s))


# Stage names of litho_abbe_profile. "peak_pass" is the compute-only synthesis
# pass of peak-normalised outputs (on grids without the pair-FFT synthesis it
# is the direct synthesis and "synthesis" the separate normalising pass).
STAGES = ("pupil_table", "band_rows", "band_cols", "coarse", "coarse_reduce", "peak_pass", "synthesis")


def profile_abbe(pd: AbbePlanData, masks_dev, reps: int = 10, rebuild_table: bool = False) -> dict:
    """Mean device milliseconds of each pipeline stage over `reps` runs
    (stage "pupil_table" is ~0 unless rebuild_table)."""
    torch = nat.require_cuda()
    import ctypes as C
    L = nat.lib()
    dev = masks_dev.device
    out = torch.empty((pd.n_out, pd.plan.n, pd.plan.n), dtype=torch.float32, device=dev)
    peak = torch.empty((pd.n_out,), dtype=torch.float32, device=dev)
    run_abbe(pd, masks_dev, out, peak)
    ws = nat.Workspace.get(torch, dev, 0, tag="fused")
    ms = (C.c_float * 8)()
    table = None if rebuild_table else pupil_table(pd, dev, nat.stream_ptr(torch, dev)).data_ptr()
    nat.check("litho_abbe_profile", L.litho_abbe_profile(
        C.byref(pd.plan), pd._blob_dev.data_ptr(), table, masks_dev.data_ptr(), out.data_ptr(),
        peak.data_ptr(), ws.data_ptr(), ws.numel(), nat.stream_ptr(torch, dev), int(reps), ms))
    return {name: float(ms[i]) for i, name in enumerate(STAGES)}


def _grid(grid):
    return int(grid.n_pixels), float(grid.pixel_size)


def compute_aerial_batch(masks, optics, grid, planes=None, dose: float = 1.0, return_raw: bool = False,
                         engine: str = "fused", check: bool | None = None):
    """Abbe images of a batch of clips on the GPU.

    masks: (C, N, N) numpy array or torch tensor (real or complex), or a
        :class:`LevelMasks` (one byte per pixel; the band-limited engines).
    optics: one optics object for all clips, or a sequence of C of them.
    planes: None (each clip's own defocus / image index), a list of
        (defocus, n_image) shared by all clips, or a list of C such lists.
    check: synchronise and raise ``LithoError`` (status ``LITHO_E_TIMEOUT``)
        if a bounded wait inside a kernel gave up; default: for host (numpy)
        masks, whose results are read on the host anyway; device masks keep
        the call asynchronous (call :func:`check_status` when needed).
    Returns (images, peaks, clears): images (C, P, N, N) float32 CUDA tensor,
    peaks (C, P) raw maxima, clears (C, P) float64 numpy.
    """
    torch = nat.require_cuda()
    n, px = _grid(grid)
    lev = masks if isinstance(masks, LevelMasks) else None
    if lev is not None:
        dev = torch.device("cuda", torch.cuda.current_device())
        idx = lev.index if _is_torch(lev.index) else torch.from_numpy(np.ascontiguousarray(lev.index))
        md = idx.to(dev, torch.uint8).contiguous()
        lv = lev.levels if _is_torch(lev.levels) else torch.from_numpy(np.ascontiguousarray(lev.levels))
        lvd = lv.to(dev, torch.complex64).contiguous()
        if tuple(md.shape[1:]) != (n, n):
            raise ValueError(f"masks must be (C, {n}, {n}) for this grid, got {tuple(md.shape)}")
    else:
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
    pd = plan_abbe(views, n, px, pl, dose, return_raw, True if lev is not None else md.is_complex())
    if lev is not None:
        if engine != "fused" or not fused_supported(n, int(pd.plan.L)) or int(pd.plan.L) > 64:
            raise ValueError("level-map masks run on the band-limited coarse-grid engine only; pass the complex "
                             "masks (LevelMasks.expand()) for this grid and pupil")
        img, pk = run_abbe_levels(pd, md, lvd)
    else:
        img, pk = run_abbe(pd, md, engine=engine)
    if check if check is not None else (lev is not None or not _is_torch(masks)):
        check_status(pd, md.device, engine)
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
