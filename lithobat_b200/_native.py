"""ctypes binding of liblitho_b200.so (the C ABI declared in include/litho_b200.h).

The library is built in-tree by ``lithobat_b200/csrc/build.py`` and loaded from
the package folder. There is no fallback: if the library or a CUDA device is
missing, every entry point raises :class:`NativeUnavailable`.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "liblitho_b200.so"


NOALLOC_SCRATCH_BYTES = 32 << 20   # LITHO_NOALLOC_SCRATCH_BYTES
LITHO_E_UNSUPPORTED = -5           # a valid request this build does not serve
LITHO_E_BAND = -4                  # band / coarse-grid geometry inconsistent


class NativeUnavailable(RuntimeError):
    """The sm_100a engine cannot run here (library not built, or no GPU)."""


class LithoError(RuntimeError):
    """A C-ABI entry point returned a non-zero status."""

    def __init__(self, fn: str, status: int, text: str):
        super().__init__(f"{fn} failed with status {status}: {text}")
        self.status = status


# --- struct layouts (must match include/litho_b200.h) ------------------------

PUPIL_DTYPE = np.dtype([
    ("wavelength", "<f8"), ("NA", "<f8"), ("defocus", "<f8"), ("n_image", "<f8"),
    ("zernike", "<f8", (21,)), ("exact_defocus", "<i4"), ("vector", "<i4"),
    ("obliquity", "<i4"), ("has_zernike", "<i4"),
], align=True)

JOB_DTYPE = np.dtype([
    ("fsx", "<f8"), ("fsy", "<f8"), ("jx", "<f8"), ("jy", "<f8"), ("weight", "<f8"),
    ("pupil", "<i4"), ("clip", "<i4"), ("out", "<i4"), ("cx", "<i4"), ("cy", "<i4"),
    ("ncomp", "<i4"), ("tab", "<i4"),
], align=True)

ITEM_DTYPE = np.dtype([("out", "<i4"), ("job_begin", "<i4"), ("job_end", "<i4"), ("pad", "<i4")])
NORM_DTYPE = np.dtype([("mode", "<i4"), ("scale", "<f4")])

assert PUPIL_DTYPE.itemsize == 216 and JOB_DTYPE.itemsize == 72


class AbbePlan(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("n_clips", C.c_int32), ("n_out", C.c_int32), ("n_jobs", C.c_int32),
        ("n_items", C.c_int32), ("n_pupils", C.c_int32), ("h", C.c_int32), ("bm", C.c_int32),
        ("L", C.c_int32), ("mask_complex", C.c_int32), ("ncomp_max", C.c_int32), ("n_tab", C.c_int32),
        ("pixel_size", C.c_double),
        ("off_jobs", C.c_int64), ("off_pupils", C.c_int64), ("off_items", C.c_int64),
        ("off_out_items", C.c_int64), ("off_norm", C.c_int64), ("off_slots", C.c_int64),
        ("mirrored", C.c_int32), ("pad_m", C.c_int32), ("off_mirrors", C.c_int64),
    ]


class UnevenGroup(C.Structure):
    _fields_ = [
        ("plan", AbbePlan), ("blob_host", C.c_void_p), ("blob_dev", C.c_void_p), ("table_dev", C.c_void_p),
        ("masks_dev", C.c_void_p), ("image_dev", C.c_void_p), ("peak_dev", C.c_void_p),
        ("workspace_dev", C.c_void_p), ("ws_bytes", C.c_size_t), ("slot_kib", C.c_int32), ("n_slots", C.c_int32),
        ("a_units", C.c_int32), ("b_rows", C.c_int32),
    ]


QUEUE_TASK_DTYPE = np.dtype([(k, "<i4") for k in (
    "kind", "group", "slot", "base", "first", "count", "rows", "wait_ctr", "wait_value", "done_ctr")])

MIRROR_DTYPE = np.dtype([
    ("wavelength", "<f8"), ("reduction", "<f8"), ("tilt_sign", "<f8"), ("sin_cx", "<f8"), ("sin_cy", "<f8"),
    ("n_theta", "<i4"), ("pad", "<i4"), ("off_table", "<i8"),
], align=True)

ILT_SCHED_DTYPE = np.dtype([
    ("beta", "<f8"), ("beta_next", "<f8"), ("growth", "<f8"), ("it", "<i4"), ("c1", "<f4"), ("c2", "<f4"),
    ("pad", "<i4"),
], align=True)

assert C.sizeof(AbbePlan) == 120 and MIRROR_DTYPE.itemsize == 56 and ILT_SCHED_DTYPE.itemsize == 40
assert C.sizeof(UnevenGroup) == 200 and QUEUE_TASK_DTYPE.itemsize == 40

_lib = None


def lib():
    """Load the engine once; raise NativeUnavailable if it cannot run."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise NativeUnavailable(
            f"{LIB_PATH.name} is not built; run `python lithobat_b200/csrc/build.py` "
            "(or __graft_entry__.build()) first")
    L = C.CDLL(str(LIB_PATH))
    L.litho_status_string.restype = C.c_char_p
    L.litho_status_string.argtypes = [C.c_int]
    L.litho_version.restype = C.c_int
    L.litho_abbe_workspace.argtypes = [C.POINTER(AbbePlan), C.POINTER(C.c_size_t)]
    L.litho_abbe.argtypes = [C.POINTER(AbbePlan), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                             C.c_void_p, C.c_size_t, C.c_void_p]
    L.litho_abbe_plain_workspace.argtypes = [C.POINTER(AbbePlan), C.c_int, C.POINTER(C.c_size_t)]
    L.litho_abbe_plain.argtypes = [C.POINTER(AbbePlan), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]
    L.litho_abbe_profile.argtypes = [C.POINTER(AbbePlan), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_int,
                                     C.POINTER(C.c_float)]
    L.litho_abbe_table_bytes.argtypes = [C.POINTER(AbbePlan), C.POINTER(C.c_size_t)]
    L.litho_abbe_pupil_table.argtypes = [C.POINTER(AbbePlan), C.c_void_p, C.c_void_p, C.c_void_p]
    L.litho_abbe_tabled.argtypes = [C.POINTER(AbbePlan), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]
    L.litho_abbe_status.argtypes = [C.POINTER(AbbePlan), C.c_void_p, C.c_void_p]
    L.litho_abbe_noalloc.argtypes = [C.POINTER(AbbePlan), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p]
    L.litho_socs_workspace.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_size_t)]
    L.litho_socs_build.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                   C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]
    L.litho_socs_status.argtypes = [C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_int), C.c_void_p]
    L.litho_socs_debug.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    for fn in ("litho_socs_workspace", "litho_socs_build", "litho_socs_status", "litho_socs_debug"):
        getattr(L, fn).restype = C.c_int
    vp, i32, f32, sz = C.c_void_p, C.c_int, C.c_float, C.c_size_t
    sigs = {
        "litho_coarse_image": [C.POINTER(AbbePlan), vp, vp, vp, vp, vp, sz, vp],
        "litho_abbe_levels": [C.POINTER(AbbePlan), vp, vp, vp, vp, i32, vp, vp, vp, sz, vp],
        "litho_abbe_engine": [C.POINTER(AbbePlan), vp, i32],
        "litho_abbe_noalloc_status": [C.POINTER(AbbePlan), vp],
        "litho_abbe_clear": [C.POINTER(AbbePlan), vp, vp, vp],
        "litho_socs_forward_workspace": [i32, i32, i32, i32, i32, C.POINTER(sz)],
        "litho_socs_forward": [vp, vp, i32, i32, vp, i32, i32, i32, i32, f32, vp, vp, vp, sz, vp],
        "litho_socs_backward_workspace": [i32, i32, i32, i32, C.POINTER(sz)],
        "litho_socs_backward": [vp, vp, i32, i32, vp, i32, i32, vp, f32, vp, vp, sz, vp],
        "litho_socs_tcc_bytes": [i32, i32, C.POINTER(sz)],
        "litho_socs_tcc_build": [vp, vp, i32, vp, vp, i32, i32, vp, sz, vp, vp],
        "litho_socs_tcc_image": [vp, i32, i32, vp, i32, vp, vp],
        "litho_socs_tcc_adjoint": [vp, i32, i32, vp, vp, i32, vp, vp],
        "litho_set_wait_limit": [C.c_longlong],
        "litho_wait_probe": [vp, C.c_longlong, vp],
        "litho_band_spectrum_workspace": [i32, i32, i32, C.POINTER(sz)],
        "litho_band_spectrum": [vp, i32, i32, i32, i32, f32, vp, vp, sz, vp],
        "litho_band_synthesis_workspace": [i32, i32, C.POINTER(sz)],
        "litho_band_synthesis": [vp, i32, i32, i32, i32, vp, vp, sz, vp],
        "litho_socs_adjoint_workspace": [i32, i32, i32, C.POINTER(sz)],
        "litho_socs_adjoint": [C.POINTER(AbbePlan), vp, vp, vp, vp, vp, vp, vp, sz, vp],
        "litho_ilt_objective": [vp, vp, i32, i32, f32, f32, f32, f32, vp, vp, vp, vp, i32, vp],
        "litho_ilt_image_objective_workspace": [i32, i32, i32, vp],
        "litho_ilt_image_objective": [vp, i32, i32, i32, vp, f32, f32, f32, f32, vp, vp, vp, vp, vp, sz, vp],
        "litho_ilt_image_objective_band_workspace": [i32, i32, i32, i32, vp],
        "litho_ilt_step_workspace": [i32, i32, i32, C.POINTER(sz)],
        "litho_ilt_step": [vp, i32, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, f32, f32, f32, f32, f32, f32, f32,
                           f32, vp, vp, vp, sz, vp],
        "litho_ilt_step_status": [i32, i32, i32, vp, vp],
        "litho_ilt_image_objective_band": [vp, i32, i32, i32, vp, f32, f32, f32, f32, i32, f32, vp, vp, vp, vp, vp,
                                           sz, vp],
        "litho_ilt_objective_totals": [vp, vp, i32, i32, f32, f32, f32, f32, vp, vp, vp, vp, i32, vp, vp, vp,
                                       vp],
        "litho_ilt_penalties": [vp, i32, i32, f32, f32, vp, vp, i32, vp],
        "litho_ilt_mask": [vp, C.c_longlong, f32, vp, vp],
        "litho_ilt_theta_grad": [vp, vp, C.c_longlong, f32, vp, vp],
        "litho_ilt_adam": [vp, C.c_longlong, f32, f32, f32, f32, i32, vp, vp, vp, vp],
        "litho_gaussian_blur": [vp, vp, vp, i32, i32, vp, i32, vp],
        "litho_ilt_update": [vp, C.c_longlong, f32, f32, f32, f32, f32, f32, i32, vp, vp, vp, vp, vp],
        "litho_ilt_update_sched": [vp, C.c_longlong, vp, f32, f32, f32, f32, vp, vp, vp, vp, vp],
        "litho_dose_stack": [vp, vp, vp, i32, i32, C.c_longlong, vp, i32, vp, vp],
        "litho_clamp": [vp, C.c_longlong, f32, f32, vp],
        "litho_depth_interp": [vp, i32, C.c_longlong, vp, vp, i32, vp, vp, vp],
        "litho_uneven_group_workspace": [C.POINTER(UnevenGroup), C.POINTER(sz)],
        "litho_uneven_schedule": [C.POINTER(UnevenGroup), i32, vp, i32, C.POINTER(i32), C.POINTER(i32)],
        "litho_uneven_queue_workspace": [i32, C.POINTER(sz)],
        "litho_uneven_run": [C.POINTER(UnevenGroup), i32, vp, i32, i32, vp, sz, vp],
        "litho_uneven_status": [vp, vp],
        "litho_plain_socs_workspace": [i32, i32, C.POINTER(sz)],
        "litho_plain_socs_forward": [vp, i32, i32, i32, vp, vp, vp, vp, i32, vp, vp, vp, sz, vp],
        "litho_plain_socs_adjoint": [vp, vp, i32, i32, i32, vp, vp, vp, vp, i32, vp, vp, sz, vp],
    }
    for fn, at in sigs.items():
        getattr(L, fn).argtypes = at
        getattr(L, fn).restype = C.c_int
    for fn in ("litho_abbe_workspace", "litho_abbe", "litho_abbe_plain_workspace", "litho_abbe_plain",
               "litho_abbe_profile", "litho_abbe_table_bytes", "litho_abbe_pupil_table",
               "litho_abbe_tabled", "litho_abbe_status", "litho_abbe_noalloc"):
        getattr(L, fn).restype = C.c_int
    _lib = L
    return L


def check(fn: str, status: int) -> None:
    if status != 0:
        raise LithoError(fn, status, lib().litho_status_string(status).decode())


def exported_symbols() -> list[str]:
    """Names the header declares; used by the ABI test."""
    hdr = Path(__file__).resolve().parent.parent / "include" / "litho_b200.h"
    import re
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\*?(litho_\w+)\s*\(", hdr.read_text(), re.M)))


def require_cuda():
    """torch with a visible CUDA device, or NativeUnavailable."""
    import torch
    if not torch.cuda.is_available():
        raise NativeUnavailable("no CUDA device is visible; the sm_100a engine has no CPU path")
    lib()
    return torch


def stream_ptr(torch, device=None) -> int:
    return int(torch.cuda.current_stream(device).cuda_stream)


class Workspace:
    """A grow-only device scratch buffer per (device, purpose)."""

    _bufs: dict = {}

    @classmethod
    def get(cls, torch, device, nbytes: int, tag: str = "main"):
        key = (str(device), tag)
        buf = cls._bufs.get(key)
        if buf is None or buf.numel() < nbytes:
            buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
            cls._bufs[key] = buf
        return buf


def blob(arrays: list[np.ndarray]) -> tuple[np.ndarray, list[int]]:
    """Pack structured arrays into one 16-byte-aligned byte blob; return offsets."""
    offs, size = [], 0
    for a in arrays:
        size = (size + 15) & ~15
        offs.append(size)
        size += a.nbytes
    out = np.zeros(max(size, 16), dtype=np.uint8)
    for a, o in zip(arrays, offs):
        out[o:o + a.nbytes] = np.frombuffer(np.ascontiguousarray(a).tobytes(), dtype=np.uint8)
    return out, offs


def env_flag(name: str, default: str = "") -> str:
    return os.environ.get(name, default)
