"""Process-window and print helpers on the GPU, on top of the imaging path.

* :func:`dose_focus_images` — the imaging part of
  ``analysis/process_window.py:sweep_dose_focus`` (:215-300): one Abbe sum
  per focus (here all foci are planes of one batched launch), every dose a
  rescale of its raw sum.
* :func:`apply_peb` — ``bake/peb.py:apply_peb`` (:24-70): Gaussian acid
  diffusion (scipy's reflect-mode filter, radius int(4 sigma + 0.5)),
  clipped to [0, 1].
* :func:`develop_threshold` — ``develop/resist.py:develop_field`` (:452-511)
  for the ``"threshold"`` model: (PEB-diffused aerial image, threshold).
* :func:`print_image` — ``opc/model.py:PrintModel.print`` (:228-245) after
  rasterisation: SOCS kernels when the optics allow them (``imaging="auto"``),
  the Abbe sum otherwise, then the dose and the threshold development.
* :func:`exposure_volume` — ``develop/resist3d.py:exposure_volume``
  (:113-193): the aerial image through the resist film, its optical planes
  in one batched Abbe launch and the depth interpolation onto the voxel
  planes on the device (``litho_depth_interp``).

numpy in -> numpy float64 out; torch CUDA in -> torch float32 CUDA out.
"""

from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _native as nat
from .aerial import _as_device_masks, _is_torch, compute_aerial_batch, normalisation_scale
from .config import NORMALISATIONS, optics_view

_MODES = {"none": 0, "peak": 1, "clear": 2}


def _with_normalisation(optics, normalisation):
    if normalisation is None:
        return optics
    if dataclasses.is_dataclass(optics):
        return dataclasses.replace(optics, normalisation=normalisation)
    import copy
    c = copy.copy(optics)
    c.normalisation = normalisation
    return c


def dose_focus_images(mask, optics, grid, doses, defoci_nm, normalisation: str | None = "clear"):
    """(F, D, N, N) aerial images for every defocus [nm] x dose.

    normalisation: the mode the sweep uses (the reference's default "clear":
    under "peak" the same dose number would deliver a different energy at
    every focus); None keeps the optics' own."""
    torch = nat.require_cuda()
    L = nat.lib()
    base = _with_normalisation(optics, normalisation)
    v = optics_view(base)
    mode = v.normalisation.lower()
    if mode not in NORMALISATIONS:
        raise ValueError(f"normalisation must be 'peak', 'clear' or 'none', got '{v.normalisation}'")
    defoci = [float(d) for d in defoci_nm]
    dz = [float(x) for x in doses]
    if not defoci or not dz:
        raise ValueError("need at least one defocus and one dose")
    n = int(grid.n_pixels)
    md = _as_device_masks(torch, mask, n)
    if md.shape[0] != 1:
        raise ValueError("dose_focus_images takes one mask")
    raw, peak, clear = compute_aerial_batch(md, base, grid, [(d * 1e-9, v.image_index) for d in defoci],
                                            return_raw=True)
    F, D = len(defoci), len(dz)
    dev = raw.device
    clear_d = torch.from_numpy(np.asarray(clear[0], dtype=np.float32)).to(dev)
    doses_d = torch.tensor(dz, dtype=torch.float32, device=dev)
    out = torch.empty((F, D, n, n), dtype=torch.float32, device=dev)
    nat.check("litho_dose_stack", L.litho_dose_stack(
        raw.data_ptr(), peak.data_ptr(), clear_d.data_ptr(), _MODES[mode], F, n * n, doses_d.data_ptr(), D,
        out.data_ptr(), nat.stream_ptr(torch, dev)))
    return out if _is_torch(mask) else out.cpu().numpy().astype(np.float64)


def apply_peb(pac_map, diffusion_sigma: float, pixel_size: float):
    """Gaussian PEB diffusion of a (ny, nx) map, clipped to [0, 1] (bake/peb.py:24-70)."""
    from .ilt import gaussian_weights
    torch = nat.require_cuda()
    L = nat.lib()
    nd = pac_map.dim() if _is_torch(pac_map) else np.ndim(pac_map)
    if nd != 2:
        raise ValueError(f"apply_peb expects a 2-D (ny, nx) map, got ndim={nd}; use apply_peb_3d for volumes.")
    if diffusion_sigma < 0:
        raise ValueError(f"diffusion_sigma must be >= 0, got {diffusion_sigma!r}")
    if pixel_size <= 0:
        raise ValueError(f"pixel_size must be > 0, got {pixel_size!r}")
    shape = tuple(pac_map.shape)
    if shape[0] != shape[1]:
        raise ValueError(f"the GPU PEB takes square maps, got {shape}")
    sigma_px = diffusion_sigma / pixel_size
    x = _as_device_masks(torch, pac_map, shape[0]).to(torch.float32)
    if sigma_px < 1e-3:
        out = x[0].clone()
    else:
        wt = gaussian_weights(sigma_px)
        w = torch.from_numpy(wt.astype(np.float32)).to(x.device)
        out = torch.empty_like(x)
        tmp = torch.empty_like(x)
        s = nat.stream_ptr(torch, x.device)
        nat.check("litho_gaussian_blur", L.litho_gaussian_blur(
            x.data_ptr(), out.data_ptr(), tmp.data_ptr(), 1, shape[0], w.data_ptr(), (wt.size - 1) // 2, s))
        nat.check("litho_clamp", L.litho_clamp(out.data_ptr(), out.numel(), 0.0, 1.0, s))
        out = out[0]
    return out if _is_torch(pac_map) else out.cpu().numpy().astype(np.float64)


def develop_threshold(aerial, cfg, grid, model: str = "threshold"):
    """(field, threshold) of the threshold resist model (develop/resist.py:452-511).

    cfg: any object with ``diffusion_sigma`` [m] and ``threshold`` (the
    reference's ResistConfig). The chemistry models ("mack", "car") are not
    part of this library."""
    if model != "threshold":
        if model in ("mack", "car"):
            raise NotImplementedError(f"resist model '{model}' is outside the accelerated imaging path; "
                                      "develop with the threshold model or on the CPU")
        raise ValueError(f"unknown resist model '{model}'")
    return apply_peb(aerial, float(cfg.diffusion_sigma), float(grid.pixel_size)), float(cfg.threshold)


def print_image(mask, optics, grid, resist, dose: float = 1.0, imaging: str = "auto", socs_tol: float = 1e-8,
                normalisation: str | None = "clear", kernels=None):
    """Image a rasterised mask and develop it: (aerial, field, level)
    (opc/model.py:PrintModel.print, :228-245, after its rasterisation).

    imaging: "auto" (SOCS kernels when the optics allow them, else Abbe),
    "socs" or "abbe"; kernels: prebuilt SOCSKernels for these optics/grid."""
    from .aerial import compute_aerial_image
    from .hopkins import SOCSKernels
    if imaging not in ("auto", "socs", "abbe"):
        raise ValueError(f"imaging must be 'auto', 'socs' or 'abbe', got '{imaging}'")
    o = _with_normalisation(optics, normalisation)
    v = optics_view(o)
    if imaging == "socs" and not SOCSKernels.supports(o):
        raise ValueError("imaging='socs' needs the scalar thin-mask process; got "
                         f"imaging_model={v.imaging_model!r}, mask_model={v.mask_model!r}")
    use_k = imaging == "socs" or (imaging == "auto" and SOCSKernels.supports(o))
    if use_k:
        k = kernels if kernels is not None else SOCSKernels.build(o, grid, tol=socs_tol)
        raw, peak, clear = k.raw(mask)
    else:
        raw, peak, clear = compute_aerial_image(mask, o, grid, return_raw=True)
    aerial = raw * normalisation_scale(v.normalisation, peak, clear, dose)
    fld, level = develop_threshold(aerial, resist, grid)
    return aerial, fld, level


def focus_reference_depth(resist) -> float:
    """Depth below the resist top that the optics' defocus refers to [m]
    (develop/resist3d.py:focus_reference_depth, :66-81)."""
    ref = resist.focus_reference
    if ref == "top":
        return 0.0
    if ref == "mid":
        return resist.thickness / 2.0
    if ref == "bottom":
        return resist.thickness
    raise ValueError(f"focus_reference must be 'top', 'mid', or 'bottom', got '{ref}'")


def effective_defocus(depth: float, optics, resist) -> float:
    """Defocus [m] of the plane ``depth`` metres below the resist top, in the
    immersion medium's units (develop/resist3d.py:effective_defocus, :84-110)."""
    d_ref = focus_reference_depth(resist)
    return optics.defocus - (depth - d_ref) * (optics.n_immersion / resist.n_resist)


def depth_intervals(z_query, depths):
    """For every query depth: (lower plane, upper plane, weight) of the linear
    interpolation np.interp(z, depths, f) takes, in FP64: the end values
    outside [depths[0], depths[-1]], else f[j] + w (f[j+1] - f[j]) on the
    interval with depths[j] <= z < depths[j+1]."""
    xp = np.asarray(depths, dtype=np.float64)
    z = np.asarray(z_query, dtype=np.float64).reshape(-1)
    last = xp.size - 1
    k = np.zeros((z.size, 2), dtype=np.int32)
    w = np.zeros(z.size, dtype=np.float64)
    if last == 0:
        return k, w
    hi = z >= xp[last]
    inside = (z > xp[0]) & ~hi
    j = np.clip(np.searchsorted(xp, z, side="right") - 1, 0, last - 1)
    k[hi] = last
    k[inside, 0] = j[inside]
    k[inside, 1] = j[inside] + 1
    w[inside] = (z[inside] - xp[j[inside]]) / (xp[j[inside] + 1] - xp[j[inside]])
    return k, w


def exposure_volume(mask, optics, grid, resist, dose: float = 1.0, check: bool | None = None):
    """(intensity, z): the aerial image through the resist film
    (develop/resist3d.py:exposure_volume, :113-193).

    ``grid.n_z_slices`` optical planes (at least 2, at most the voxel count)
    span the film top to bottom; each images at its effective defocus
    converted to resist units with the resist as the image medium
    (sin theta = NA / n_resist), all planes in one batched Abbe launch and
    each normalised on its own. They are interpolated linearly in depth onto
    the ``round(thickness / dz)`` voxel planes, iz = 0 at the bottom of the
    film. intensity: (nz, N, N), numpy float64 for a numpy mask, torch float32
    on the device for a torch CUDA mask; z: the voxel heights above the film
    bottom [m], numpy float64. ``resist``: the reference's ResistConfig or
    :class:`~lithobat_b200.config.ResistConfig` (thickness, n_resist,
    focus_reference). check: synchronise and raise ``LithoError`` if a
    device status word reports a failure; default: for host (numpy) masks,
    whose result is read on the host anyway (device masks keep the call
    asynchronous, as :func:`~lithobat_b200.aerial.compute_aerial_batch`)."""
    torch = nat.require_cuda()
    L = nat.lib()
    nz = max(int(round(resist.thickness / grid.dz)), 1)
    n_slices = int(np.clip(grid.n_z_slices, 2, nz))
    depths = np.linspace(0.0, resist.thickness, n_slices)
    index_ratio = resist.n_resist / optics.n_immersion
    planes = [(effective_defocus(float(d), optics, resist) * index_ratio, resist.n_resist) for d in depths]
    n = int(grid.n_pixels)
    md = _as_device_masks(torch, mask, n)
    if md.shape[0] != 1:
        raise ValueError("exposure_volume takes one mask")
    if check is None:
        check = not _is_torch(mask)
    img, _pk, _cl = compute_aerial_batch(md, optics, grid, planes, dose, False, check=check)
    stack = img[0].contiguous()                      # (n_slices, N, N)
    dev = stack.device
    z_depth = ((np.arange(nz) + 0.5) * grid.dz)[::-1]   # depth below the top, bottom voxel first
    k, w = depth_intervals(z_depth, depths)
    k_d = torch.from_numpy(k.reshape(-1)).to(dev)
    w_d = torch.from_numpy(w.astype(np.float32)).to(dev)
    status = torch.zeros((1,), dtype=torch.int32, device=dev)
    out = torch.empty((nz, n, n), dtype=torch.float32, device=dev)
    nat.check("litho_depth_interp", L.litho_depth_interp(
        stack.data_ptr(), n_slices, n * n, k_d.data_ptr(), w_d.data_ptr(), nz, out.data_ptr(), status.data_ptr(),
        nat.stream_ptr(torch, dev)))
    if check:
        nat.check("litho_depth_interp", int(status.item()))
    z = (np.arange(nz) + 0.5) * grid.dz
    return (out if _is_torch(mask) else out.cpu().numpy().astype(np.float64)), np.asarray(z, dtype=np.float64)


__all__ = ["dose_focus_images", "apply_peb", "develop_threshold", "print_image", "focus_reference_depth",
           "effective_defocus", "depth_intervals", "exposure_volume"]
