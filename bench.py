"""Benchmark of the imaging hot path on B200s (one process per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python -m torch.distributed.run --nproc-per-node N bench.py --gpus N ...

Workload (one step, per GPU): a batch of 512 seeded 1024 x 1024 clips at 1 nm —
6 %-transmission attenuated phase-shift masks (phase pi) of contact-hole
arrays, pitch 80-140 nm, hole 40-70 nm — imaged with the vector (Ex, Ey, Ez)
Abbe model, NA 1.35 water immersion, azimuthal (TE) polarisation, annular
source sigma 0.5-0.9 sampled on a 31 x 31 grid (400 source points, 1200
coherent transforms per image), peak normalisation. Each rank images its own
clips (weak scaling, no collective on the data path).

Prints one JSON line (rank 0). ``value`` is whole-job images/s with inputs
resident in HBM; ``e2e`` is the same metric through the public host-to-host
API (``lithobat_b200.pipeline.AbbePipeline``) from pinned host buffers, the
H2D and D2H copies inside the timed region. Extra keys time the other
workloads (``c1``, ``c2``, ``ilt``, ``uneven``). ``cpu_baseline`` is one whole
workload image through the FP64 numpy restatement of the reference's
algorithm (``oracle/``) on the host cores; its output is also the FP64
reference of ``max_rel_err_vs_fp64`` (one image of the timed batch).
``--impl reference`` times that CPU algorithm for the reference arm: every
step a bounded sample (a fixed set of the image's source points), reported
as images/s of the work the step really did.
"""

from __future__ import annotations

import argparse
import dataclasses
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Abbe images/s & ILT grad-steps/s @1024² fused vs plain, 1 B200, err≤1e-5"
N, PX = 1024, 1e-9
IMAGES_PER_STEP = 512    # one batched call per step
ROTATE = 2               # distinct input batches of 4 GiB each (> 126 MiB L2)
E2E_IMAGES = 64          # images per public-API call in the end-to-end measurement
PLAIN_IMAGES = 8         # images per call of the plain (full-grid) comparison engine
WORKLOAD = ("vector Abbe 1024^2 @1 nm, NA 1.35/1.44 TE, annular 0.5-0.9 (source_grid 31, 400 pts), "
            "6% att-PSM contact holes")


def optics_c3():
    import lithobat_b200 as lb
    return lb.OpticsConfig(NA=1.35, n_immersion=1.44, imaging_model="vector", polarisation="te",
                           source_type="annular", sigma_inner=0.5, sigma_outer=0.9, source_grid=31)


def masks_c3(seed: int, count: int) -> np.ndarray:
    from lithobat_b200 import patterns
    rng = np.random.default_rng(seed)
    out = np.empty((count, N, N), dtype=np.complex64)
    for i in range(count):
        p = rng.uniform(80e-9, 140e-9)
        hole = rng.uniform(40e-9, 70e-9)
        c = patterns.contact_array(N, PX, p, p, hole)
        out[i] = patterns.to_attenuated_psm(1.0 - c, 0.06, 180.0)
    return out


def masks_c3_device(torch, seed: int, count: int, dev):
    """The same seeded clip family, generated on the device (complex64)."""
    g = torch.Generator(device="cpu").manual_seed(seed)
    pitch = 80e-9 + 60e-9 * torch.rand(count, generator=g, dtype=torch.float64)
    hole = 40e-9 + 30e-9 * torch.rand(count, generator=g, dtype=torch.float64)
    coords = ((torch.arange(N, dtype=torch.float64) - N // 2) * PX).to(dev)
    p, h = pitch.to(dev)[:, None], hole.to(dev)[:, None]
    opened = (torch.remainder(coords[None, :] + p / 2, p) < h).to(torch.float32)   # (count, N)
    chrome = 1.0 - opened[:, :, None] * opened[:, None, :]
    absorber = torch.tensor(complex(np.sqrt(0.06) * np.exp(1j * np.pi)), dtype=torch.complex64, device=dev)
    one = torch.ones((), dtype=torch.complex64, device=dev)
    return torch.where(chrome > 0.5, absorber, one).contiguous()


ILT_CLIPS = 16
ILT_WORKLOAD = ("ILT 1024^2 @1 nm x16 clips, ArF-imm annular 0.5-0.8 (124 pts), SOCS K=24 (TCC Gram on "
                "tensor cores, FP64 eig), resist level 0.3 a=50, clear normalisation, Adam")


def ilt_optics():
    import lithobat_b200 as lb
    return lb.OpticsConfig(wavelength=193e-9, NA=1.35, n_immersion=1.44, source_type="annular",
                           sigma_inner=0.5, sigma_outer=0.8, normalisation="clear")


def ilt_inputs(seed: int, count: int):
    from lithobat_b200 import patterns
    rng = np.random.default_rng(seed)
    targets = np.stack([patterns.manhattan_clip(rng, N, PX) for _ in range(count)]).astype(np.float32)
    theta = (0.5 * rng.standard_normal((count, N, N))).astype(np.float32)
    return targets, theta


def bench_ilt(args, torch, dev, world, max_over_ranks, barrier) -> dict:
    """ILT gradient steps/s: the fused band-limited iteration and the plain one."""
    import lithobat_b200 as lb
    from lithobat_b200 import ilt
    rank = int(os.environ.get("RANK", "0"))
    g = lb.GridConfig(n_pixels=N, pixel_size=PX)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lb.SOCSKernels.build(ilt_optics(), g, tol=0.0, max_kernels=24)  # warm
    torch.cuda.synchronize()
    e0.record()
    k = lb.SOCSKernels.build(ilt_optics(), g, tol=0.0, max_kernels=24)
    e1.record()
    torch.cuda.synchronize()
    build_ms = e0.elapsed_time(e1)
    nclip = args.ilt_clips
    targets, theta = ilt_inputs(500 + rank, nclip)
    params = ilt.IltParams(scale=1.0 / k.clear, level=0.3, steepness=15.0, step=0.4, beta=4.0, growth=1.0)
    b = ilt.IltBatch(k, torch.from_numpy(targets).to(dev), torch.from_numpy(theta).to(dev), params)
    for _ in range(args.warmup):
        b.step(want_signed=False)
    b.run(1)              # records the step as a CUDA graph (replayed below), outside the timed region
    torch.cuda.synchronize()
    barrier()
    e0.record()
    b.run(args.steps)
    e1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1))
    b.check_status()
    value = world * nclip * args.steps / (ms / 1000.0)
    # stage times of one step (events on the launching stream)
    st = b.st
    nat_ = __import__("lithobat_b200._native", fromlist=["x"])
    if b.fast:
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(8)]
        th, m1, m2 = b.theta.clone(), b.m1.clone(), b.m2.clone()
        mk = torch.empty_like(th)
        cpart = torch.empty((nclip, 64), dtype=torch.float64, device=dev)
        ppart = torch.empty((nclip, 64), dtype=torch.int32, device=dev)
        for _rep in range(2):   # the first pass sizes workspaces and loads kernels; the second is timed
            # a device-side delay ahead of the stages, so the host has queued
            # every stage before the GPU reaches it: the events then time the
            # kernels, not the Python launch gaps between them
            torch.cuda._sleep(4_000_000)
            ev[0].record()
            gm = st.synth(b.hbox, st.h, False)
            ev[1].record()
            nat_.check("update", st.L.litho_ilt_update(gm.data_ptr(), gm.numel(), b.beta, b.beta, 0.4, 0.9, 0.999,
                                                       1e-8, 5, th.data_ptr(), m1.data_ptr(), m2.data_ptr(),
                                                       mk.data_ptr(), st.stream()))
            ev[2].record()
            mbox = st.mask_box(mk)
            ev[3].record()
            ibox = st.image_box(mbox)
            ev[4].record()
            # the step's own objective call: synthesis + resist objective + the
            # band of dJ/dI in one pass when the band form serves the grid
            _c, gbox, _s, _p = st.objective_from_box(ibox, b.target, float(params.scale), 0.3, 1.0,
                                                     float(params.steepness), want_signed=False)
            ev[5].record()
            ev[6].record()
            st.adjoint_box(gbox, mbox)
            ev[7].record()
            torch.cuda.synchronize()
        names = ["gradient_synthesis", "theta_grad+adam+mask", "mask_band_spectrum",
                 "image_band_box (band TCC)", "image synthesis + objective + dJ/dI band box",
                 "(in the previous stage)", "adjoint: gradient band box (band TCC)"]
    else:
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(9)]
        ev[0].record()
        gt = st.grad_theta(b.grad_m, b.mask, b.beta, 0.0)
        ev[1].record()
        th = b.theta.clone(); m1 = b.m1.clone(); m2 = b.m2.clone()
        nat_.check("adam", st.L.litho_ilt_adam(gt.data_ptr(), gt.numel(), 0.4, 0.9, 0.999, 1e-8, 5, th.data_ptr(),
                                               m1.data_ptr(), m2.data_ptr(), st.stream()))
        mk = st.mask_of(th, b.beta, 0.0)
        ev[2].record()
        mbox = st.mask_box(mk)
        ev[3].record()
        raw = st.image(mbox)
        ev[4].record()
        dfield = torch.empty_like(raw)
        cpart = torch.empty((nclip, 64), dtype=torch.float64, device=dev)
        ppart = torch.empty((nclip, 64), dtype=torch.int32, device=dev)
        nat_.check("obj", st.L.litho_ilt_objective(raw.data_ptr(), b.target.data_ptr(), nclip, N,
                                                   float(params.scale), 0.3, 1.0, 50.0, dfield.data_ptr(), None,
                                                   cpart.data_ptr(), ppart.data_ptr(), 64, st.stream()))
        ev[5].record()
        st.band(dfield, 2 * st.h, float(params.scale) / (N * N))
        ev[6].record()
        st.adjoint(dfield, scale=float(params.scale), mbox=mbox)
        ev[7].record()
        torch.cuda.synchronize()
        names = ["grad_theta", "adam_and_mask", "mask_band_spectrum", "coarse_image_and_synthesis", "objective",
                 "sensitivity_band_spectrum", "adjoint_band_spectrum+coarse+synthesis"]
    stages = {nm: ev[i].elapsed_time(ev[i + 1]) for i, nm in enumerate(names)}
    plain = None
    if "iltplain" not in args.skip:
        # plain engine, same inputs
        pb = ilt.IltBatch(k, torch.from_numpy(targets).to(dev), torch.from_numpy(theta).to(dev), params,
                          engine="plain")
        fb = ilt.IltBatch(k, torch.from_numpy(targets).to(dev), torch.from_numpy(theta).to(dev), params)
        agree = float(((fb.grad_m.double() - pb.grad_m.double()).abs().amax(dim=(1, 2))
                       / pb.grad_m.double().abs().amax(dim=(1, 2))).max())
        pb.step(want_signed=False)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(2):
            pb.step(want_signed=False)
        e1.record()
        torch.cuda.synchronize()
        plain_ms = max_over_ranks(e0.elapsed_time(e1) / 2)
        plain_value = world * nclip / (plain_ms / 1000.0)
        plain = {"value": plain_value, "unit": "clip-steps/s", "fused_over_plain": value / plain_value,
                 "max_rel_diff_grad_fused_vs_plain": agree}
        del pb, fb
    # end to end from pinned host memory: upload theta/targets, K steps through
    # IltBatch.run (the graph is recorded inside the timed region), every
    # step's costs read back to the host, download theta
    tp = torch.from_numpy(targets).pin_memory()
    hp = torch.from_numpy(theta).pin_memory()
    out = torch.empty_like(hp).pin_memory()
    # one untimed pass of the same calls first (a batch built, stepped through
    # its graph recording and released), so the timed pass meets a warm
    # process as the other legs do: kernels loaded, allocator pools in place
    wb = ilt.IltBatch(k, tp.to(dev, non_blocking=True), hp.to(dev, non_blocking=True), params)
    for _ in range(max(args.warmup, 3)):
        wb.run(1)
    float(wb.cost.sum())
    del wb
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0.record()
    eb = ilt.IltBatch(k, tp.to(dev, non_blocking=True), hp.to(dev, non_blocking=True), params)
    # every step's costs come back to pinned host memory; the host reads step
    # i's total once step i + 1 is queued, so the read overlaps the next step
    costs_h = [torch.empty((nclip,), dtype=torch.float64).pin_memory() for _ in range(2)]
    done = [None, None]
    totals = []
    for i in range(args.steps):
        eb.run(1)                  # the public stepping call: graph-recorded on first use, then replayed
        costs_h[i % 2].copy_(eb.cost, non_blocking=True)
        done[i % 2] = torch.cuda.Event()
        done[i % 2].record()
        if i > 0:
            done[(i - 1) % 2].synchronize()
            totals.append(float(costs_h[(i - 1) % 2].sum()))
    done[(args.steps - 1) % 2].synchronize()
    totals.append(float(costs_h[(args.steps - 1) % 2].sum()))
    out.copy_(eb.theta)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1000.0))
    NN = N * N
    # the FP64 check of one clip at the batch's initial state (same 16-clip stages)
    chk = ilt.IltBatch(k, torch.from_numpy(targets).to(dev), torch.from_numpy(theta).to(dev), params)
    chk.check_status()
    fp64_case = {"target": targets[0], "theta": theta[0], "beta": float(params.beta),
                 "cost": float(chk.cost[0]), "grad": chk.grad_m[0].double().cpu().numpy()}
    del chk
    # algorithmic bytes of one fast step per clip pixel: gradient synthesis
    # writes g (4); the update reads g and theta, m1, m2 (16) and writes
    # theta, m1, m2 and the mask (16); the mask's band rows read it (4); the
    # image objective reads the target (4) and, unless it forms dJ/dI's band
    # rows itself (litho_ilt_image_objective_band), writes dJ/dI (4) for the
    # band rows to read (4). Band boxes and kernel tables are below 0.1 %.
    ilt_bytes = {"gradient_write": 4, "update_read": 16, "update_write": 16, "mask_band_read": 4,
                 "objective_target_read": 4}
    if not b.st.image_objective_band_ok():
        ilt_bytes.update({"objective_dJdI_write": 4, "sensitivity_band_read": 4})
    per_px = sum(ilt_bytes.values())
    hbm = float(measured_peaks()["hbm_gbs"])
    ach = per_px * NN * nclip / (ms / args.steps / 1000.0) / 1e9
    upd_ms = stages.get("theta_grad+adam+mask")
    roof = {"bound": "hbm", "kernel": "whole step (graph replay)", "achieved": ach, "peak": hbm, "unit": "GB/s",
            "frac": ach / hbm, "bytes_per_clip_pixel": ilt_bytes, "bytes_per_step": per_px * NN * nclip}
    if upd_ms:
        roof["update_kernel"] = {"bytes_per_launch": 32 * NN * nclip, "ms": upd_ms,
                                 "frac": 32 * NN * nclip / (upd_ms / 1000.0) / 1e9 / hbm}
    return {
        "_fp64_case": fp64_case, "roofline": roof,
        "metric": "ILT gradient steps/s @1024^2 (clip-steps)", "value": value, "unit": "clip-steps/s",
        "ms_per_step": ms / args.steps, "clips_per_step": nclip, "workload": ILT_WORKLOAD,
        "kernels": len(k), "socs_build_ms": build_ms, "fast_step": bool(b.fast),
        "graph_replay": b._graph is not None, "stages_ms": stages,
        "plain": plain,
        "e2e": {"value": world * nclip * args.steps / (e2e_ms / 1000.0), "unit": "clip-steps/s",
                "h2d_bytes_per_step": 2 * nclip * NN * 4 // args.steps, "d2h_bytes_per_step":
                nclip * 8 + nclip * NN * 4 // args.steps},
        "dense_fft_equivalent_bytes_per_clip_step": NN * (16 * (2 * len(k) + 2) + 40),
    }


UNEVEN_WORKLOAD = ("uneven EUV batch: 256 seeded Manhattan clips, sizes 256^2/512^2/1024^2/2048^2 at weights "
                   "4:3:2:1, 2 nm pixels, lambda 13.5 nm NA 0.33, dipole 0.6-0.9 +-30 deg (source_grid 43)")


def uneven_optics():
    import lithobat_b200 as lb
    from lithobat_b200.source import Source
    return lb.OpticsConfig(wavelength=13.5e-9, NA=0.33, source_grid=43,
                           source_spec=Source.dipole(0.9, 0.6, opening_deg=60).to_dict())


def bench_next(args, torch, dev) -> dict:
    """Device times of the callers either side of the imaging path, each on a
    device-resident seeded input (1 warm-up call, then the mean of 3 timed
    calls by CUDA events): the exposure volume through a resist film, a
    dose-focus sweep, a threshold print through SOCS kernels and EUV imaging
    with the multilayer blank."""
    import dataclasses

    import lithobat_b200 as lb
    from lithobat_b200 import patterns, process

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {}
    g = lb.GridConfig(n_pixels=N, pixel_size=PX)
    mask = masks_c3_device(torch, 77, 1, dev)[0]
    r = lb.ResistConfig()                      # 100 nm film, n 1.70, focus at mid-film
    nz = int(round(r.thickness / g.dz))
    ms = timed(lambda: process.exposure_volume(mask, optics_c3(), g, r))
    out["exposure_volume"] = {
        "workload": f"one {N}^2 clip at 1 nm, vector TE annular 0.5-0.9 (400 source points), "
                    f"{g.n_z_slices} optical planes through a 100 nm film -> {nz} voxel planes at 2 nm",
        "ms": ms, "voxel_planes_per_s": nz / (ms / 1000.0),
        "api": "lithobat_b200.process.exposure_volume"}
    foci, doses = [float(f) for f in np.linspace(-75.0, 75.0, 11)], [0.85, 0.9, 1.0, 1.1, 1.15]
    ms = timed(lambda: process.dose_focus_images(mask, optics_c3(), g, doses, foci))
    out["dose_focus"] = {
        "workload": f"one {N}^2 clip, vector TE annular (400 source points), {len(foci)} foci x {len(doses)} doses",
        "ms": ms, "images_per_s": len(foci) * len(doses) / (ms / 1000.0),
        "api": "lithobat_b200.process.dose_focus_images"}
    ko = ilt_optics()
    k = lb.SOCSKernels.build(ko, g, tol=0.0, max_kernels=24)
    tgt = torch.from_numpy(patterns.manhattan_clip(np.random.default_rng(78), N, PX).astype(np.float32)).to(dev)
    ms = timed(lambda: process.print_image(tgt, ko, g, r, kernels=k))
    out["print_socs"] = {
        "workload": f"one {N}^2 clip, ArF immersion annular 0.5-0.8, SOCS K=24 (prebuilt), PEB sigma 20 nm, threshold",
        "ms": ms, "prints_per_s": 1000.0 / ms, "api": "lithobat_b200.process.print_image(kernels=...)"}
    n_ml, c_ml = 512, 64
    gm = lb.GridConfig(n_pixels=n_ml, pixel_size=2e-9)
    om = dataclasses.replace(uneven_optics(), mask_model="multilayer", chief_ray_deg=6.0, normalisation="clear")
    rng = np.random.default_rng(79)
    mm = torch.from_numpy(np.stack([patterns.manhattan_clip(rng, n_ml, 2e-9, n_rect=(20, 60), width_nm=(20.0, 80.0))
                                    for _ in range(c_ml)]).astype(np.float32)).to(dev)
    ms = timed(lambda: lb.compute_aerial_batch(mm, om, gm))
    out["multilayer_euv"] = {
        "workload": f"{c_ml} clips of {n_ml}^2 at 2 nm, EUV NA 0.33 dipole (204 source points), multilayer blank, "
                    "chief ray 6 deg",
        "ms": ms, "images_per_s": c_ml / (ms / 1000.0), "api": "lithobat_b200.compute_aerial_batch"}
    out["parity"] = ("reference fixtures and the FP64 oracle at 1e-5: tests/test_gpu_process.py, "
                     "tests/test_gpu_multilayer.py")
    return out


def bench_uneven(args, torch, dev, world, max_over_ranks, barrier) -> dict:
    """Images/s of the uneven batch: one CUDA-graph replay per batch, work-item
    sizes tuned per grid size on first use."""
    import lithobat_b200 as lb
    from lithobat_b200 import patterns
    from lithobat_b200.uneven import UnevenAbbe
    rank = int(os.environ.get("RANK", "0"))
    rng = np.random.default_rng(700 + rank)
    count = args.uneven_clips
    sizes = list(rng.choice([256, 512, 1024, 2048], size=count, p=[0.4, 0.3, 0.2, 0.1]))
    o = uneven_optics()
    masks = [torch.from_numpy(patterns.manhattan_clip(rng, int(n), 2e-9, n_rect=(20, 60),
                                                      width_nm=(20.0, 80.0)).astype(np.float32)).to(dev)
             for n in sizes]
    t0 = time.perf_counter()
    run = UnevenAbbe(sizes, o, 2e-9, tune=not args.no_tune, graph=True)
    setup_s = time.perf_counter() - t0
    run.load(masks)
    for _ in range(max(1, args.warmup)):
        run.run()
    torch.cuda.synchronize()
    barrier()
    steps = max(1, min(args.steps, 20))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        run.run()
    e1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / steps)
    # agreement with one-clip-at-a-time imaging on one clip of each size
    imgs = run(masks)
    worst = 0.0
    for n in sorted(set(sizes)):
        i = sizes.index(n)
        ref = lb.compute_aerial_batch(masks[i][None], o, lb.GridConfig(n_pixels=int(n), pixel_size=2e-9))[0][0, 0]
        worst = max(worst, float((imgs[i].double() - ref.double()).abs().max() / ref.double().abs().max()))
    ilt_line = None
    if "unevenilt" not in args.skip:
        from lithobat_b200 import ilt
        from lithobat_b200.uneven import UnevenIlt
        o_ilt = dataclasses.replace(o, normalisation="clear")
        th = [0.5 * torch.randn((int(n), int(n)), device=dev, generator=torch.Generator(device=dev).manual_seed(
            900 + i)) for i, n in enumerate(sizes)]
        t1 = time.perf_counter()
        uni = UnevenIlt([m for m in masks], th, o_ilt, 2e-9,
                        lambda k: ilt.IltParams(scale=1.0 / k.clear, level=0.3, steepness=15.0, step=0.2, beta=4.0),
                        max_kernels=24)
        torch.cuda.synchronize()
        build_s = time.perf_counter() - t1
        uni.run(2)        # records each group's step as a CUDA graph, outside the timed region
        torch.cuda.synchronize()
        c0 = float(sum(float(c) for c in uni.run(1)))
        n_steps = 20
        e0.record()
        uni.run(n_steps)  # groups' graph replays on parallel streams
        e1.record()
        torch.cuda.synchronize()
        ims = max_over_ranks(e0.elapsed_time(e1) / n_steps)
        c1 = float(sum(float(c) for c in uni.run(1)))
        ilt_line = {"metric": "uneven-batch ILT clip-steps/s", "value": world * count / (ims / 1000.0),
                    "unit": "clip-steps/s", "ms_per_step": ims, "steps": n_steps, "kernels": 24,
                    "socs_build_and_setup_s": build_s, "band_limited_groups": {
                        int(n): bool(b.fast) for n, _i, _k, b in uni.groups},
                    "total_cost_before_after": [c0, c1], "graph_replay": True,
                    "groups_on_parallel_streams": True}
        del uni
    return {"metric": "uneven-batch Abbe images/s", "value": world * count / (ms / 1000.0), "unit": "images/s",
            "ilt": ilt_line,
            "ms_per_batch": ms, "steps": steps, "workload": UNEVEN_WORKLOAD, "clips": count,
            "clips_per_size": {int(n): int(sum(1 for x in sizes if x == n)) for n in sorted(set(sizes))},
            "source_points": len(lb.source_points(o)), "graph_replay": run.graph is not None,
            "engine": run.engine, "queue_tasks": run.queue.n_tasks if run.queue is not None else 0,
            "tuned_items_per_block": {int(k): v["items_per_block"] for k, v in run.tuned.items()},
            "tuned": {int(k): {kk: vv for kk, vv in v.items() if kk != "ms"} for k, v in run.tuned.items()},
            "setup_and_tuning_s": setup_s, "max_rel_diff_vs_single_clip": worst}


def cpu_ilt_check(case: dict) -> tuple[float, float, float]:
    """FP64 numpy objective (forward + adjoint, K = 24) of one clip of the ILT
    batch at the GPU's state: (seconds, cost error, gradient error)."""
    from oracle import litho_oracle as O
    o = ilt_optics()

    class G:
        n_pixels, pixel_size = N, PX
    k = O.socs_build(o, G, tol=0.0, max_kernels=24)
    m = O.mask_of(case["theta"].astype(np.float64), case["beta"], 0.0)
    t0 = time.perf_counter()
    cost, grad, _, _ = O.objective(k, case["target"].astype(np.float64), m, 1.0 / k.clear, 0.3, 0.0, 1.0, 15.0)
    t = time.perf_counter() - t0
    e_cost = abs(case["cost"] - cost) / abs(cost)
    e_grad = float(np.abs(case["grad"] - grad).max() / np.abs(grad).max())
    return t, e_cost, e_grad


def cpu_config_check(case: dict) -> dict:
    """One image of a config through the FP64 reference algorithm on the host:
    its time (the config's CPU baseline) and the GPU image's error against it."""
    from oracle import litho_oracle as O

    class G:
        n_pixels, pixel_size = case["n"], case["px"]
    t0 = time.perf_counter()
    raw, pk, _ = O.compute_aerial_image(case["mask"], case["optics"], G, return_raw=True)
    t = time.perf_counter() - t0
    ref = raw / pk if case["peak_normalised"] else raw
    return {"cpu_baseline": {"value": 1.0 / t, "unit": "images/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": "one whole image of the timed batch, FP64 numpy/scipy (FFT workers=-1)"},
            "max_rel_err_vs_fp64": float(np.abs(case["gpu"] - ref).max() / np.abs(ref).max())}


C1_WORKLOAD = ("scalar Abbe 256^2 @4 nm, ArF dry NA 0.93, annular 0.5-0.8 (source_grid 31, 264 pts), "
               "L/S 200/100 nm binary mask, peak normalisation")
C2_WORKLOAD = ("scalar Abbe 512^2 @2 nm x64 Manhattan clips (complex64), NA 1.35/1.44 quadrupole 0.7-0.9 30 deg, "
               "per-clip defocus U(-60,60) nm and Z4-Z21 U(-0.02,0.02) waves, peak normalisation")


def bench_config(tag: str, args, torch, dev, world, max_over_ranks, barrier) -> dict:
    """Images/s of the first two workloads (c1: 1024 images of 256^2 per step;
    c2: the 64-clip 512^2 batch per step), two rotating input batches larger
    than L2, with stage times, the HBM roofline of the streaming stages and
    (C1) the latency of one single-image call."""
    import lithobat_b200 as lb
    from lithobat_b200 import aerial, patterns
    rank = int(os.environ.get("RANK", "0"))
    if tag == "c1":
        n, px, B = 256, 4e-9, 1024
        o = lb.OpticsConfig(wavelength=193e-9, NA=0.93, source_type="annular", sigma_inner=0.5, sigma_outer=0.8,
                            source_grid=31)
        one = patterns.lines_and_spaces(n, px, 200e-9, 100e-9).astype(np.float32)
        host = [np.broadcast_to(one, (B, n, n)) for _ in range(ROTATE)]
        optics = [o] * B
        workload = C1_WORKLOAD
    else:
        n, px, B = 512, 2e-9, 64
        src = lb.Source.quadrupole(0.9, 0.7, 30, 0).to_dict()
        host, optics = [], None
        for r in range(ROTATE):
            rng = np.random.default_rng(40 + 10 * rank + r)
            host.append(np.stack([patterns.manhattan_clip(rng, n, px) for _ in range(B)]).astype(np.complex64))
            if optics is None:
                optics = [lb.OpticsConfig(NA=1.35, n_immersion=1.44, source_spec=src,
                                          defocus=float(rng.uniform(-60e-9, 60e-9)),
                                          zernike_coeffs={j: float(rng.uniform(-0.02, 0.02)) for j in range(4, 22)})
                          for _ in range(B)]
        workload = C2_WORKLOAD
    views = [lb.config.optics_view(x) for x in optics]
    dmasks = [torch.from_numpy(np.ascontiguousarray(h)).to(dev) for h in host]
    pd = aerial.plan_abbe(views, n, px, [[(v.defocus, v.image_index)] for v in views], 1.0, False,
                          bool(dmasks[0].is_complex()))
    out = torch.empty((B, n, n), dtype=torch.float32, device=dev)
    peak = torch.empty((B,), dtype=torch.float32, device=dev)
    for i in range(max(3, args.warmup)):
        aerial.run_abbe(pd, dmasks[i % ROTATE], out, peak)
    torch.cuda.synchronize()
    barrier()
    steps = args.steps
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(steps):
        aerial.run_abbe(pd, dmasks[i % ROTATE], out, peak)
    e1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / steps)
    aerial.check_status(pd, dev)
    stages = aerial.profile_abbe(pd, dmasks[0], reps=max(3, min(steps, 10)))
    NN = n * n
    Bm = 2 * pd.plan.bm + 1
    esz = 8 if dmasks[0].is_complex() else 4
    stage_bytes = {"band_rows": B * (NN * esz + n * Bm * 8), "synthesis": B * NN * 4}
    dom = max(stage_bytes, key=stages.get)
    hbm = float(measured_peaks()["hbm_gbs"])
    achieved = stage_bytes[dom] / (stages[dom] / 1000.0) / 1e9
    res = {"workload": workload, "value": world * B / (ms / 1000.0), "unit": "images/s", "ms_per_step": ms,
           "images_per_step": B, "source_points": pd.jobs // B, "transforms_per_image": pd.transforms // B,
           "engine": aerial.engine_info(pd), "stages_ms": stages,
           "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                        "frac": achieved / hbm, "bytes_per_launch": stage_bytes[dom]},
           "l2": f"{ROTATE} rotating input batches of {B * NN * esz >> 20} MiB"}
    if tag == "c1":
        # one image per call: the latency a single-image caller sees
        pd1 = aerial.plan_abbe(views[:1], n, px, [[(views[0].defocus, views[0].image_index)]], 1.0, False, False)
        m1 = dmasks[0][:1].contiguous()
        o1 = torch.empty((1, n, n), dtype=torch.float32, device=dev)
        p1 = torch.empty((1,), dtype=torch.float32, device=dev)
        for _ in range(3):
            aerial.run_abbe(pd1, m1, o1, p1)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(20):
            aerial.run_abbe(pd1, m1, o1, p1)
        e1.record()
        torch.cuda.synchronize()
        res["single_image_ms"] = e0.elapsed_time(e1) / 20
    aerial.run_abbe(pd, dmasks[0], out, peak)
    res["_fp64_case"] = {"n": n, "px": px, "optics": optics[0], "mask": host[0][0].astype(np.complex128),
                         "gpu": out[0].double().cpu().numpy(), "peak_normalised": True}
    del dmasks, out
    return res


def measured_peaks() -> dict:
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        return json.loads(f.read_text())
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0, "_fallback": True}


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "20"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.p = None
        # start the timed region only once the sampler is producing rows
        t0 = time.perf_counter()
        while self.p is not None and time.perf_counter() - t0 < 5.0:
            self.f.flush()
            if Path(self.f.name).stat().st_size > 0:
                break
            time.sleep(0.01)
        self.skip = Path(self.f.name).read_text().count("\n") if self.p is not None else 0
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self) -> dict:
        self.f.flush()
        rows = []
        # rows written before the timed region started are not counted
        for line in Path(self.f.name).read_text().splitlines()[getattr(self, "skip", 0):]:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# CPU (reference algorithm) timing
# ---------------------------------------------------------------------------
def cpu_info() -> dict:
    """The host CPU the CPU numbers ran on: model name and logical cores."""
    model = "unknown"
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"model": model, "logical_cores": os.cpu_count()}


class CpuAbbeSample:
    """The FP64 numpy Abbe sum (the reference algorithm, restated in the
    oracle) of one workload image, whole or over its first k source points."""

    def __init__(self, mask=None):
        from oracle import litho_oracle as O
        self.O = O
        self.o = optics_c3()
        self.S = len(O.source_points(self.o))
        self.mask = (masks_c3(1, 1)[0] if mask is None else np.asarray(mask)).astype(np.complex128)

        class G:
            n_pixels, pixel_size = N, PX
        self.G = G
        self.planes = [(self.o.defocus, self.o.image_index)]
        self(2)  # warm the FFT plans

    def __call__(self, k: int | None = None) -> float:
        t0 = time.perf_counter()
        self.last = self.O.abbe_sum(self.mask, self.o, self.G, self.planes,
                                    source_subset=None if k is None else range(k))
        return time.perf_counter() - t0


def run_reference(args) -> None:
    """The reference arm: the reference's CPU algorithm on the host cores.

    Each step is a bounded sample of the workload, the same first k source
    points of one workload image (3k of its 1200 coherent transforms, FP64,
    scipy FFTs on all cores), with k sized so the whole warm-up + timed run
    takes about 150 s. ``value`` is the images/s that work amounts to
    (k / 400 of an image per step) and ``ms_per_step`` its measured time."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    smp = CpuAbbeSample()
    S = smp.S
    t1 = smp(2) / 2.0
    k = int(max(1, min(S, 150.0 / max(1, args.warmup + args.steps) / max(t1, 1e-3))))
    for _ in range(args.warmup):
        smp(k)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        smp(k)
    total = time.perf_counter() - t0
    v = (k / S) * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "images/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128/f64",
        "data": "synthetic (seeded att-PSM contact-hole clips)",
        "config": {"workload": WORKLOAD, "images_per_step": k / S, "source_points_per_step": k,
                   "source_points_per_image": S},
        "cpu": cpu_info(),
        "cpu_baseline": {"value": v, "unit": "images/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"each step: the first {k} of one image's {S} source points ({3 * k} of its "
                                   f"{3 * S} coherent transforms), FP64 numpy/scipy (FFT workers=-1)"},
        "e2e": {"value": v, "unit": "images/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    import lithobat_b200 as lb
    from lithobat_b200 import aerial

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier(device_ids=[local])

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    o = optics_c3()
    g = lb.GridConfig(n_pixels=N, pixel_size=PX)
    B = args.images
    dmasks = [masks_c3_device(torch, 1000 * rank + r, B, dev) for r in range(ROTATE)]
    view = lb.config.optics_view(o)
    pd = aerial.plan_abbe([view] * B, N, PX, [[(view.defocus, view.image_index)]] * B, 1.0, False, True)
    out = torch.empty((B, N, N), dtype=torch.float32, device=dev)
    peak = torch.empty((B,), dtype=torch.float32, device=dev)
    # twiddles, band rows, band columns, coarse, reduce, then the synthesis: on the tensor cores
    # (enough 128 x 256 output tiles for about 8 per SM) P planes, Q planes, peak pass, peak,
    # writing pass, peak; otherwise column stage, peak pass, peak, writing pass, peak
    tensor_synth = aerial.engine_info(pd)["synthesis"] == "tensor_cores"
    launches_per_step = 5 + (6 if tensor_synth else 5)

    def step(i):
        aerial.run_abbe(pd, dmasks[i % ROTATE], out, peak)

    # ---- device-resident throughput (fused engine) ----
    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        e0.record()
        for i in range(args.steps):
            step(i)
        e1.record()
        torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    aerial.check_status(pd, dev)      # no bounded wait gave up in the timed steps
    clocks = clk.summary()
    value = world * B * args.steps / (ms / 1000.0)
    line = {
        "metric": METRIC, "value": value, "unit": "images/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64/f32", "data": "synthetic (seeded att-PSM contact-hole clips)",
        "clocks": clocks, "gpu_launches": launches_per_step * args.steps,
    }
    NN = N * N
    transforms = pd.transforms // B
    line["config"] = {"workload": WORKLOAD, "images_per_step": B, "grid": N, "pixel_nm": 1.0,
                      "source_points": pd.jobs // B, "transforms_per_image": transforms,
                      "coarse_grid": int(pd.plan.L), "parallelism": f"replicas x{world}",
                      "l2": f"{ROTATE} rotating input batches of {B * NN * 8 >> 20} MiB"}
    pd_small = aerial.plan_abbe([view] * PLAIN_IMAGES, N, PX, [[(view.defocus, view.image_index)]] * PLAIN_IMAGES,
                                1.0, False, True)

    # ---- per-stage device times (CUDA events between the stages) ----
    if "profile" not in args.skip:
        stages = aerial.profile_abbe(pd, dmasks[0], reps=max(3, args.steps))
        step_ms = sum(stages.values())
        table_ms = aerial.profile_abbe(pd_small, dmasks[0][:PLAIN_IMAGES].contiguous(), reps=3,
                                       rebuild_table=True)["pupil_table"]
        peaks = measured_peaks()
        hbm = float(peaks["hbm_gbs"])
        Bm = 2 * pd.plan.bm + 1
        stage_bytes = {   # algorithmic bytes of each stage per launch (the whole batch)
            "pupil_table": pd.plan.n_tab * 3 * (2 * pd.plan.h + 1) ** 2 * 8,
            "band_rows": B * (NN * 8 + N * Bm * 8),
            "band_cols": B * (N * Bm * 8 + Bm * Bm * 8),
            "coarse": pd.plan.n_tab * 3 * (2 * pd.plan.h + 1) ** 2 * 8 + pd.plan.n_items * 32 * 32 * 4,
            "coarse_reduce": pd.plan.n_items * 32 * 32 * 4,
            "peak_pass": 0,                 # compute only: no per-pixel HBM traffic
            "synthesis": B * NN * 4,
        }
        # the roofline object is for the slowest HBM-bound stage (the stages
        # that stream pixels); the on-chip FFT stages are FP32-issue bound and
        # are reported against the FP32 peak instead
        dom = max(("band_rows", "synthesis"), key=stages.get)
        achieved = stage_bytes[dom] / (stages[dom] / 1000.0) / 1e9
        Lc, hc = int(pd.plan.L), int(pd.plan.h)
        fft_flops = 5 * Lc * math.log2(Lc)
        coarse_flops = pd.transforms * ((2 * hc + 1) * fft_flops + Lc * fft_flops + 3 * Lc * Lc)
        fp32_peak = 148 * 128 * 2 * float(peaks.get("sm_max_mhz", 1965.0)) * 1e6 / 1e12
        formula_bytes = NN * (16 * transforms + 24)  # dense two-pass FFT equivalent, per image
        line["config"]["pupil_table"] = f"built once per optics ({table_ms:.3f} ms), reused across steps"
        # DRAM bytes (read + write) of one launch, from an ncu capture of the
        # 96-image case (805.33 MB read + 9.52 MB written) scaled by images per
        # launch: traffic grows in proportion to the images processed
        traffic = {"band_rows": (805.33e6 + 9.52e6) / 96 * B}.get(dom)
        line["roofline"] = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                            "frac": achieved / hbm, "traffic": traffic,
                            "peak_source": "measured" if not peaks.get("_fallback") else "fallback"}
        line["stages_ms"] = stages
        line["fp32_stages"] = {
            "coarse": {"tflops": coarse_flops / (stages["coarse"] / 1000.0) / 1e12, "peak_tflops": fp32_peak,
                       "flops_per_transform": coarse_flops / pd.transforms,
                       "frac": coarse_flops / (stages["coarse"] / 1000.0) / 1e12 / fp32_peak}}
        line["dense_fft_equivalent"] = {"bytes_per_image": formula_bytes,
                                        "GBps": formula_bytes * B / (step_ms / 1000.0) / 1e9}

    # ---- fused vs plain on the same clips, and their agreement ----
    if "plain" not in args.skip:
        sub = dmasks[0][:PLAIN_IMAGES].contiguous()
        fused_img, _ = aerial.run_abbe(pd_small, sub)
        fused_img = fused_img.clone()
        plain_img, _ = aerial.run_abbe(pd_small, sub, engine="plain")  # warm
        torch.cuda.synchronize()
        p_steps = 2
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record()
        for i in range(p_steps):
            plain_img, _ = aerial.run_abbe(pd_small, sub, engine="plain")
        e3.record()
        torch.cuda.synchronize()
        plain_ms = max_over_ranks(e2.elapsed_time(e3) / p_steps)
        plain_value = world * PLAIN_IMAGES / (plain_ms / 1000.0)
        agree = float(((fused_img.double() - plain_img.double()).abs().amax(dim=(1, 2))
                       / plain_img.double().abs().amax(dim=(1, 2))).max())
        del plain_img
        # a perfect dense-FFT plain loop moves N^2 (16 T + 24) bytes per image
        dense_ceiling = measured_peaks()["hbm_gbs"] * 1e9 / (NN * (16 * transforms + 24))
        line["plain"] = {"value": plain_value, "unit": "images/s", "fused_over_plain": value / plain_value,
                         "images_per_call": PLAIN_IMAGES, "max_rel_diff_fused_vs_plain": agree,
                         "dense_fft_roofline_images_per_s": dense_ceiling,
                         "fused_over_dense_roofline": value / dense_ceiling}

    # ---- end to end from pinned host memory: masks in, images out ----
    if "e2e" not in args.skip:
        from lithobat_b200.pipeline import AbbePipeline
        pinned = [dmasks[r][:E2E_IMAGES].cpu().pin_memory() for r in range(ROTATE)]
        res = [torch.empty((E2E_IMAGES, N, N), dtype=torch.float32).pin_memory() for _ in range(2)]
        pipe = AbbePipeline(o, g, E2E_IMAGES, mask_complex=True)
        pipe.run([pinned[i % ROTATE] for i in range(max(1, args.warmup))],
                 [res[i % 2] for i in range(max(1, args.warmup))])
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        pipe.run([pinned[i % ROTATE] for i in range(args.steps)], [res[i % 2] for i in range(args.steps)])
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1000.0)
        # the same images through the one-call API, serially (upload, image, download)
        t1 = time.perf_counter()
        ser = min(args.steps, 10)
        for i in range(ser):
            img, _pk, _cl = lb.compute_aerial_batch(pinned[i % ROTATE], o, g)
            res[0].copy_(img[:, 0])
        torch.cuda.synchronize()
        ser_ms = max_over_ranks((time.perf_counter() - t1) * 1000.0)
        line["e2e"] = {"value": world * E2E_IMAGES * args.steps / (e2e_ms / 1000.0), "unit": "images/s",
                       "h2d_bytes_per_step": E2E_IMAGES * NN * 8, "d2h_bytes_per_step": E2E_IMAGES * NN * 4,
                       "images_per_step": E2E_IMAGES, "api": "lithobat_b200.pipeline.AbbePipeline (copies of "
                       "consecutive batches overlapped with compute)",
                       "serial_one_call_value": world * E2E_IMAGES * ser / (ser_ms / 1000.0)}
    # ---- the same workload with the masks as level maps (1 byte per pixel) ----
    lv_img0 = None
    if "levels" not in args.skip:
        absorber = torch.tensor(complex(np.sqrt(0.06) * np.exp(1j * np.pi)), dtype=torch.complex64, device=dev)
        lv = torch.stack([torch.ones((), dtype=torch.complex64, device=dev), absorber]).repeat(B, 1)
        imaps = [(dmasks[r] != 1).to(torch.uint8).contiguous() for r in range(ROTATE)]
        aerial.run_abbe_levels(pd, imaps[0], lv, out, peak)
        lv_img = out.clone()
        aerial.run_abbe(pd, dmasks[0], out, peak)
        lv_diff = float(((lv_img.double() - out.double()).abs().amax(dim=(1, 2))
                         / out.double().abs().amax(dim=(1, 2))).max())
        lv_img0 = lv_img[0].double().cpu().numpy()   # its FP64 error is taken with the CPU sample below
        del lv_img
        for i in range(args.warmup):
            aerial.run_abbe_levels(pd, imaps[i % ROTATE], lv, out, peak)
        torch.cuda.synchronize()
        barrier()
        e0.record()
        for i in range(args.steps):
            aerial.run_abbe_levels(pd, imaps[i % ROTATE], lv, out, peak)
        e1.record()
        torch.cuda.synchronize()
        lms = max_over_ranks(e0.elapsed_time(e1))
        aerial.check_status(pd, dev)
        lvl = {"value": world * B * args.steps / (lms / 1000.0), "unit": "images/s",
               "ms_per_step": lms / args.steps, "max_rel_diff_vs_complex_masks": lv_diff,
               "input": "uint8 level map per clip + its two complex levels (litho_abbe_levels)",
               "l2": f"{ROTATE} rotating input batches of {B * NN >> 20} MiB"}
        if "e2e" not in args.skip:
            from lithobat_b200.pipeline import AbbePipeline
            pin_i = [imaps[r][:E2E_IMAGES].cpu().pin_memory() for r in range(ROTATE)]
            lv_h = lv[:E2E_IMAGES].cpu()
            res = [torch.empty((E2E_IMAGES, N, N), dtype=torch.float32).pin_memory() for _ in range(2)]
            lpipe = AbbePipeline(o, g, E2E_IMAGES, mask_complex=True, level_masks=True)
            lpipe.run([pin_i[i % ROTATE] for i in range(max(1, args.warmup))],
                      [res[i % 2] for i in range(max(1, args.warmup))], levels=lv_h)
            torch.cuda.synchronize()
            barrier()
            t0 = time.perf_counter()
            lpipe.run([pin_i[i % ROTATE] for i in range(args.steps)], [res[i % 2] for i in range(args.steps)],
                      levels=lv_h)
            torch.cuda.synchronize()
            le2e = max_over_ranks((time.perf_counter() - t0) * 1000.0)
            lvl["e2e"] = {"value": world * E2E_IMAGES * args.steps / (le2e / 1000.0), "unit": "images/s",
                          "h2d_bytes_per_step": E2E_IMAGES * NN + E2E_IMAGES * 2 * 8,
                          "d2h_bytes_per_step": E2E_IMAGES * NN * 4, "images_per_step": E2E_IMAGES,
                          "api": "lithobat_b200.pipeline.AbbePipeline(level_masks=True)"}
            del lpipe, pin_i, res
        line["level_maps"] = lvl
        del imaps
    for key in ("c1", "c2"):
        if key not in args.skip:
            line[key] = bench_config(key, args, torch, dev, world, max_over_ranks, barrier)
    if "ilt" not in args.skip:
        line["ilt"] = bench_ilt(args, torch, dev, world, max_over_ranks, barrier)
    if "uneven" not in args.skip:
        line["uneven"] = bench_uneven(args, torch, dev, world, max_over_ranks, barrier)
    if "next" not in args.skip and rank == 0:
        line["next_rows"] = bench_next(args, torch, dev)
    if rank == 0 and world == 1 and not args.no_cpu:
        # one whole image of the timed batch through the FP64 reference
        # algorithm: the CPU baseline, and the FP64 reference of that image
        aerial.run_abbe(pd, dmasks[0], out, peak)
        gpu0 = out[0].double().cpu().numpy()
        smp = CpuAbbeSample(dmasks[0][0].cpu().numpy())
        t = smp()
        raw, rpk, _ = smp.last
        line["cpu_baseline"] = {"value": 1.0 / t, "unit": "images/s", "cores": os.cpu_count(), "kind": "port",
                                "sample": f"one whole image of the timed batch ({smp.S} source points, "
                                          f"{3 * smp.S} coherent transforms), FP64 numpy/scipy (FFT workers=-1)"}
        line["cpu"] = cpu_info()
        line["max_rel_err_vs_fp64"] = float(np.abs(gpu0 - raw[0] / rpk[0]).max())
        if line.get("level_maps") is not None and lv_img0 is not None:
            line["level_maps"]["max_rel_err_vs_fp64"] = float(np.abs(lv_img0 - raw[0] / rpk[0]).max())
        if line.get("ilt") and line["ilt"].get("_fp64_case"):
            case = line["ilt"].pop("_fp64_case")
            ti, e_cost, e_grad = cpu_ilt_check(case)
            line["ilt"]["cpu_baseline"] = {"value": 1.0 / ti, "unit": "clip-steps/s", "cores": os.cpu_count(),
                                           "kind": "port",
                                           "sample": "one 1024^2 clip of the batch: FP64 objective + adjoint, K=24"}
            line["ilt"]["max_rel_err_vs_fp64"] = {"cost": e_cost, "gradient": e_grad}
        for key in ("c1", "c2"):
            if line.get(key) and line[key].get("_fp64_case"):
                line[key].update(cpu_config_check(line[key].pop("_fp64_case")))
    for key in ("ilt", "c1", "c2"):
        if line.get(key):
            line[key].pop("_fp64_case", None)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--images", type=int, default=IMAGES_PER_STEP,
                    help="images per step (a small value makes a profiling case)")
    ap.add_argument("--skip", default="", help="comma list of phases to skip: plain,e2e,levels,profile,cpu,c1,c2,ilt,iltplain,uneven,"
                                        "unevenilt,next")
    ap.add_argument("--ilt-clips", type=int, default=ILT_CLIPS, help="clips per ILT step")
    ap.add_argument("--uneven-clips", type=int, default=256, help="clips in the uneven-size batch")
    ap.add_argument("--no-tune", action="store_true",
                    help="uneven batch with the library's default queue sizes (no search; for profiling)")
    args = ap.parse_args()
    args.skip = set(x for x in args.skip.split(",") if x)
    if "cpu" in args.skip:
        args.no_cpu = True
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
