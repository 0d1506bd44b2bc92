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
resident in HBM; ``e2e`` is the same metric through the public API
(``compute_aerial_batch``) from pinned host buffers, copies included.
``--impl reference`` times the reference's algorithm on the host CPU (the
FP64 numpy restatement in ``oracle/``, the same numpy/scipy calls), on a
bounded sample of source points, and prints the same line for it.
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
        ev[0].record()
        gm = st.synth(b.hbox, st.h, False)
        ev[1].record()
        nat_.check("update", st.L.litho_ilt_update(gm.data_ptr(), gm.numel(), b.beta, b.beta, 0.4, 0.9, 0.999, 1e-8,
                                                   5, th.data_ptr(), m1.data_ptr(), m2.data_ptr(), mk.data_ptr(),
                                                   st.stream()))
        ev[2].record()
        mbox = st.mask_box(mk)
        ev[3].record()
        raw = st.image(mbox)
        ev[4].record()
        dfield = torch.empty_like(raw)
        nat_.check("obj", st.L.litho_ilt_objective(raw.data_ptr(), b.target.data_ptr(), nclip, N,
                                                   float(params.scale), 0.3, 1.0, 50.0, dfield.data_ptr(), None,
                                                   cpart.data_ptr(), ppart.data_ptr(), 64, st.stream()))
        ev[5].record()
        gbox = st.band(dfield, 2 * st.h, float(params.scale) / (N * N))
        ev[6].record()
        st.adjoint_box(gbox, mbox)
        ev[7].record()
        torch.cuda.synchronize()
        names = ["gradient_synthesis", "theta_grad+adam+mask", "mask_band_spectrum",
                 "coarse_image_and_synthesis", "objective", "sensitivity_band_spectrum",
                 "adjoint: dJ/dI on the 64 grid, per-kernel adjoint, gradient band box"]
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
    # end to end from pinned host memory: upload theta/targets, K steps reading
    # the cost back every step, download theta
    tp = torch.from_numpy(targets).pin_memory()
    hp = torch.from_numpy(theta).pin_memory()
    out = torch.empty_like(hp).pin_memory()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0.record()
    eb = ilt.IltBatch(k, tp.to(dev, non_blocking=True), hp.to(dev, non_blocking=True), params)
    for _ in range(args.steps):
        eb.step(want_signed=False)
        float(eb.cost.sum())
    out.copy_(eb.theta)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1000.0))
    NN = N * N
    return {
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
    run = UnevenAbbe(sizes, o, 2e-9, tune=True, graph=True)
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
        for _ in range(2):
            uni.step()
        torch.cuda.synchronize()
        c0 = float(sum(float(c) for c in uni.step()))
        n_steps = 20
        e0.record()
        for _ in range(n_steps):
            uni.step()
        e1.record()
        torch.cuda.synchronize()
        ims = max_over_ranks(e0.elapsed_time(e1) / n_steps)
        c1 = float(sum(float(c) for c in uni.step()))
        ilt_line = {"metric": "uneven-batch ILT clip-steps/s", "value": world * count / (ims / 1000.0),
                    "unit": "clip-steps/s", "ms_per_step": ims, "steps": n_steps, "kernels": 24,
                    "socs_build_and_setup_s": build_s, "band_limited_groups": {
                        int(n): bool(b.fast) for n, _i, _k, b in uni.groups},
                    "total_cost_before_after": [c0, c1]}
        del uni
    return {"metric": "uneven-batch Abbe images/s", "value": world * count / (ms / 1000.0), "unit": "images/s",
            "ilt": ilt_line,
            "ms_per_batch": ms, "steps": steps, "workload": UNEVEN_WORKLOAD, "clips": count,
            "clips_per_size": {int(n): int(sum(1 for x in sizes if x == n)) for n in sorted(set(sizes))},
            "source_points": len(lb.source_points(o)), "graph_replay": run.graph is not None,
            "tuned_items_per_block": {int(k): v["items_per_block"] for k, v in run.tuned.items()},
            "setup_and_tuning_s": setup_s, "max_rel_diff_vs_single_clip": worst}


def cpu_ilt_seconds() -> tuple[float, int]:
    """FP64 numpy objective (forward + adjoint) of one clip of the ILT workload, K = 24."""
    from oracle import litho_oracle as O
    o = ilt_optics()

    class G:
        n_pixels, pixel_size = N, PX
    k = O.socs_build(o, G, tol=0.0, max_kernels=24)
    targets, theta = ilt_inputs(500, 1)
    m = O.mask_of(theta[0].astype(np.float64), 4.0, 0.0)
    t0 = time.perf_counter()
    O.objective(k, targets[0].astype(np.float64), m, 1.0 / k.clear, 0.3, 0.0, 1.0, 15.0)
    return time.perf_counter() - t0, 1


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
class CpuAbbeSample:
    """The FP64 numpy Abbe sum (the reference algorithm, restated in the
    oracle) over the first k source points of one workload image."""

    def __init__(self):
        from oracle import litho_oracle as O
        self.O = O
        self.o = optics_c3()
        self.S = len(O.source_points(self.o))
        self.mask = masks_c3(1, 1)[0].astype(np.complex128)

        class G:
            n_pixels, pixel_size = N, PX
        self.G = G
        self.planes = [(self.o.defocus, self.o.image_index)]
        self(2)  # warm the FFT plans

    def __call__(self, k: int) -> float:
        t0 = time.perf_counter()
        self.O.abbe_sum(self.mask, self.o, self.G, self.planes, source_subset=range(k))
        return time.perf_counter() - t0


def cpu_sample_seconds(n_src: int = 12, repeats: int = 2) -> tuple[float, int, int]:
    """Median seconds of the CPU Abbe sum over the first n_src source points
    of one workload image; returns (t, n_src, S_total)."""
    smp = CpuAbbeSample()
    return statistics.median(smp(n_src) for _ in range(repeats)), n_src, smp.S


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    smp = CpuAbbeSample()
    # source points per step: the whole run stays near 150 s of CPU work
    t1 = smp(2) / 2.0
    k = int(max(1, min(12, 150.0 / max(1, args.warmup + args.steps) / max(t1, 1e-3))))
    S = smp.S
    vals = []
    for i in range(args.warmup + args.steps):
        t = smp(k)
        if i >= args.warmup:
            vals.append(1.0 / (t * S / k))
    v = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "images/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / v, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128/f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "images_per_step": 1},
        "cpu_baseline": {"value": v, "unit": "images/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"{k} of {S} source points of one image per step, scaled by {S}/{k}"},
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
    # (enough 128 x 256 output tiles for about 16 per SM) P planes, Q planes, peak pass, peak,
    # writing pass, peak; otherwise column stage, peak pass, peak, writing pass, peak
    g0 = 2 * int(pd.plan.h)
    tensor_synth = g0 <= 31 and B * (N // 256) * (N // 128) >= 16 * 148
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
        line["plain"] = {"value": plain_value, "unit": "images/s", "fused_over_plain": value / plain_value,
                         "images_per_call": PLAIN_IMAGES, "max_rel_diff_fused_vs_plain": agree}

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
    if "ilt" not in args.skip:
        line["ilt"] = bench_ilt(args, torch, dev, world, max_over_ranks, barrier)
    if "uneven" not in args.skip:
        line["uneven"] = bench_uneven(args, torch, dev, world, max_over_ranks, barrier)
    if rank == 0 and world == 1 and not args.no_cpu:
        t, k, S = cpu_sample_seconds()
        cv = 1.0 / (t * S / k)
        line["cpu_baseline"] = {"value": cv, "unit": "images/s", "cores": os.cpu_count(), "kind": "port",
                                "sample": f"{k} of {S} source points of one image, scaled by {S}/{k}"}
        if "ilt" in line:
            ti, _ = cpu_ilt_seconds()
            line["ilt"]["cpu_baseline"] = {"value": 1.0 / ti, "unit": "clip-steps/s", "cores": os.cpu_count(),
                                           "kind": "port", "sample": "one 1024^2 clip objective + adjoint (K=24)"}
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
    ap.add_argument("--skip", default="", help="comma list of phases to skip: plain,e2e,profile,cpu,ilt,iltplain,uneven,unevenilt")
    ap.add_argument("--ilt-clips", type=int, default=ILT_CLIPS, help="clips per ILT step")
    ap.add_argument("--uneven-clips", type=int, default=256, help="clips in the uneven-size batch")
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
