"""Uneven batches (clips of mixed sizes in one CUDA-graph replay) against
one-clip-at-a-time imaging; same 1e-5 bar."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.fixture(scope="module")
def lb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lithobat_b200
    return lithobat_b200


def _euv(lb):
    from lithobat_b200.source import Source
    return lb.OpticsConfig(wavelength=13.5e-9, NA=0.33, source_grid=21,
                           source_spec=Source.dipole(0.9, 0.6, opening_deg=60).to_dict())


def _clips(seed, sizes):
    from lithobat_b200.patterns import manhattan_clip
    rng = np.random.default_rng(seed)
    return [manhattan_clip(rng, n, 2e-9, n_rect=(6, 16), width_nm=(20, 80)).astype(np.float32) for n in sizes]


def test_uneven_batch_matches_one_clip_at_a_time(lb):
    """128^2 (32-point coarse grid), 256^2 (64), 512^2 (wide, 128) in one
    replay; two batches in a row through the same graph."""
    import torch
    from lithobat_b200.uneven import UnevenAbbe
    o = _euv(lb)
    sizes = [256, 128, 512, 256, 128]
    run = UnevenAbbe(sizes, o, 2e-9, tune=True, graph=True)
    assert run.graph is not None and set(run.tuned) == {128, 256, 512}
    for seed in (1, 2):
        clips = _clips(seed, sizes)
        imgs = run([torch.from_numpy(c).cuda() for c in clips])
        torch.cuda.synchronize()
        for c, im in zip(clips, imgs):
            g = lb.GridConfig(n_pixels=c.shape[0], pixel_size=2e-9)
            ref = lb.compute_aerial_image(c.astype(np.float64), o, g)
            got = im.double().cpu().numpy()
            assert float(np.abs(got - ref).max() / np.abs(ref).max()) <= TOL


def test_uneven_function_numpy_in_numpy_out(lb):
    from lithobat_b200.uneven import compute_aerial_uneven
    o = _euv(lb)
    clips = _clips(3, [128, 256])
    out = compute_aerial_uneven(clips, o, 2e-9, return_raw=True)
    for c, im in zip(clips, out):
        assert isinstance(im, np.ndarray) and im.dtype == np.float64 and im.shape == c.shape
        g = lb.GridConfig(n_pixels=c.shape[0], pixel_size=2e-9)
        ref = lb.compute_aerial_image(c.astype(np.float64), o, g, return_raw=True)[0]
        assert float(np.abs(im - ref).max() / np.abs(ref).max()) <= TOL


def test_uneven_ilt_groups_and_steps(lb):
    """Mixed sizes: 128^2 (kernel band on chip) and 256^2 (wide band) at 2 nm
    EUV; each group's step equals its own IltBatch step, costs fall."""
    import torch
    from lithobat_b200 import ilt
    from lithobat_b200.uneven import UnevenIlt
    o = lb.OpticsConfig(wavelength=13.5e-9, NA=0.33, source_grid=15, normalisation="clear",
                        source_spec=__import__("lithobat_b200.source", fromlist=["Source"]).Source.dipole(
                            0.9, 0.6, opening_deg=60).to_dict())
    sizes = [256, 128, 128]
    tg = _clips(7, sizes)
    rng = np.random.default_rng(8)
    th = [0.5 * rng.standard_normal((n, n)).astype(np.float32) for n in sizes]

    def params(k):
        return ilt.IltParams(scale=1.0 / k.clear, level=0.3, steepness=15.0, step=0.1, beta=4.0)
    u = UnevenIlt(tg, th, o, 2e-9, params, max_kernels=12)
    assert [g[0] for g in u.groups] == [128, 256]
    assert u.groups[0][2].halfwidth <= 15 < u.groups[1][2].halfwidth
    c0 = [float(c) for c in u.step()]
    for _ in range(4):
        c = [float(x) for x in u.step()]
    assert all(b < a for a, b in zip(c0, c))
    # the 256^2 group against its own batch
    k = u.groups[1][2]
    b = ilt.IltBatch(k, torch.from_numpy(tg[0][None]).cuda(), torch.from_numpy(th[0][None]).cuda(), params(k))
    for _ in range(5):
        b.step(want_signed=False)
    assert float((b.theta[0] - u.theta()[0]).abs().max()) < 1e-5


def test_work_queue_matches_the_per_group_launches(lb):
    """The persistent work queue (one launch for the coherent passes of the
    512^2, 1024^2 and 2048^2 groups; 256^2 on the on-chip grid) against the
    per-group launch sequences and against one-clip-at-a-time imaging."""
    import torch
    from lithobat_b200.uneven import UnevenAbbe
    o = _euv(lb)
    sizes = [512, 256, 2048, 1024, 512, 1024]
    clips = [torch.from_numpy(c).cuda() for c in _clips(11, sizes)]
    q = UnevenAbbe(sizes, o, 2e-9, tune=False, graph=True, engine="queue")
    assert q.queue is not None and q.queue.n_tasks > 0
    got = [im.clone() for im in q(clips)]
    q.check_status()
    g = UnevenAbbe(sizes, o, 2e-9, tune=False, graph=False, engine="groups")
    ref = g(clips)
    torch.cuda.synchronize()
    worst = max(float((a.double() - b.double()).abs().max() / b.double().abs().max()) for a, b in zip(got, ref))
    print(f"PARITY uneven_queue_vs_groups {worst:.3e}")
    assert worst <= 2e-6
    for i in (0, 2):
        gr = lb.GridConfig(n_pixels=sizes[i], pixel_size=2e-9)
        r = lb.compute_aerial_image(clips[i].cpu().numpy().astype(np.float64), o, gr)
        assert float(np.abs(got[i].double().cpu().numpy() - r).max() / np.abs(r).max()) <= TOL
    # a second batch through the same graph
    clips2 = [torch.from_numpy(c).cuda() for c in _clips(12, sizes)]
    got2 = q(clips2)
    ref2 = g(clips2)
    torch.cuda.synchronize()
    assert max(float((a.double() - b.double()).abs().max() / b.double().abs().max())
               for a, b in zip(got2, ref2)) <= 2e-6


def test_work_queue_wait_that_runs_out_is_reported(lb):
    """A task list whose pass-B task waits for one signal more than its chunk
    gives: with a short wait limit the wait gives up, the queue's status word
    reads LITHO_E_TIMEOUT and the launch ends; the next run is clean and
    matches the first. Nothing faults or hangs (every wait is bounded)."""
    import ctypes as C
    import torch
    from lithobat_b200 import _native as nat
    from lithobat_b200.uneven import UnevenAbbe
    L = nat.lib()
    o = _euv(lb)
    sizes = [512, 512]
    run = UnevenAbbe(sizes, o, 2e-9, tune=False, graph=False)
    clips = [torch.from_numpy(c).cuda() for c in _clips(13, sizes)]
    first = [im.clone() for im in run(clips)]
    run.check_status()
    qu = run.queue
    bad = qu.tasks_host.copy()
    kb = int(np.flatnonzero(bad["kind"] == 1)[0])
    bad["wait_value"][kb] += 1
    bad_dev = torch.from_numpy(bad.view(np.uint8).copy()).cuda()
    s = nat.stream_ptr(torch)
    nat.check("litho_set_wait_limit", L.litho_set_wait_limit(200000))
    try:
        nat.check("litho_uneven_run", L.litho_uneven_run(qu.arr, qu.n_groups, bad_dev.data_ptr(), qu.n_tasks,
                                                         qu.n_counters, qu.ws.data_ptr(), qu.ws.numel(), s))
        st = L.litho_uneven_status(qu.ws.data_ptr(), s)
    finally:
        nat.check("litho_set_wait_limit", L.litho_set_wait_limit(0))
    assert st == 1000001   # LITHO_E_TIMEOUT
    with pytest.raises(nat.LithoError):
        run.check_status()
    again = run(clips)
    run.check_status()
    assert L.litho_uneven_status(qu.ws.data_ptr(), s) == 0
    for a, b in zip(first, again):
        assert torch.equal(a, b)


def test_tuned_sizes_persist_as_json(lb, tmp_path):
    """The tuner searches each group once and writes its choice; a second
    runner of the same batch reads it back instead of searching."""
    import json
    from lithobat_b200 import uneven
    o = _euv(lb)
    path = tmp_path / "tune.json"
    sizes = [512, 512, 256]
    uneven._TUNED.clear()
    a = uneven.UnevenAbbe(sizes, o, 2e-9, tune=True, graph=False, tune_cache=path)
    assert a.tuned[512]["source"] == "search" and a.tuned[512]["ms"]["candidates"] >= 5
    data = json.loads(path.read_text())
    assert any(k.endswith("|queue") and "n=512" in k for k in data)
    assert any(k.endswith("|launches") and "n=256" in k for k in data)
    uneven._TUNED.clear()
    b = uneven.UnevenAbbe(sizes, o, 2e-9, tune=True, graph=False, tune_cache=path)
    assert b.tuned[512]["source"] == "cache" and b.tuned[256]["source"] == "cache"
    assert b.groups[1].tune == a.groups[1].tune


def test_uneven_ilt_run_replays_groups_on_parallel_streams(lb):
    """UnevenIlt.run: each group's step recorded as a CUDA graph and the
    groups' replays on parallel streams give the iterates of eager steps."""
    import torch
    from lithobat_b200 import ilt
    from lithobat_b200.source import Source
    from lithobat_b200.uneven import UnevenIlt
    o = lb.OpticsConfig(wavelength=13.5e-9, NA=0.33, source_grid=15, normalisation="clear",
                        source_spec=Source.dipole(0.9, 0.6, opening_deg=60).to_dict())
    sizes = [256, 128, 256, 128]
    tg = _clips(17, sizes)
    rng = np.random.default_rng(18)
    th = [0.5 * rng.standard_normal((n, n)).astype(np.float32) for n in sizes]

    def params(k):
        return ilt.IltParams(scale=1.0 / k.clear, level=0.3, steepness=15.0, step=0.1, beta=4.0, growth=1.02)
    a = UnevenIlt(tg, th, o, 2e-9, params, max_kernels=12)
    b = UnevenIlt(tg, th, o, 2e-9, params, max_kernels=12)
    for _ in range(4):
        a.step()
    cb = b.run(4)
    torch.cuda.synchronize()
    for ta, tb in zip(a.theta(), b.theta()):
        assert float((ta - tb).abs().max()) < 1e-6
    ca = [float(c) for c in a.step()]   # one more eager step of a against one more replay of b
    cb = [float(c) for c in b.run(1)]
    np.testing.assert_allclose(cb, ca, rtol=1e-6)
